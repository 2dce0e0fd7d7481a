// denoise_umma.cuh — 3x3x3 convolution on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory), included by denoise.cu.
//
// A CTA owns output tiles of tz x 16 x 8 voxels (d x h x w) of one batch
// item, every output channel.  Per tile it stages the input halo
// (tz+2) x 18 x 10 voxels in shared memory as 16-byte rows, one plane per
// 8-channel chunk: halo[q][pos][8], pos = (zz * 18 + yy) * 10 + xx.  Row r of
// the 128-row A operand (output voxel (r / 8, r % 8) of an h-w slice) at tap
// (dz, dy, dx) and chunk q then sits at halo + q * plane + pos(s + dz, r / 8 +
// dy, r % 8 + dx) * 16: 8-row core matrices of consecutive 16-byte rows, the
// next 8 rows (next h) 160 bytes on.  That is the K-major no-swizzle canonical
// layout of a UMMA shared-memory descriptor (start address, LBO = distance
// of the second 8-element K half, SBO = 160 B), so every tap is one
// descriptor offset into the same halo and no im2col copy exists.  Weights
// sit in shared memory as w[chunk][cout][8] (the B operand, SBO = 128 B,
// LBO = cout * 16 B).  One thread issues the MMAs (M = 128, N = cout,
// K = 16 per instruction); tcgen05.commit arrives on an mbarrier that every
// thread waits on, with a time limit that records a failure instead of
// hanging.  The epilogue reads the fp32 accumulators from tensor memory
// (tcgen05.ld, one row per thread), adds the bias, applies ReLU and stores
// bf16.  With cin = 8 a K step pairs two taps: the second half's LBO is the
// distance between the two taps' rows, and the last tap pairs with a zero
// weight chunk.
#pragma once

namespace pmd {

constexpr int kUTY = 16, kUTX = 8;             // output tile: 16 h-rows x 8 w-columns = M
constexpr int kUHY = kUTY + 2, kUHX = kUTX + 2;  // halo rows / columns
constexpr int kUSlack = 256;                   // zeroed bytes after the halo (cin = 8 pairing)
constexpr unsigned long long kUWaitNs = 1000000000ull;  // give up an mbarrier wait after 1 s

__device__ int g_umma_failures = 0;

struct UmmaConv {
    ConvShape s;
    int tz;             // output d-slices per tile
    int taps_per_pass;  // taps whose weights are staged at once
    int passes;
    int tiles_d, tiles_h, tiles_w, n_tiles;
    unsigned halo_bytes, plane_bytes;
    unsigned w_chunks;  // weight chunks staged per pass (incl. the cin = 8 pad partner)
    unsigned k_steps;   // K steps (16-wide) per pass: descriptor table entries
    unsigned tmem_cols;
    int ystride;        // channels per voxel of the output tensor (>= cout: a channel slice)
};

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    // start address, leading and stride byte offsets in 16-byte units; version 1
    // (bits 46-47); base offset 0, legacy LBO mode, no swizzle (bits 61-63 = 0).
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t umma_instr_desc(int n) {
    // fp32 accumulate (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1), both
    // K-major, N >> 3 at bits 17-22, M >> 4 = 8 at bits 24-28.
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | (8u << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Poll the mbarrier phase until it completes or kUWaitNs have passed (then
// false); each poll may suspend the thread for a short while.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    const unsigned long long start = global_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
        if (global_ns() - start > kUWaitNs) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of tap t's first halo row relative to the slice's origin.
__device__ __forceinline__ uint32_t tap_offset(int t) {
    return (uint32_t)(((t / 9) * kUHY * kUHX + ((t / 3) % 3) * kUHX + t % 3) * 16);
}

// Tap t's first halo row relative to the slice's origin, in 16-byte units.
__host__ __device__ constexpr uint32_t tap_off16(int t) {
    return (uint32_t)((t / 9) * kUHY * kUHX + ((t / 3) % 3) * kUHX + t % 3);
}

// Issues the MMAs of all 27 taps over CG 8-channel chunks for the tz slices of
// a tile: A from the halo planes at a_addr (plane_bytes apart), B from the
// weight chunks [tap * CG + q][N][8] at b_addr, slice sl into accumulator
// columns d0 + sl * N, in the order slice, tap, chunk pair.  Every descriptor is
// the slice's base descriptor plus an offset fixed at compile time within a
// group of 9 taps (7 tap pairs for CG = 1), so the issuing thread runs no loads
// and little arithmetic between MMAs (a thread issuing from a descriptor table
// in shared memory measured ~50-120 cycles per MMA, well above the tensor
// cores' ~35 for M = 128, N <= 32).  The tap loop stays a loop of such groups
// and the slice loop is not unrolled: with the 14 or 27 MMAs of a slice
// unrolled in full for CG = 1 and 2, this build computed wrong sums (tested
// against the oracle), while the grouped form is exact for every CG.  With CG = 1 a K step
// pairs two taps: the second half's LBO is the distance between their rows and
// the last tap pairs with a zero weight chunk.  accumulate: whether the first
// K step adds to the accumulator (a later channel group of the same tile).
template <int CG>
__device__ __forceinline__ void umma_issue_taps(uint32_t d0, uint32_t a_addr, uint32_t plane_bytes,
                                                uint32_t b_addr, int N, int tz, uint32_t idesc,
                                                bool accumulate) {
    constexpr uint64_t slice16 = (uint64_t)(kUHY * kUHX);
    const uint64_t a0 = umma_smem_desc(a_addr, CG == 1 ? 0u : plane_bytes, kUHX * 16);
    const uint64_t b0 = umma_smem_desc(b_addr, (uint32_t)N * 16, 128);
    const uint64_t plane16 = plane_bytes >> 4;
#pragma unroll 1
    for (int sl = 0; sl < tz; ++sl) {
        const uint32_t d = d0 + (uint32_t)(sl * N);
        const uint64_t as = a0 + slice16 * (uint64_t)sl;
        if constexpr (CG == 1) {
#pragma unroll 7
            for (int tap = 0; tap < 27; tap += 2) {
                const uint64_t lbo16 = tap + 1 < 27 ? tap_off16(tap + 1) - tap_off16(tap) : 1u;
                umma_bf16(d, as + tap_off16(tap) + (lbo16 << 16), b0 + (uint64_t)(tap * N), idesc,
                          (accumulate || tap > 0) ? 1u : 0u);
            }
        } else {
#pragma unroll 9
            for (int tap = 0; tap < 27; ++tap)
#pragma unroll
                for (int q = 0; q < CG; q += 2)
                    umma_bf16(d, as + tap_off16(tap) + plane16 * (uint64_t)q,
                              b0 + (uint64_t)((tap * CG + q) * N), idesc,
                              (accumulate || tap > 0 || q > 0) ? 1u : 0u);
        }
    }
}

// CPT = cin / 8, the 8-channel chunks (halo planes) per tap.
template <int CPT>
__global__ void __launch_bounds__(128, 4)
conv3d_umma_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wt,
                   const float* __restrict__ bias, __nv_bfloat16* __restrict__ y, UmmaConv u,
                   int relu) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const ConvShape& s = u.s;
    const int N = s.cout;
    constexpr int cpt = CPT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* halo = smem;
    unsigned char* wbuf = smem + u.halo_bytes + kUSlack;
    // per-pass descriptor table: A (slice 0) and B descriptor of every K step
    uint64_t* dtab = reinterpret_cast<uint64_t*>(wbuf + (size_t)u.w_chunks * N * 16);
    uint64_t* mbar_p = dtab + 2 * u.k_steps;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar_p + 1);
    const uint32_t halo_s = smem_u32(halo), w_s = smem_u32(wbuf), mbar = smem_u32(mbar_p);

    for (int i = tid; i < kUSlack / 4; i += blockDim.x)
        reinterpret_cast<uint32_t*>(halo + u.halo_bytes)[i] = 0u;
    if (tid == 0) mbar_init(mbar, 1);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(u.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_instr_desc(N);
    const int npos = (u.tz + 2) * kUHY * kUHX;
    uint32_t phase = 0;
    int failed = 0;
    bool weights_resident = false;

    for (int tile = blockIdx.x; tile < u.n_tiles && !failed; tile += gridDim.x) {
        int t = tile;
        const int tx = t % u.tiles_w;
        t /= u.tiles_w;
        const int ty = t % u.tiles_h;
        t /= u.tiles_h;
        const int tzi = t % u.tiles_d;
        const int nb = t / u.tiles_d;
        const int z0 = tzi * u.tz, y0 = ty * kUTY, x0 = tx * kUTX;

        for (int pass = 0; pass < u.passes && !failed; ++pass) {
            if (pass == 0) {
                // halo: index -> (8 consecutive positions, chunk, position block), so a
                // warp writes whole 128-byte runs of one plane
                const int total = ((npos + 7) / 8) * 8 * cpt;
                for (int i = tid; i < total; i += blockDim.x) {
                    const int pos = (i / (8 * cpt)) * 8 + (i & 7);
                    const int q = (i >> 3) % cpt;
                    if (pos >= npos) continue;
                    const int xx = pos % kUHX, r = pos / kUHX;
                    const int yy = r % kUHY, zz = r / kUHY;
                    const int z = z0 + zz - 1, yg = y0 + yy - 1, xg = x0 + xx - 1;
                    const bool in = (unsigned)z < (unsigned)s.d && (unsigned)yg < (unsigned)s.h &&
                                    (unsigned)xg < (unsigned)s.w;
                    const __nv_bfloat16* src =
                        in ? x + ((((long long)nb * s.d + z) * s.h + yg) * s.w + xg) * s.cin + q * 8 : x;
                    cp_async16(halo + (size_t)q * u.plane_bytes + (size_t)pos * 16, src, in);
                }
            }
            const int t0 = pass * u.taps_per_pass;
            const int t1 = min(27, t0 + u.taps_per_pass);
            const int j0 = t0 * cpt;
            const int j1 = t1 * cpt;
            const int k_begin = j0 / 2, k_end = (j1 + 1) / 2;
            if (u.passes > 1 || !weights_resident) {
                const int n_chunks = (int)u.w_chunks < (j1 - j0 + (j1 - j0) % 2) ? (int)u.w_chunks
                                                                               : (j1 - j0 + (j1 - j0) % 2);
                for (int i = tid; i < n_chunks * N; i += blockDim.x) {
                    const int n = i % N, jj = i / N;
                    cp_async16(wbuf + ((size_t)jj * N + n) * 16,
                               wt + (long long)n * s.kpad + (long long)(j0 + jj) * 8, true);
                }
                for (int k = k_begin + tid; k < k_end; k += blockDim.x) {
                    const int j = 2 * k;
                    const int tap = j / cpt, q = j % cpt;
                    const uint32_t a_addr = halo_s + (uint32_t)q * u.plane_bytes + tap_offset(tap);
                    uint32_t a_lbo = u.plane_bytes;
                    if (cpt == 1) a_lbo = tap + 1 < 27 ? tap_offset(tap + 1) - tap_offset(tap) : 16u;
                    dtab[2 * (k - k_begin)] = umma_smem_desc(a_addr, a_lbo, kUHX * 16);
                    dtab[2 * (k - k_begin) + 1] =
                        umma_smem_desc(w_s + (uint32_t)(j - j0) * N * 16, N * 16, 128);
                }
                weights_resident = true;
            }
            cp_async_commit();
            cp_async_wait<0>();
            fence_async_smem();
            __syncthreads();
            if (tid == 0 && u.passes == 1) {
                tc_fence_after();
                umma_issue_taps<CPT>(tmem, halo_s, u.plane_bytes, w_s, N, u.tz, idesc, false);
                umma_commit(mbar);
            } else if (tid == 0) {
                tc_fence_after();
                const int n_k = k_end - k_begin;
                // slice sl reads the halo kUHY * kUHX rows further: add to the start-address field
                constexpr uint64_t slice_inc = (uint64_t)(kUHY * kUHX * 16) >> 4;
                for (int sl = 0; sl < u.tz; ++sl) {
                    const uint32_t d_tmem = tmem + (uint32_t)(sl * N);
                    for (int k = 0; k < n_k; ++k)
                        umma_bf16(d_tmem, dtab[2 * k] + slice_inc * (uint64_t)sl, dtab[2 * k + 1],
                                  idesc, (pass > 0 || k > 0) ? 1u : 0u);
                }
                umma_commit(mbar);
            }
            const int ok = mbar_wait(mbar, phase) ? 1 : 0;
            phase ^= 1u;
            failed = __syncthreads_or(!ok);
        }
        if (failed) break;

        // epilogue: one accumulator row (output voxel) per thread
        tc_fence_after();
        const int r = warp * 32 + lane;
        const int yg = y0 + r / kUTX, xg = x0 + r % kUTX;
        for (int sl = 0; sl < u.tz; ++sl) {
            const int z = z0 + sl;
            const bool ok = z < s.d && yg < s.h && xg < s.w;
            __nv_bfloat16* out = y + ((((long long)nb * s.d + (ok ? z : 0)) * s.h + (ok ? yg : 0)) * s.w +
                                      (ok ? xg : 0)) * u.ystride;
            for (int c = 0; c < N / 16; ++c) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(sl * N + c * 16), v);
                if (ok) {
                    union {
                        uint4 u4[2];
                        __nv_bfloat162 h[8];
                    } pk;
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        float a = v[2 * e], b = v[2 * e + 1];
                        if (bias) {
                            a += bias[c * 16 + 2 * e];
                            b += bias[c * 16 + 2 * e + 1];
                        }
                        if (relu) {
                            a = fmaxf(a, 0.0f);
                            b = fmaxf(b, 0.0f);
                        }
                        pk.h[e] = __floats2bfloat162_rn(a, b);
                    }
                    uint4* o = reinterpret_cast<uint4*>(out + c * 16);
                    o[0] = pk.u4[0];
                    o[1] = pk.u4[1];
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }

    if (failed) {
        if (tid == 0) atomicAdd(&g_umma_failures, 1);
        mbar_wait(mbar, phase ^ 1u);  // one more bounded wait for MMAs still in flight
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(u.tmem_cols)
                     : "memory");
    }
}

// ---- pipelined variant ---------------------------------------------------------
// The same tile, halo layout, descriptors and epilogue, with two halo buffers
// (each followed by its own zeroed slack) and two accumulators in tensor
// memory: while the MMAs of tile i run, the copies of tile i+1's halo are in
// flight and the epilogue of tile i-1 reads the other accumulator.  Only warp
// 0 polls the mbarrier; the other warps wait at the block barrier.  Needs the
// weights resident (one pass) and 2 * tz * cout <= 512 tensor-memory columns.

__device__ __forceinline__ void umma_tile_origin(const UmmaConv& u, int tile, int& nb, int& z0,
                                                 int& y0, int& x0) {
    int t = tile;
    const int tx = t % u.tiles_w;
    t /= u.tiles_w;
    const int ty = t % u.tiles_h;
    t /= u.tiles_h;
    const int tzi = t % u.tiles_d;
    nb = t / u.tiles_d;
    z0 = tzi * u.tz;
    y0 = ty * kUTY;
    x0 = tx * kUTX;
}

template <int CPT>
__device__ __forceinline__ void umma_load_halo(const __nv_bfloat16* __restrict__ x, const UmmaConv& u,
                                               int tile, unsigned char* buf, int tid) {
    const ConvShape& s = u.s;
    int nb, z0, y0, x0;
    umma_tile_origin(u, tile, nb, z0, y0, x0);
    const int npos = (u.tz + 2) * kUHY * kUHX;
    const int total = ((npos + 7) / 8) * 8 * CPT;
    for (int i = tid; i < total; i += blockDim.x) {
        const int pos = (i / (8 * CPT)) * 8 + (i & 7);
        const int q = (i >> 3) % CPT;
        if (pos >= npos) continue;
        const int xx = pos % kUHX, r = pos / kUHX;
        const int yy = r % kUHY, zz = r / kUHY;
        const int z = z0 + zz - 1, yg = y0 + yy - 1, xg = x0 + xx - 1;
        const bool in = (unsigned)z < (unsigned)s.d && (unsigned)yg < (unsigned)s.h &&
                        (unsigned)xg < (unsigned)s.w;
        const __nv_bfloat16* src =
            in ? x + ((((long long)nb * s.d + z) * s.h + yg) * s.w + xg) * s.cin + q * 8 : x;
        cp_async16(buf + (size_t)q * u.plane_bytes + (size_t)pos * 16, src, in);
    }
}

// One accumulator row (output voxel) per thread: bias, ReLU, bf16 store.
__device__ __forceinline__ void umma_epilogue(const UmmaConv& u, uint32_t acc, int tile,
                                              const float* __restrict__ bias,
                                              __nv_bfloat16* __restrict__ y, int relu, int warp,
                                              int lane) {
    const ConvShape& s = u.s;
    const int N = s.cout;
    int nb, z0, y0, x0;
    umma_tile_origin(u, tile, nb, z0, y0, x0);
    const int r = warp * 32 + lane;
    const int yg = y0 + r / kUTX, xg = x0 + r % kUTX;
    for (int sl = 0; sl < u.tz; ++sl) {
        const int z = z0 + sl;
        const bool ok = z < s.d && yg < s.h && xg < s.w;
        __nv_bfloat16* out =
            y + ((((long long)nb * s.d + (ok ? z : 0)) * s.h + (ok ? yg : 0)) * s.w + (ok ? xg : 0)) *
                    u.ystride;
        for (int c = 0; c < N / 16; ++c) {
            float v[16];
            tmem_ld16(acc + ((uint32_t)(warp * 32) << 16) + (uint32_t)(sl * N + c * 16), v);
            if (ok) {
                union {
                    uint4 u4[2];
                    __nv_bfloat162 h[8];
                } pk;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    float a = v[2 * e], b = v[2 * e + 1];
                    if (bias) {
                        a += bias[c * 16 + 2 * e];
                        b += bias[c * 16 + 2 * e + 1];
                    }
                    if (relu) {
                        a = fmaxf(a, 0.0f);
                        b = fmaxf(b, 0.0f);
                    }
                    pk.h[e] = __floats2bfloat162_rn(a, b);
                }
                uint4* o = reinterpret_cast<uint4*>(out + c * 16);
                o[0] = pk.u4[0];
                o[1] = pk.u4[1];
            }
        }
    }
}

template <int CPT>
__global__ void __launch_bounds__(128, 4)
conv3d_umma_pipe_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wt,
                        const float* __restrict__ bias, __nv_bfloat16* __restrict__ y, UmmaConv u,
                        int relu) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const ConvShape& s = u.s;
    const int N = s.cout;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned buf_stride = u.halo_bytes + kUSlack;  // halo + its zeroed slack
    unsigned char* halo0 = smem;
    unsigned char* wbuf = smem + 2 * buf_stride;
    uint64_t* dtab = reinterpret_cast<uint64_t*>(wbuf + (size_t)u.w_chunks * N * 16);
    uint64_t* mbar_p = dtab + 2 * u.k_steps;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar_p + 1);
    const uint32_t halo_s = smem_u32(halo0), w_s = smem_u32(wbuf), mbar = smem_u32(mbar_p);

    for (int b = 0; b < 2; ++b)
        for (int i = tid; i < kUSlack / 4; i += blockDim.x)
            reinterpret_cast<uint32_t*>(halo0 + b * buf_stride + u.halo_bytes)[i] = 0u;
    if (tid == 0) mbar_init(mbar, 1);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(u.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_instr_desc(N);
    const uint32_t acc_cols = (uint32_t)(u.tz * N);

    // resident weights and the descriptor table (A relative to buffer 0)
    const int n_chunks = (int)u.w_chunks;
    for (int i = tid; i < n_chunks * N; i += blockDim.x) {
        const int n = i % N, jj = i / N;
        cp_async16(wbuf + ((size_t)jj * N + n) * 16, wt + (long long)n * s.kpad + (long long)jj * 8, true);
    }
    if ((int)blockIdx.x < u.n_tiles) umma_load_halo<CPT>(x, u, blockIdx.x, halo0, tid);
    cp_async_commit();

    uint32_t phase = 0;
    int failed = 0, i = 0, prev = -1;
    for (int tile = blockIdx.x; tile < u.n_tiles; tile += gridDim.x, ++i) {
        const int b = i & 1;
        // this tile's halo (and, first time, the weights and table) has landed
        cp_async_wait<0>();
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            umma_issue_taps<CPT>(tmem + (uint32_t)b * acc_cols, halo_s + (uint32_t)b * buf_stride,
                                 u.plane_bytes, w_s, N, u.tz, idesc, false);
            umma_commit(mbar);
        }
        // the next tile's halo into the other buffer (its last reader, the MMAs
        // of the previous tile, completed before the previous wait returned)
        const int next = tile + gridDim.x;
        if (next < u.n_tiles) umma_load_halo<CPT>(x, u, next, halo0 + (b ^ 1) * buf_stride, tid);
        cp_async_commit();
        // the previous tile's epilogue from the other accumulator
        if (prev >= 0) {
            tc_fence_after();
            umma_epilogue(u, tmem + (uint32_t)(b ^ 1) * acc_cols, prev, bias, y, relu, warp, lane);
        }
        const int ok = warp == 0 ? (mbar_wait(mbar, phase) ? 1 : 0) : 1;
        phase ^= 1u;
        tc_fence_before();
        failed = __syncthreads_or(!ok);
        if (failed) break;
        prev = tile;
    }
    if (!failed && prev >= 0) {
        tc_fence_after();
        umma_epilogue(u, tmem + (uint32_t)((i - 1) & 1) * acc_cols, prev, bias, y, relu, warp, lane);
    }
    cp_async_wait<0>();
    if (failed) {
        if (tid == 0) atomicAdd(&g_umma_failures, 1);
        if (warp == 0) mbar_wait(mbar, phase ^ 1u);  // one more bounded wait for MMAs in flight
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(u.tmem_cols)
                     : "memory");
    }
}

}  // namespace pmd
