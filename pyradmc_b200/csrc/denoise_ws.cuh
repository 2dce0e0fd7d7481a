// denoise_ws.cuh — the 3x3x3 convolution as a warp-specialized pipeline on the
// 5th-generation tensor cores, included by denoise.cu after denoise_umma.cuh.
//
// The tile, the halo layout and the descriptors are those of
// conv3d_umma_kernel: output tiles of tz x 16 x 8 voxels (M = 128 rows, one
// per h-w position of a slice), N = cout, the input halo staged as 16-byte rows
// halo[chunk][position][8 channels] so that every tap is a descriptor offset
// into the same planes.  What changes is who moves the data and when:
//   * warp 0 (one lane) is the producer.  It walks the CTA's tiles and, per
//     tile, the channel groups (cg 8-channel chunks each).  A stage is one
//     (tile, group): one TMA tensor copy per chunk of the NDHWC activation, box
//     (8 ch, 10 w, 18 h, tz + 2 d, 1 n), which the copy engine writes in exactly
//     the plane layout above and fills with zeros outside the tensor (the
//     convolution's padding); where the weights do not fit shared memory for
//     the whole launch, one TMA copy per 8-channel weight chunk (box 8 x cout of
//     the [cout][kpad] matrix) joins the stage.  The innermost coordinate of
//     every copy is a multiple of 8 bf16 = 16 bytes.
//   * warp 1 (one lane) issues the tcgen05.mma of each stage into one of two
//     accumulators in tensor memory, commits each stage to release its buffer
//     to the producer and each finished tile to the epilogue.
//   * warps 2-5 drain an accumulator (tcgen05.ld, bias, ReLU, bf16 stores, one
//     output voxel per thread) and release it.
// Resident weights are staged once per block as [group][tap][chunk][cout][8].
// With one channel group and resident weights the MMAs of a slice are issued
// in the order of conv3d_umma_kernel, so the two produce identical bits.
// Every mbarrier wait gives up after kUWaitNs, records the failure in shared
// memory and in g_umma_failures, and every role then leaves its loop; the
// producer waits (bounded) for its copies in flight and the MMA thread for its
// MMAs before the tensor memory is freed.  No multicast anywhere.
#pragma once

#include <cuda.h>

namespace pmd {

constexpr int kWsThreads = 192;  // producer warp, MMA warp, four epilogue warps
constexpr int kWsMaxStages = 4;

struct WsConv {
    ConvShape s;
    int tz;                  // output d-slices per tile
    int tiles_d, tiles_h, tiles_w, n_tiles;
    int cg;                  // 8-channel chunks per stage (channel group)
    int groups;              // stages per tile: cin / 8 / cg
    int stages;              // stage buffers in shared memory
    int streamed;            // 1: weights travel with every stage; 0: resident for the launch
    unsigned plane_bytes;    // stride between halo planes (a box, rounded up to 128 bytes)
    unsigned box_bytes;      // bytes one halo copy writes
    unsigned halo_part;      // cg planes + zeroed slack: offset of a stage's weights
    unsigned stage_bytes;    // stride between stage buffers
    unsigned w_chunks;       // weight chunks of one channel group (cg = 1: with a zero partner)
    unsigned tx_bytes;       // bytes the copy engine writes per stage
    unsigned acc_cols;       // tensor-memory columns of one accumulator: tz * cout
    unsigned tmem_cols;      // allocated: two accumulators, a power of two >= 32
    int ystride;             // channels per voxel of the output tensor
};

// An optional 1x1x1 head fused into the epilogue: out[m] = b + base[m] +
// sum_c w[c] * y[m][c] over the bf16 outputs, which are then not stored.
struct WsHead {
    const float* w = nullptr;     // [cout]; null: no head, y is written
    const float* b = nullptr;     // [1]
    const float* base = nullptr;  // [voxels] or null
    float* out = nullptr;         // [voxels]
};

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, int c4, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(mbar)
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(mbar)
        : "memory");
}

// Bounded wait for the completion of phase `parity`: false once kUWaitNs have
// passed (the shared failure flag is then set) or another role has failed.
__device__ __forceinline__ bool ws_wait(uint32_t mbar, uint32_t parity, volatile int* failed) {
    const unsigned long long start = global_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (*failed) return false;
        if (global_ns() - start > kUWaitNs) {
            *failed = 1;
            return false;
        }
    }
}

__device__ __forceinline__ void ws_tile_origin(const WsConv& p, int tile, int& nb, int& z0, int& y0,
                                               int& x0) {
    int t = tile;
    const int tx = t % p.tiles_w;
    t /= p.tiles_w;
    const int ty = t % p.tiles_h;
    t /= p.tiles_h;
    const int tzi = t % p.tiles_d;
    nb = t / p.tiles_d;
    z0 = tzi * p.tz;
    y0 = ty * kUTY;
    x0 = tx * kUTX;
}

// CG = cg, the 8-channel chunks of a stage.
template <int CG>
__global__ void __launch_bounds__(kWsThreads, 1)
conv3d_ws_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap wmap,
                 const __nv_bfloat16* __restrict__ wt, const float* __restrict__ bias,
                 __nv_bfloat16* __restrict__ y, WsConv p, int relu, WsHead head) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const ConvShape& s = p.s;
    const int N = s.cout;
    const int cpt = s.cin / 8, S = p.stages;
    constexpr int cg = CG;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* stage0 = smem;  // stage b at stage0 + b * stage_bytes
    unsigned char* wres = smem + (size_t)S * p.stage_bytes;  // resident weights (streamed: empty)
    // resident weights: [group][tap][chunk][cout][8], w_chunks per group
    const size_t group_bytes = (size_t)p.w_chunks * N * 16;
    const size_t wres_bytes = p.streamed ? 0 : (size_t)p.groups * group_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(wres + wres_bytes);  // full[S], empty[S], acc_full[2], acc_free[2]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 4);
    volatile int* failed = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t st_s = smem_u32(stage0), bar_s = smem_u32(bars);
    const uint32_t wbase = p.streamed ? st_s + p.halo_part : smem_u32(wres);
    auto full = [&](int b) { return bar_s + 8u * (uint32_t)b; };
    auto empty = [&](int b) { return bar_s + 8u * (uint32_t)(S + b); };
    auto acc_full = [&](int a) { return bar_s + 8u * (uint32_t)(2 * S + a); };
    auto acc_free = [&](int a) { return bar_s + 8u * (uint32_t)(2 * S + 2 + a); };

    // ---- set-up.  The copy engine writes only the boxes and the weight chunks
    // of a stage; the rest of each stage (plane padding, the slack after the
    // planes, with cg = 1 the zero partner of the last tap's weights) is zeroed
    // here once: the cg = 1 tap pairing reads past the last box and multiplies
    // those bytes by the zero weights, so they must be finite.
    for (int b = 0; b < S; ++b) {
        uint32_t* st = reinterpret_cast<uint32_t*>(stage0 + (size_t)b * p.stage_bytes);
        for (int i = tid; i < (int)(p.halo_part / 4); i += blockDim.x) {
            const unsigned byte = 4u * (unsigned)i;
            if (byte >= (unsigned)cg * p.plane_bytes || byte % p.plane_bytes >= p.box_bytes) st[i] = 0u;
        }
        if (p.streamed && cg == 1)
            for (int i = tid; i < N * 4; i += blockDim.x) st[(p.halo_part + 27u * N * 16u) / 4 + i] = 0u;
    }
    if (!p.streamed)
        for (int i = tid; i < p.groups * (int)p.w_chunks * N; i += blockDim.x) {
            const int n = i % N, c = i / N;
            const int g = c / (int)p.w_chunks, jj = c % (int)p.w_chunks;
            const int chunk = (jj / cg) * cpt + g * cg + jj % cg;  // tap * cpt + channel chunk
            const uint4 v = jj < 27 * cg
                                ? *reinterpret_cast<const uint4*>(wt + (long long)n * s.kpad + chunk * 8)
                                : make_uint4(0u, 0u, 0u, 0u);  // the cg = 1 pad partner
            *reinterpret_cast<uint4*>(wres + ((size_t)c * N + n) * 16) = v;
        }
    if (tid == 0) {
        for (int i = 0; i < 2 * S + 2; ++i) mbar_init(bar_s + 8u * i, 1);
        for (int i = 2 * S + 2; i < 2 * S + 4; ++i) mbar_init(bar_s + 8u * i, 128);
        *failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(p.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();  // zeroed bytes and resident weights are read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---- producer ----
        if (lane == 0) {
            int st = 0;  // stages issued
            bool stop = false;
            for (int tile = blockIdx.x; tile < p.n_tiles && !stop; tile += gridDim.x) {
                int nb, z0, y0, x0;
                ws_tile_origin(p, tile, nb, z0, y0, x0);
                for (int g = 0; g < p.groups; ++g) {
                    const int b = st % S, use = st / S;
                    if (use >= 1 && !ws_wait(empty(b), (uint32_t)((use - 1) & 1), failed)) {
                        stop = true;
                        break;
                    }
                    mbar_arrive_expect_tx(full(b), p.tx_bytes);
                    const uint32_t dst = st_s + (uint32_t)b * p.stage_bytes;
                    for (int q = 0; q < cg; ++q)
                        tma_load_5d(dst + (uint32_t)q * p.plane_bytes, &xmap, (g * cg + q) * 8, x0 - 1,
                                    y0 - 1, z0 - 1, nb, full(b));
                    if (p.streamed)
                        for (int tap = 0; tap < 27; ++tap)
                            for (int q = 0; q < cg; ++q)
                                tma_load_2d(dst + p.halo_part + (uint32_t)(tap * cg + q) * N * 16, &wmap,
                                            (tap * cpt + g * cg + q) * 8, 0, full(b));
                    ++st;
                }
            }
            // copies still in flight land before the block can exit
            for (int t = st > S ? st - S : 0; t < st; ++t) mbar_wait(full(t % S), (uint32_t)((t / S) & 1));
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = umma_instr_desc(N);
            int st = 0, last = -1;  // stages consumed; the last one committed
            bool stop = false;
            for (int i = 0, tile = blockIdx.x; tile < p.n_tiles && !stop; ++i, tile += gridDim.x) {
                const int a = i & 1;
                if (i >= 2 && !ws_wait(acc_free(a), (uint32_t)(((i >> 1) & 1) ^ 1), failed)) break;
                tc_fence_after();
                const uint32_t d0 = tmem + (uint32_t)a * p.acc_cols;
                for (int g = 0; g < p.groups; ++g, ++st) {
                    const int b = st % S;
                    if (!ws_wait(full(b), (uint32_t)((st / S) & 1), failed)) {
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t stage = st_s + (uint32_t)b * p.stage_bytes;
                    const uint32_t wg = p.streamed ? stage + p.halo_part
                                                   : wbase + (uint32_t)((size_t)g * group_bytes);
                    umma_issue_taps<CG>(d0, stage, p.plane_bytes, wg, N, p.tz, idesc, g > 0);
                    umma_commit(empty(b));
                    last = st;
                }
                if (!stop) umma_commit(acc_full(a));
            }
            // MMAs still in flight finish before the tensor memory is freed
            if (last >= 0) mbar_wait(empty(last % S), (uint32_t)((last / S) & 1));
        }
    } else {
        // ---- epilogue: one accumulator row (output voxel) per thread ----
        const int quarter = warp & 3;  // the tensor-memory lanes this warp may read
        const int r = quarter * 32 + lane;
        for (int i = 0, tile = blockIdx.x; tile < p.n_tiles; ++i, tile += gridDim.x) {
            const int a = i & 1;
            int ok = lane == 0 ? (ws_wait(acc_full(a), (uint32_t)((i >> 1) & 1), failed) ? 1 : 0) : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);  // the warp leaves or reads together
            if (!ok) break;
            tc_fence_after();
            int nb, z0, y0, x0;
            ws_tile_origin(p, tile, nb, z0, y0, x0);
            const int yg = y0 + r / kUTX, xg = x0 + r % kUTX;
            for (int sl = 0; sl < p.tz; ++sl) {
                const int z = z0 + sl;
                const bool in = z < s.d && yg < s.h && xg < s.w;
                const long long m = (((long long)nb * s.d + (in ? z : 0)) * s.h + (in ? yg : 0)) * s.w +
                                    (in ? xg : 0);
                __nv_bfloat16* out = y + m * p.ystride;
                // the fused head: bias + base + its weights over the stored bf16
                // channel values, in channel order (pmd_head's arithmetic)
                float hacc = 0.0f;
                if (head.w && in) hacc = __ldg(head.b) + (head.base ? head.base[m] : 0.0f);
                for (int c = 0; c < N / 16; ++c) {
                    float v[16];
                    tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)a * p.acc_cols +
                                  (uint32_t)(sl * N + c * 16), v);
                    if (in) {
                        union {
                            uint4 u4[2];
                            __nv_bfloat162 h[8];
                        } pk;
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            float lo = v[2 * e], hi = v[2 * e + 1];
                            if (bias) {
                                lo += bias[c * 16 + 2 * e];
                                hi += bias[c * 16 + 2 * e + 1];
                            }
                            if (relu) {
                                lo = fmaxf(lo, 0.0f);
                                hi = fmaxf(hi, 0.0f);
                            }
                            pk.h[e] = __floats2bfloat162_rn(lo, hi);
                        }
                        if (head.w) {
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                hacc += __ldg(head.w + c * 16 + 2 * e) * __low2float(pk.h[e]);
                                hacc += __ldg(head.w + c * 16 + 2 * e + 1) * __high2float(pk.h[e]);
                            }
                        } else {
                            uint4* o = reinterpret_cast<uint4*>(out + c * 16);
                            o[0] = pk.u4[0];
                            o[1] = pk.u4[1];
                        }
                    }
                }
                if (head.w && in) head.out[m] = hacc;
            }
            tc_fence_before();
            mbar_arrive(acc_free(a));
        }
    }

    tc_fence_before();
    __syncthreads();
    if (tid == 0 && *failed) atomicAdd(&g_umma_failures, 1);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(p.tmem_cols)
                     : "memory");
    }
}

}  // namespace pmd
