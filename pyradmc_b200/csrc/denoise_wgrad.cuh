// denoise_wgrad.cuh — the weight gradient of the 3x3x3 convolution on the
// 5th-generation tensor cores, included by denoise.cu after denoise_ws.cuh.
//
//   dW[co][tap * cin + ci] += sum_m dY[m][co] * X[m + tap][ci]
//   dbias[co]              += sum_m dY[m][co]
//
// Per tap this is a GEMM with M = cout, N = cin and the reduction K running
// over voxels, so both operands are read voxel-major ("MN-major" for the
// tensor cores: 16-byte rows of 8 channels, one row per voxel).  The forward
// kernels' halo layout already is that canonical layout: halo[chunk][pos][8],
// 8 consecutive w positions form one 8 x 16-byte core matrix, the next h row
// (the second 8 voxels of a K = 16 step) sits 160 bytes on (LBO) and the next
// 8-channel chunk one plane on (SBO).  So tap (dz, dy, dx) of output rows
// (y, y + 1) is again one start-address offset into the same halo, as in the
// forward pass, and no im2col copy exists.  The output gradient tile is staged
// as dy[row of 8 voxels][co chunk][8 voxels][8 co] (SBO 128 bytes between co
// chunks, LBO = cout / 8 * 128 between rows).  M is 64 for cout <= 64, else
// 128; the co chunks it reads past cout land on the next rows or the zeroed
// margin and only produce accumulator rows that are never read.
//
// One CTA per SM owns a group of taps (its accumulators, taps x cin fp32
// columns, fill the tensor memory) and a strided share of the tiles; it sums
// over all of them in tensor memory and adds its partial gradient into dW with
// one fp32 atomic per weight at the end.  Roles, as in conv3d_ws_kernel:
//   * warp 0 (one lane): per stage (tile, channel group) one TMA tensor copy
//     per 8-channel chunk of the input halo (box 8 ch x 10 w x 18 h x
//     (tz + 2) d x 1 n, zero fill outside: the padding);
//   * warps 2-5: load the stage's output-gradient tile with 16-byte loads
//     (zeros outside the volume), publish it to the tensor cores
//     (fence.proxy.async) and, in the CTAs of tap group 0, sum the bias
//     gradient from it;
//   * warp 1 (one lane): issues M = 128, N = 8 * chunks, K = 16 MMAs with
//     both operands MN-major, commits each stage back to its producers and,
//     after its last tile, the accumulators to the epilogue.  With cin = 8 the
//     halo operand's 8-channel groups are instead taken 16 bytes apart, i.e.
//     one w position apart: one N = 32 MMA covers the taps dx = 0, 1, 2 of a
//     (dz, dy) row (the fourth group is discarded), a third of the MMAs;
//   * warps 2-5 then read the accumulators (tcgen05.ld, one co row per lane)
//     and add them into dW.
// Every mbarrier wait is bounded (kUWaitNs), records a failure in shared
// memory and in g_umma_failures, and ends every role's loop; the producer and
// the MMA thread wait (bounded) for their copies and MMAs in flight before the
// tensor memory is freed.  No multicast anywhere.
#pragma once

namespace pmd {

constexpr int kWgThreads = 192;

struct WgConv {
    ConvShape s;
    int tz;                  // output d-slices per tile
    int tiles_d, tiles_h, tiles_w, n_tiles;
    int ncg;                 // 8-channel chunks of the halo per stage
    int chunk_groups;        // stages per tile: cin / 8 / ncg
    int n_mma;               // MMA N: 8 * ncg (cin = 8: 32, the three w taps and a discarded fourth)
    int dx_fold;             // cin = 8: one MMA per (dz, dy) covers the three dx taps
    int m64;                 // cout <= 64: M = 64 (accumulator row m in lane m % 16 + 32 (m / 16))
    int n_units;             // accumulator units: 27 taps, or 9 tap rows when dx_fold
    int units;               // units per unit group (one CTA's accumulators)
    int unit_groups;
    int stages;              // stage buffers
    unsigned plane_bytes;    // halo plane stride (a box rounded up to 128 bytes)
    unsigned box_bytes;      // bytes one halo copy writes
    unsigned halo_bytes;     // planes of a stage (ncg = 1: one more, zeroed, for N = 16)
    unsigned dy_lbo;         // bytes between output-gradient rows of 8 voxels: cout / 8 * 128
    unsigned dy_bytes;       // output-gradient rows of a stage + the M = 128 over-read margin
    unsigned stage_bytes;
    unsigned tx_bytes;       // bytes the copy engine writes per stage
    unsigned b_sbo;          // halo operand: bytes between its 8-channel groups (a plane; dx_fold: 16)
    unsigned cols_per_unit;  // accumulator columns of one unit: cin (dx_fold: 32)
    unsigned tmem_cols;      // allocated: a power of two >= units * cols_per_unit
};

__device__ __forceinline__ void wg_tile_origin(const WgConv& p, int tile, int& nb, int& z0, int& y0,
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

// dst[0..3] += (a, b, c, d): one vector reduction at the L2 (dst 16-byte aligned).
__device__ __forceinline__ void red_add_v4(float* dst, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

__device__ __forceinline__ uint32_t wgrad_instr_desc(int n, int m) {
    // as umma_instr_desc with A and B MN-major (bits 15 and 16) and M = m (64 or 128)
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

__global__ void __launch_bounds__(kWgThreads, 1)
conv3d_wgrad_umma_kernel(const __grid_constant__ CUtensorMap xmap,
                         const __nv_bfloat16* __restrict__ g, float* __restrict__ dw,
                         float* __restrict__ dbias, WgConv p) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const ConvShape& s = p.s;
    const int S = p.stages;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cgo = s.cout / 8;  // 16-byte chunks of one output-gradient voxel
    const int unit_group = (int)blockIdx.x % p.unit_groups;
    const int cta_in_group = (int)blockIdx.x / p.unit_groups;
    const int ctas_per_group = (int)gridDim.x / p.unit_groups;
    const int u0 = unit_group * p.units;
    const int units = min(p.units, p.n_units - u0);

    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * p.stage_bytes);
    // full[S] (copy engine), dfull[S] (output-gradient loaders), empty[S], acc_full
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * S + 1);
    volatile int* failed = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t st_s = smem_u32(smem), bar_s = smem_u32(bars);
    auto full = [&](int b) { return bar_s + 8u * (uint32_t)b; };
    auto dfull = [&](int b) { return bar_s + 8u * (uint32_t)(S + b); };
    auto empty = [&](int b) { return bar_s + 8u * (uint32_t)(2 * S + b); };
    const uint32_t acc_full = bar_s + 8u * (uint32_t)(3 * S);

    // ---- set-up: zero every stage once (plane padding, the ncg = 1 partner
    // plane and the output-gradient margin are never written by a copy but
    // are read by the tensor cores; they only reach accumulator rows and
    // columns that are discarded, and zeros keep them finite)
    for (int i = tid; i < (int)((size_t)S * p.stage_bytes / 16); i += blockDim.x)
        reinterpret_cast<uint4*>(smem)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(full(i), 1);
            mbar_init(dfull(i), 4);
            mbar_init(empty(i), 1);
        }
        mbar_init(acc_full, 1);
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
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int my_tiles = cta_in_group < p.n_tiles ? (p.n_tiles - 1 - cta_in_group) / ctas_per_group + 1 : 0;
    const int n_stages = my_tiles * p.chunk_groups;

    if (warp == 0) {
        // ---- producer: the halo planes of each stage ----
        if (lane == 0) {
            int st = 0;
            for (; st < n_stages; ++st) {
                const int b = st % S, use = st / S;
                if (use >= 1 && !ws_wait(empty(b), (uint32_t)((use - 1) & 1), failed)) break;
                const int tile = cta_in_group + (st / p.chunk_groups) * ctas_per_group;
                const int h = st % p.chunk_groups;
                int nb, z0, y0, x0;
                wg_tile_origin(p, tile, nb, z0, y0, x0);
                mbar_arrive_expect_tx(full(b), p.tx_bytes);
                const uint32_t dst = st_s + (uint32_t)b * p.stage_bytes;
                for (int q = 0; q < p.ncg; ++q)
                    tma_load_5d(dst + (uint32_t)q * p.plane_bytes, &xmap, (h * p.ncg + q) * 8, x0 - 1,
                                y0 - 1, z0 - 1, nb, full(b));
            }
            for (int t = st > S ? st - S : 0; t < st; ++t) mbar_wait(full(t % S), (uint32_t)((t / S) & 1));
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = wgrad_instr_desc(p.n_mma, p.m64 ? 64 : 128);
            int st = 0, last = -1;
            for (; st < n_stages; ++st) {
                const int b = st % S;
                const uint32_t par = (uint32_t)((st / S) & 1);
                if (!ws_wait(full(b), par, failed) || !ws_wait(dfull(b), par, failed)) break;
                tc_fence_after();
                const int h = st % p.chunk_groups;
                const bool first_tile = st < p.chunk_groups;
                const uint32_t halo = st_s + (uint32_t)b * p.stage_bytes;
                const uint32_t dyt = halo + p.halo_bytes;
                // descriptors as base + offsets in 16-byte units (the start
                // address field; shared addresses stay below 256 KB, no carry)
                const uint64_t a0 = umma_smem_desc(dyt, p.dy_lbo, 128u);
                const uint64_t b0 = umma_smem_desc(halo, kUHX * 16u, p.b_sbo);
                const uint32_t a_row = p.dy_lbo >> 4;  // one output row of 8 voxels
                for (int t = 0; t < units; ++t) {
                    const uint32_t d = tmem + (uint32_t)t * p.cols_per_unit + (uint32_t)(h * p.ncg * 8);
                    const uint64_t bt = b0 + tap_off16(p.dx_fold ? 3 * (u0 + t) : u0 + t);
                    for (int sl = 0; sl < p.tz; ++sl) {
                        const uint64_t as = a0 + (uint64_t)(sl * kUTY) * a_row;
                        const uint64_t bs = bt + (uint64_t)(sl * kUHY * kUHX);
                        const uint32_t acc0 = (first_tile && sl == 0) ? 0u : 1u;
#pragma unroll
                        for (int r = 0; r < kUTY / 2; ++r)  // K = 16 voxels: output rows 2r, 2r + 1
                            umma_bf16(d, as + (uint64_t)(2 * r) * a_row, bs + (uint64_t)(2 * r * kUHX), idesc,
                                      r == 0 ? acc0 : 1u);
                    }
                }
                umma_commit(empty(b));
                last = st;
            }
            if (st == n_stages && n_stages > 0) umma_commit(acc_full);
            if (last >= 0) mbar_wait(empty(last % S), (uint32_t)((last / S) & 1));
        }
    } else {
        // ---- output-gradient loaders, then the epilogue ----
        const int lt = tid - 64;  // 0..127
        const int quarter = warp & 3;
        const int per_stage = p.tz * kUTY * kUTX * cgo;  // 16-byte chunks of a stage
        // kUTX * cgo divides 128, so this thread always loads the same co chunk
        // (and w position): it sums those 8 channels for the bias gradient
        const int my_c = (lt % (kUTX * cgo)) / kUTX;
        float bsum[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const bool bias_cta = dbias != nullptr && unit_group == 0;
        bool ok = true;
        for (int st = 0; st < n_stages; ++st) {
            const int b = st % S, use = st / S;
            int w_ok = 1;
            if (use >= 1 && lane == 0) w_ok = ws_wait(empty(b), (uint32_t)((use - 1) & 1), failed) ? 1 : 0;
            if (!__shfl_sync(0xffffffffu, w_ok, 0)) {
                ok = false;
                break;
            }
            const int tile = cta_in_group + (st / p.chunk_groups) * ctas_per_group;
            const int h = st % p.chunk_groups;
            int nb, z0, y0, x0;
            wg_tile_origin(p, tile, nb, z0, y0, x0);
            unsigned char* dyt = smem + (size_t)b * p.stage_bytes + p.halo_bytes;
            for (int i = lt; i < per_stage; i += 128) {
                // i -> (row of 8 voxels, co chunk, voxel): consecutive threads
                // write consecutive 16-byte rows of the staged tile
                const int row = i / (kUTX * cgo), rem = i % (kUTX * cgo);
                const int c = rem / kUTX, vx = rem % kUTX;
                const int sl = row / kUTY, vy = row % kUTY;
                const int z = z0 + sl, yy = y0 + vy, xx = x0 + vx;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (z < s.d && yy < s.h && xx < s.w)
                    v = __ldg(reinterpret_cast<const uint4*>(
                        g + ((((long long)nb * s.d + z) * s.h + yy) * s.w + xx) * s.cout + c * 8));
                *reinterpret_cast<uint4*>(dyt + (size_t)row * p.dy_lbo + (size_t)rem * 16) = v;
                if (bias_cta && h == 0) {
                    const __nv_bfloat162* e = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        bsum[2 * k] += __low2float(e[k]);
                        bsum[2 * k + 1] += __high2float(e[k]);
                    }
                }
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(dfull(b));
        }
        if (bias_cta && lt < per_stage)
            for (int k = 0; k < 8; ++k)
                if (bsum[k] != 0.0f) atomicAdd(dbias + my_c * 8 + k, bsum[k]);
        // ---- epilogue: this CTA's partial gradient, one co row per lane ----
        int a_ok = 0;
        if (ok && n_stages > 0 && lane == 0) a_ok = ws_wait(acc_full, 0u, failed) ? 1 : 0;
        a_ok = __shfl_sync(0xffffffffu, a_ok, 0);
        // accumulator row co: lane co of quarter co / 32 (M = 128), lane co % 16
        // of quarter co / 16 (M = 64)
        const int rows = p.m64 ? 16 : 32;
        if (a_ok && quarter * rows < s.cout) {
            tc_fence_after();
            const int co = lane < rows ? quarter * rows + lane : s.cout;
            const unsigned cols = (unsigned)units * p.cols_per_unit;
            for (unsigned c0 = 0; c0 < cols; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + c0, v);
                if (co < s.cout) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        // four columns of one unit (cols_per_unit is a multiple of
                        // 16) -> four consecutive weights, one vector reduction
                        const unsigned col = c0 + (unsigned)j;
                        const int t = (int)(col / p.cols_per_unit), rem = (int)(col % p.cols_per_unit);
                        // the unit's column -> (tap, input channel); dx_fold: 8 columns per dx tap
                        const int tap = p.dx_fold ? 3 * (u0 + t) + rem / 8 : u0 + t;
                        const int ci = p.dx_fold ? rem % 8 : rem;
                        if (p.dx_fold ? rem < 24 : ci < s.cin)
                            red_add_v4(dw + (long long)co * s.kpad + (long long)tap * s.cin + ci, v[j], v[j + 1],
                                       v[j + 2], v[j + 3]);
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (*failed && tid == 0) atomicAdd(&g_umma_failures, 1);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols)
                     : "memory");
    }
}

}  // namespace pmd
