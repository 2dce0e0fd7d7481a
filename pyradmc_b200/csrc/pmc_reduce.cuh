// pmc_reduce.cuh — batch fold, finalize and Dij truncation/compaction.
//
// These are HBM-streaming kernels over the [columns][voxels] maps; the
// engine's fold, finalize and truncation visit only the 32-byte sectors that
// deposits touched (sector bitmaps below).  Every
// float64 operation is written with an explicit round-to-nearest intrinsic, so
// nothing is contracted into an FMA: the results equal, bit for bit, the numpy
// scorers they restate —
//   fold      BatchedBeamletScorer.end_batch   scoring/dij.py:155-174
//             (BatchedDoseScorer.end_batch     scoring/dose.py:169-186)
//   finalize  BatchedBeamletScorer.finalize    scoring/dij.py:176-191
//   truncate  DijAssembler.add_block           scoring/dij.py:351-366
// The compaction's prefix sum runs on the device (the Warp engine read the
// per-chunk counts back and scanned them with numpy, engine.py:1517-1525).
#pragma once

#include "pmc_common.cuh"

namespace pmc {

constexpr int kReduceThreads = 256;
constexpr int kTileVoxels = 4096;  // truncation tile: one block per (column, tile)

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ bool keep_entry(double m, double threshold) {
    return m >= threshold && m > 0.0;
}

// ---- sector bitmaps ----------------------------------------------------------------
// The engine's dense maps (int64 quanta, float64 sums) are laid out
// [column][stride] with the column stride a multiple of kTileVoxels, so that
// entry e of the map belongs to the 32-byte sector e >> 2 and to bit
// (e >> 2) & 31 of bitmap word e >> 7 (128 entries per word, 32 words per
// truncation tile).  Every atomic deposit also ORs its sector's bit into the
// `dirty` bitmap; the fold visits only dirty sectors, clears their bits and
// records them in the `touched` bitmap (every sector any batch ever scored).
// The sums are never cleared in bulk: a sector's first fold writes all four of
// its entries (d or +0.0), and finalize / truncation read touched sectors
// only.  0.0 + d == d, so a first write equals the reference's s += d.
constexpr int kSectorEntries = 4;
constexpr int kWordEntries = 128;
static_assert(kTileVoxels == 32 * kWordEntries, "one bitmap word per lane of a tile's warp");

__device__ __forceinline__ void mark_dirty(unsigned int* dirty, long long flat) {
    atomicOr(dirty + (flat >> 7), 1u << ((unsigned)(flat >> 2) & 31u));
}

// One warp holds the 32 bitmap words of a tile (word j in lane j); lane order
// then bit order is ascending sector order.  `incl` is the warp's inclusive
// scan of the words' popcounts.  Returns the lane whose word holds set bit
// number k (of the whole tile) and that bit's position; every lane must call
// it (it shuffles), and the result is meaningless for k >= the tile's total.
__device__ __forceinline__ int nth_set_sector(unsigned int w, int incl, int k, int& bit) {
    int j = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const int v = __shfl_sync(0xffffffffu, incl, j + step - 1);
        if (v <= k) j += step;
    }
    const unsigned int wj = __shfl_sync(0xffffffffu, w, j);
    const int before = __shfl_sync(0xffffffffu, incl, j) - __popc(wj);
    bit = (int)__fns(wj, 0u, k - before + 1);
    return j;
}

__device__ __forceinline__ int warp_inclusive_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += y;
    }
    return v;
}

// Fold one batch's quanta into the running sums and consume them (reset the
// folded entries): d = q * 1e-9 / (mass * n), s1 += d, s2 += d^2
// (kernels.py:804-852).  One warp per (column, tile), dirty sectors only.
__global__ void __launch_bounds__(kReduceThreads)
fold_sparse_kernel(unsigned long long* __restrict__ edep, const double* __restrict__ mass,
                   const double* __restrict__ col_nhist, long long n_vox, long long stride,
                   int tiles_per_col, long long n_tiles, double* __restrict__ s1,
                   double* __restrict__ s2, unsigned int* __restrict__ dirty,
                   unsigned int* __restrict__ touched, unsigned long long* __restrict__ total_q) {
    const int lane = threadIdx.x & 31;
    const long long t = (long long)blockIdx.x * (kReduceThreads / 32) + (threadIdx.x >> 5);
    if (t >= n_tiles) return;  // warp-uniform
    const long long widx = t * 32 + lane;
    const unsigned int w = dirty[widx];
    if (__ballot_sync(0xffffffffu, w != 0u) == 0u) return;
    const unsigned int tw = touched[widx];
    const int incl = warp_inclusive_scan(__popc(w));
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const long long col = t / tiles_per_col;
    const long long tile_v0 = (t - col * tiles_per_col) * (long long)kTileVoxels;
    const double nh = col_nhist[col];
    unsigned long long* q_col = edep + col * stride;
    double* a = s1 + col * stride;
    double* b = s2 + col * stride;
    unsigned long long local = 0;
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int bit;
        const int j = nth_set_sector(w, incl, k, bit);
        const unsigned int twj = __shfl_sync(0xffffffffu, tw, j);
        if (k >= total) continue;
        const bool first = ((twj >> bit) & 1u) == 0u;
        const long long v0 = tile_v0 + (long long)j * kWordEntries + bit * kSectorEntries;
#pragma unroll
        for (int e = 0; e < kSectorEntries; ++e) {
            const long long v = v0 + e;
            if (v >= n_vox) break;
            const unsigned long long q = q_col[v];
            if (q != 0ull) {
                q_col[v] = 0ull;
                const double m = mass[v];
                double d = 0.0;
                if (m > 0.0) {
                    const double energy = __dmul_rn((double)(long long)q, kQuantum);
                    d = __ddiv_rn(energy, __dmul_rn(m, nh));
                }
                if (first) {
                    a[v] = d;
                    b[v] = __dmul_rn(d, d);
                } else {
                    a[v] = __dadd_rn(a[v], d);
                    b[v] = __dadd_rn(b[v], __dmul_rn(d, d));
                }
                local += q;
            } else if (first) {
                a[v] = 0.0;
                b[v] = 0.0;
            }
        }
    }
    if (w != 0u) {
        dirty[widx] = 0u;
        touched[widx] = tw | w;
    }
    local = warp_sum_u64(local);
    if (lane == 0 && local) atomicAdd(total_q, local);
}

// mean = S1/n, sigma = sqrt(max(0, S2/n - mean^2) * n / (n - 1) / n), written in
// place over the touched sectors; the column maximum of the mean rides along
// (one atomic per warp).  One warp per (column, tile).
__global__ void __launch_bounds__(kReduceThreads)
finalize_sparse_kernel(double* __restrict__ s1, double* __restrict__ s2, long long n_vox,
                       long long stride, int tiles_per_col, long long n_tiles, int n_batches,
                       const unsigned int* __restrict__ touched,
                       unsigned long long* __restrict__ col_max_bits) {
    const int lane = threadIdx.x & 31;
    const long long t = (long long)blockIdx.x * (kReduceThreads / 32) + (threadIdx.x >> 5);
    if (t >= n_tiles) return;
    const unsigned int w = touched[t * 32 + lane];
    if (__ballot_sync(0xffffffffu, w != 0u) == 0u) return;
    const int incl = warp_inclusive_scan(__popc(w));
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const long long col = t / tiles_per_col;
    const long long tile_v0 = (t - col * tiles_per_col) * (long long)kTileVoxels;
    double* a = s1 + col * stride;
    double* b = s2 + col * stride;
    const double n = (double)n_batches;
    unsigned long long best = 0ull;
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int bit;
        const int j = nth_set_sector(w, incl, k, bit);
        if (k >= total) continue;
        const long long v0 = tile_v0 + (long long)j * kWordEntries + bit * kSectorEntries;
#pragma unroll
        for (int e = 0; e < kSectorEntries; ++e) {
            const long long v = v0 + e;
            if (v >= n_vox) break;
            const double x = a[v];
            const double y = b[v];
            if (x == 0.0 && y == 0.0) continue;  // mean and sigma are already +0.0
            const double mean = __ddiv_rn(x, n);
            double sigma = 0.0;
            if (n_batches > 1) {
                double var = __dsub_rn(__ddiv_rn(y, n), __dmul_rn(mean, mean));
                var = var > 0.0 ? var : 0.0;
                var = __ddiv_rn(__dmul_rn(var, n), n - 1.0);
                sigma = __dsqrt_rn(__ddiv_rn(var, n));
            }
            a[v] = mean;
            b[v] = sigma;
            const unsigned long long bits = (unsigned long long)__double_as_longlong(mean);
            best = bits > best ? bits : best;  // mean >= 0: bit order is value order
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
    }
    if (lane == 0 && best) atomicMax(col_max_bits + col, best);
}

// Kept entries of the touched sectors of one (column, tile); one warp each.
__global__ void __launch_bounds__(kReduceThreads)
count_kept_sparse_kernel(const double* __restrict__ mean, long long n_vox, long long stride,
                         int tiles_per_col, long long n_tiles, double truncation,
                         const unsigned long long* __restrict__ col_max_bits,
                         const unsigned int* __restrict__ touched,
                         unsigned int* __restrict__ tile_counts) {
    const int lane = threadIdx.x & 31;
    const long long t = (long long)blockIdx.x * (kReduceThreads / 32) + (threadIdx.x >> 5);
    if (t >= n_tiles) return;
    const unsigned int w = touched[t * 32 + lane];
    unsigned int c = 0;
    if (__ballot_sync(0xffffffffu, w != 0u) != 0u) {
        const int incl = warp_inclusive_scan(__popc(w));
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        const long long col = t / tiles_per_col;
        const long long tile_v0 = (t - col * tiles_per_col) * (long long)kTileVoxels;
        const double thr = __dmul_rn(truncation, __longlong_as_double((long long)col_max_bits[col]));
        const double* a = mean + col * stride;
        for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + lane;
            int bit;
            const int j = nth_set_sector(w, incl, k, bit);
            if (k >= total) continue;
            const long long v0 = tile_v0 + (long long)j * kWordEntries + bit * kSectorEntries;
#pragma unroll
            for (int e = 0; e < kSectorEntries; ++e) {
                const long long v = v0 + e;
                if (v < n_vox) c += keep_entry(a[v], thr);
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if (lane == 0) tile_counts[t] = c;
}

// Write the kept entries of one (column, tile) at the tile's CSC offset, in
// ascending voxel order (sector order, then entry order): the order
// np.flatnonzero gives on the host.  One warp each.
__global__ void __launch_bounds__(kReduceThreads)
compact_sparse_kernel(const double* __restrict__ mean, const double* __restrict__ sigma,
                      long long n_vox, long long stride, int tiles_per_col, long long n_tiles,
                      double truncation, const unsigned long long* __restrict__ col_max_bits,
                      const unsigned int* __restrict__ touched,
                      const unsigned long long* __restrict__ tile_offsets,
                      long long* __restrict__ out_idx, double* __restrict__ out_dose,
                      double* __restrict__ out_sigma) {
    const int lane = threadIdx.x & 31;
    const long long t = (long long)blockIdx.x * (kReduceThreads / 32) + (threadIdx.x >> 5);
    if (t >= n_tiles) return;
    const unsigned int w = touched[t * 32 + lane];
    if (__ballot_sync(0xffffffffu, w != 0u) == 0u) return;
    const int incl = warp_inclusive_scan(__popc(w));
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const long long col = t / tiles_per_col;
    const long long tile_v0 = (t - col * tiles_per_col) * (long long)kTileVoxels;
    const double thr = __dmul_rn(truncation, __longlong_as_double((long long)col_max_bits[col]));
    const double* a = mean + col * stride;
    const double* b = sigma + col * stride;
    unsigned long long cursor = tile_offsets[t];
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int bit;
        const int j = nth_set_sector(w, incl, k, bit);
        const long long v0 = tile_v0 + (long long)j * kWordEntries + bit * kSectorEntries;
        double m[kSectorEntries];
        unsigned int keep = 0u;
#pragma unroll
        for (int e = 0; e < kSectorEntries; ++e) {
            const long long v = v0 + e;
            m[e] = (k < total && v < n_vox) ? a[v] : 0.0;
            if (k < total && v < n_vox && keep_entry(m[e], thr)) keep |= 1u << e;
        }
        const int n_keep = __popc(keep);
        const int end = warp_inclusive_scan(n_keep);
        unsigned long long pos = cursor + (unsigned long long)(end - n_keep);
#pragma unroll
        for (int e = 0; e < kSectorEntries; ++e) {
            if (keep & (1u << e)) {
                out_idx[pos] = v0 + e;
                out_dose[pos] = m[e];
                out_sigma[pos] = b[v0 + e];
                ++pos;
            }
        }
        cursor += (unsigned long long)__shfl_sync(0xffffffffu, end, 31);
    }
}

// Set every word of a bitmap (the dense entry points mark every sector).
__global__ void fill_u32_kernel(unsigned int* p, long long n, unsigned int v) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

// Column maxima of an already finalized mean map with columns `stride`
// entries apart (grid: x = tiles, y = column).
__global__ void __launch_bounds__(kReduceThreads)
colmax_kernel(const double* __restrict__ mean, long long n_vox, long long stride,
              unsigned long long* __restrict__ col_max_bits) {
    const long long col = blockIdx.y;
    const long long start = (long long)blockIdx.x * kTileVoxels;
    const long long stop = min(start + (long long)kTileVoxels, n_vox);
    const double* a = mean + col * stride;
    unsigned long long best = 0ull;
    for (long long v = start + threadIdx.x; v < stop; v += blockDim.x) {
        const double m = a[v];
        if (m > 0.0) {
            const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
            best = bits > best ? bits : best;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(col_max_bits + col, best);
}

// Count the kept entries of one (column, tile).
__global__ void __launch_bounds__(kReduceThreads)
count_kept_kernel(const double* __restrict__ mean, long long n_vox, int n_tiles, double truncation,
                  const unsigned long long* __restrict__ col_max_bits,
                  unsigned int* __restrict__ tile_counts) {
    const long long col = blockIdx.y;
    const long long start = (long long)blockIdx.x * kTileVoxels;
    const long long stop = min(start + (long long)kTileVoxels, n_vox);
    const double thr = __dmul_rn(truncation, __longlong_as_double((long long)col_max_bits[col]));
    const double* a = mean + col * n_vox;
    unsigned int c = 0;
    for (long long v = start + threadIdx.x; v < stop; v += blockDim.x) c += keep_entry(a[v], thr);
    __shared__ unsigned int warp_c[kReduceThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0) warp_c[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = 0;
        for (int w = 0; w < kReduceThreads / 32; ++w) t += warp_c[w];
        tile_counts[col * n_tiles + blockIdx.x] = t;
    }
}

// Exclusive scan of the tile counts in CSC order (column-major, tiles
// ascending) with per-column totals; one block, sequential over 1024-wide
// pieces.
__global__ void __launch_bounds__(1024)
scan_tiles_kernel(const unsigned int* __restrict__ tile_counts, long long n,
                  unsigned long long* __restrict__ tile_offsets, int n_cols, int n_tiles,
                  long long* __restrict__ col_counts, unsigned long long* __restrict__ total) {
    __shared__ unsigned long long buf[1024];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0ull;
    __syncthreads();
    for (long long base = 0; base < n; base += 1024) {
        const long long i = base + threadIdx.x;
        const unsigned long long v = i < n ? tile_counts[i] : 0ull;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan
            const unsigned long long add = threadIdx.x >= off ? buf[threadIdx.x - off] : 0ull;
            __syncthreads();
            buf[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < n) tile_offsets[i] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += buf[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
    for (int c = threadIdx.x; c < n_cols; c += blockDim.x) {
        unsigned long long s = 0;
        for (int t = 0; t < n_tiles; ++t) s += tile_counts[(long long)c * n_tiles + t];
        col_counts[c] = (long long)s;
    }
}

// Write the kept entries of one (column, tile) in ascending voxel order at the
// tile's offset: the same order np.flatnonzero gives on the host.
__global__ void __launch_bounds__(kReduceThreads)
compact_kernel(const double* __restrict__ mean, const double* __restrict__ sigma, long long n_vox,
               int n_tiles, double truncation, const unsigned long long* __restrict__ col_max_bits,
               const unsigned long long* __restrict__ tile_offsets, long long* __restrict__ out_idx,
               double* __restrict__ out_dose, double* __restrict__ out_sigma) {
    const long long col = blockIdx.y;
    const long long start = (long long)blockIdx.x * kTileVoxels;
    const long long stop = min(start + (long long)kTileVoxels, n_vox);
    const double thr = __dmul_rn(truncation, __longlong_as_double((long long)col_max_bits[col]));
    const double* a = mean + col * n_vox;
    const double* b = sigma + col * n_vox;
    __shared__ unsigned int warp_c[kReduceThreads / 32];
    __shared__ unsigned long long cursor;
    if (threadIdx.x == 0) cursor = tile_offsets[col * n_tiles + blockIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long v0 = start; v0 < stop; v0 += blockDim.x) {
        const long long v = v0 + threadIdx.x;
        const double m = v < stop ? a[v] : 0.0;
        const bool k = v < stop && keep_entry(m, thr);
        const unsigned int ballot = __ballot_sync(0xffffffffu, k);
        if (lane == 0) warp_c[warp] = __popc(ballot);
        __syncthreads();
        unsigned int before = 0, total = 0;
        for (int w = 0; w < kReduceThreads / 32; ++w) {
            if (w < warp) before += warp_c[w];
            total += warp_c[w];
        }
        if (k) {
            const unsigned long long pos =
                cursor + before + __popc(ballot & ((1u << lane) - 1u));
            out_idx[pos] = v;
            out_dose[pos] = m;
            out_sigma[pos] = b[v];
        }
        __syncthreads();
        if (threadIdx.x == 0) cursor += total;
        __syncthreads();
    }
}

__global__ void zero_u64_kernel(unsigned long long* p, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = 0ull;
}

}  // namespace pmc
