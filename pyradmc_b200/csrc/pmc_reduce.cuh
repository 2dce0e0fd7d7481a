// pmc_reduce.cuh — batch fold, finalize and Dij truncation/compaction.
//
// These are HBM-streaming kernels over the dense [columns][voxels] maps.  Every
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

constexpr int kFoldPerThread = 8;
constexpr int kFoldChunk = kReduceThreads * kFoldPerThread;  // voxels per fold block

// Fold one batch's quanta map into the running sums and consume it (reset the
// folded entries).  Grid: x = chunks of kFoldChunk voxels, y = column, so the
// column (and its history count) is known per block.  Each thread first issues
// all of its quanta loads, then folds the non-empty ones: empty entries are
// skipped, since adding +0.0 leaves the sums bit-unchanged (kernels.py:804-852).
__global__ void __launch_bounds__(kReduceThreads)
fold_kernel(unsigned long long* __restrict__ edep, const double* __restrict__ mass,
            const double* __restrict__ col_nhist, long long n_vox, double* __restrict__ s1,
            double* __restrict__ s2, unsigned long long* __restrict__ total_q) {
    const long long col = blockIdx.y;
    const long long base = col * n_vox;
    const long long start = (long long)blockIdx.x * kFoldChunk + threadIdx.x;
    unsigned long long q[kFoldPerThread];
#pragma unroll
    for (int k = 0; k < kFoldPerThread; ++k) {
        const long long v = start + (long long)k * kReduceThreads;
        q[k] = v < n_vox ? __ldcs(edep + base + v) : 0ull;
    }
    unsigned long long local = 0;
    const double nh = col_nhist[col];
#pragma unroll
    for (int k = 0; k < kFoldPerThread; ++k) {
        if (q[k] == 0ull) continue;
        const long long v = start + (long long)k * kReduceThreads;
        const long long idx = base + v;
        edep[idx] = 0ull;
        const double m = mass[v];
        double d = 0.0;
        if (m > 0.0) {
            const double energy = __dmul_rn((double)(long long)q[k], kQuantum);
            d = __ddiv_rn(energy, __dmul_rn(m, nh));
        }
        s1[idx] = __dadd_rn(s1[idx], d);
        s2[idx] = __dadd_rn(s2[idx], __dmul_rn(d, d));
        local += q[k];
    }
    local = warp_sum_u64(local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(total_q, local);
}

// mean = S1/n, sigma = sqrt(max(0, S2/n - mean^2) * n / (n - 1) / n), written in
// place; the column maximum of the mean rides along (one atomic per block).
// Grid: x = tiles of one column, y = column.
__global__ void __launch_bounds__(kReduceThreads)
finalize_kernel(double* __restrict__ s1, double* __restrict__ s2, long long n_vox, int n_batches,
                unsigned long long* __restrict__ col_max_bits) {
    const long long col = blockIdx.y;
    const long long start = (long long)blockIdx.x * kTileVoxels;
    const long long stop = min(start + (long long)kTileVoxels, n_vox);
    const double n = (double)n_batches;
    unsigned long long best = 0ull;
    double* a = s1 + col * n_vox;
    double* b = s2 + col * n_vox;
    for (long long v = start + threadIdx.x; v < stop; v += blockDim.x) {
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
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(col_max_bits + col, best);
}

// Column maxima of an already finalized mean map (grid: x = tiles, y = column).
__global__ void __launch_bounds__(kReduceThreads)
colmax_kernel(const double* __restrict__ mean, long long n_vox,
              unsigned long long* __restrict__ col_max_bits) {
    const long long col = blockIdx.y;
    const long long start = (long long)blockIdx.x * kTileVoxels;
    const long long stop = min(start + (long long)kTileVoxels, n_vox);
    const double* a = mean + col * n_vox;
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

__device__ __forceinline__ bool keep_entry(double m, double threshold) {
    return m >= threshold && m > 0.0;
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
