/*
 * pyradmc_b200_denoise.h — C-ABI of the Dij-column denoiser (libpmc_b200.so).
 *
 * No counterpart in pyRadMC: the reference has no learned component.  A small
 * 3D U-Net maps a low-history dose column (plus the density) to an estimate of
 * the high-history column.  These entry points are its building blocks; the
 * network, its training loop and its use on a Dij live in the host module
 * pyradmc_b200/denoiser.py.
 *
 * Conventions
 *   - All pointers are DEVICE pointers of the current device; `stream` is a
 *     cudaStream_t (NULL = the default stream).  Calls enqueue work and return
 *     without waiting.
 *   - Activations are bf16 (raw 16-bit storage, passed as void*) in NDHWC
 *     order: channels innermost, then x, y, z, batch.  Every channel count is
 *     a multiple of 8 (16-byte rows).
 *   - A 3x3x3 convolution's weights are bf16 [cout][kpad] with column
 *     k = tap * cin + ci, tap = kz * 9 + ky * 3 + kx (the tap at offset
 *     (kz-1, ky-1, kx-1)), and columns k >= 27 * cin zero.  kpad is 27 * cin
 *     rounded up to a multiple of 64.  Convolutions have stride 1 and zero
 *     padding 1; products accumulate in fp32.
 *   - Return 0 on success, -1 for arguments outside what the kernels support
 *     (nothing launched), -2 when a launch failed.
 */
#ifndef PYRADMC_B200_DENOISE_H
#define PYRADMC_B200_DENOISE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = act(conv3d(x, w) + bias) in bf16; relu != 0 selects ReLU.  bias is fp32
 * [cout] or NULL.  cout in {8, 16, 32, 48, 64, 96, 128, 192}.  The data
 * gradient of a convolution is this call on the output gradient with the
 * weights from pmd_flip_weights (cin and cout swapped, relu = 0). */
int pmd_conv3d(const void* x, const void* w, const float* bias, void* y, int n, int d, int h,
               int w_, int cin, int cout, int kpad, int relu, void* stream);

/* pmd_conv3d followed by the 1x1x1 head, fused in the warp-specialized
 * kernel's epilogue: out[m] = head_b[0] + base[m] + sum_c head_w[c] *
 * y[m][c] (float32; base may be NULL), y the bf16 convolution output, which
 * is not stored.  The same values as pmd_conv3d then pmd_head.  -1 (nothing
 * launched) where the warp-specialized kernel does not cover the shape or
 * another kernel is selected; the caller then runs the two steps. */
int pmd_conv3d_head(const void* x, const void* w, const float* bias, const float* head_w,
                    const float* head_b, const float* base, float* out, int n, int d, int h,
                    int w_, int cin, int cout, int kpad, int relu, void* stream);

/* Selects the convolution kernels of pmd_conv3d: 0 (default) the warp-specialized
 * kernel below wherever it applies except cin = 8, then the single-buffered
 * tensor-memory kernel (tcgen05.mma, accumulators in TMEM; cout a multiple of 16 up to 192,
 * cin 8 or a multiple of 16 up to 96) where its weights are staged in shared
 * memory in at most two passes, and the mma.sync kernel elsewhere; 1 the mma.sync kernel only; 2 the
 * tensor-memory kernel only; 3 its pipelined variant only (two halo buffers
 * and two accumulators, one CTA per SM; measured slower than the default on
 * this network's layers, kept for larger tiles); 4 the warp-specialized kernel only (a TMA producer
 * warp, one MMA-issuing thread and four epilogue warps over a ring of stage
 * buffers; cout a multiple of 16 up to 256, cin 8 or any multiple of 16, weights
 * resident or streamed with the stages).  Other shapes return -1.  impl < 0 only queries.  Returns the
 * previous setting.  Process-wide. */
int pmd_conv3d_impl(int impl);

/* The kernel pmd_conv3d would launch for this shape under the current
 * selection (16-byte aligned operands), written to info[8]: info[0] = 4
 * warp-specialized, 3 pipelined, 2 single-buffered tensor-memory, 1 mma.sync,
 * -1 none; for the warp-specialized kernel info[1..7] = 8-channel chunks per
 * stage, stages per tile, stage buffers, weights streamed (1) or resident (0),
 * output slices per tile, blocks per SM, shared memory bytes per block (the
 * single-buffered kernel fills info[5..7]).  Returns 0, or -1 for a NULL info or
 * an invalid shape. */
int pmd_conv3d_plan(int n, int d, int h, int w_, int cin, int cout, int* info);

/* Number of tensor-memory convolution launches whose wait on the tensor cores
 * ran past its time limit since the last call (their outputs are not valid),
 * and resets it; -2 when the device cannot be read.  Synchronizes the device. */
int pmd_conv3d_failures(void);

/* Weight gradient, ADDED into fp32 dw [cout][kpad] (and dbias [cout] when not
 * NULL): dw[co][k] += sum over voxels of g[v][co] * im2col(x)[v][k].
 * cout in {16, 32, 64, 128}.  Runs on the tensor cores (tcgen05.mma, both
 * operands voxel-major, the sums in tensor memory; one CTA per SM per tap
 * group, its partial sums added with fp32 atomics) unless pmd_conv3d_impl(1)
 * selected the mma.sync kernels or the shape is outside the plan
 * (pmd_conv3d_wgrad_plan); then the mma.sync kernel.  The sum order is not
 * fixed (fp32 atomics). */
int pmd_conv3d_wgrad(const void* x, const void* g, float* dw, float* dbias, int n, int d, int h,
                     int w_, int cin, int cout, int kpad, void* stream);

/* The tensor-core weight-gradient plan for this shape, written to info[8]:
 * output slices per tile, 8-channel chunks per stage, stages per tile (channel
 * groups), accumulator units per group (taps; with cin = 8 rows of three
 * taps), unit groups, stage buffers, shared memory bytes per stage,
 * tensor-memory columns.  Returns 0, or -1 when that kernel does not
 * cover the shape (or info is NULL). */
int pmd_conv3d_wgrad_plan(int n, int d, int h, int w_, int cin, int cout, int* info);

/* Data-gradient weights: wd[ci][tap * cout + co] = w[co][(26 - tap) * cin + ci],
 * bf16 [cin][kpad_d], columns past 27 * cout zero. */
int pmd_flip_weights(const void* w, void* wd, int cin, int cout, int kpad, int kpad_d, void* stream);

/* ReLU backward in place: g[i] = 0 where y[i] <= 0 (n elements, a multiple
 * of 8). */
int pmd_relu_mask(void* g, const void* y, int64_t n, void* stream);

/* 2x2x2 average pooling of x [n, d, h, w, c] into y [n, d/2, h/2, w/2, c], and
 * its gradient (written, or added onto gx when accumulate != 0).  c a multiple
 * of 8; d, h, w even; fewer than 2^31 elements. */
int pmd_avgpool(const void* x, void* y, int n, int d, int h, int w, int c, void* stream);
int pmd_avgpool_grad(const void* gy, void* gx, int n, int d, int h, int w, int c, int accumulate,
                     void* stream);

/* Decoder join: out [n, d, h, w, c_up + c_skip] = concat(nearest-upsample x2 of
 * up [n, d/2, h/2, w/2, c_up], skip), and its gradient (the skip part written,
 * or added onto gskip when accumulate != 0).  c_up, c_skip multiples of 8;
 * d, h, w even; fewer than 2^31 elements. */
int pmd_upcat(const void* up, const void* skip, void* out, int n, int d, int h, int w, int c_up,
              int c_skip, void* stream);
int pmd_upcat_grad(const void* gout, void* gup, void* gskip, int n, int d, int h, int w, int c_up,
                   int c_skip, int accumulate, void* stream);

/* Output head: out[m] = base[m] + b[0] + sum_c w[c] * f[m][c] over m voxels
 * (fp32; base may be NULL), and its gradient: df = g w^T (bf16), dw += f^T g,
 * db += sum g.  c in {8, 16, 32, 64}. */
int pmd_head(const void* f, const float* w, const float* b, const float* base, float* out,
             int64_t m, int c, void* stream);
int pmd_head_grad(const void* f, const float* w, const float* g, void* df, float* dw, float* db,
                  int64_t m, int c, void* stream);

/* Loss l = mean_m |pred - target| * (1 + lambda * weight[m]) ADDED into
 * loss[0], and grad = dl/dpred (weight may be NULL). */
int pmd_loss(const float* pred, const float* target, const float* weight, float lambda,
             float* grad, float* loss, int64_t m, void* stream);

/* Adam (Kingma & Ba) on n fp32 parameters at step >= 1; refreshes the bf16
 * copy p16 (same indexing) when not NULL. */
int pmd_adam(float* p, const float* g, float* m, float* v, void* p16, int64_t n, float lr,
             float beta1, float beta2, float eps, int step, void* stream);

/* Network input, 8 channels [m][8]: dose[m] / colmax[m / vox] (colmax NULL:
 * no scaling; a zero maximum scales by 1), density[m % vox] when
 * density_shared != 0 else density[m], sigma[m] (the dose's Monte Carlo
 * standard error; NULL: zero) on the dose's scale, and five zero channels.
 * base (fp32, may be NULL) receives the scaled dose. */
int pmd_pack_input(const float* dose, const float* density, const float* sigma,
                   const float* colmax, int64_t vox, int density_shared, void* x, float* base,
                   int64_t m, void* stream);

/* Dense columns from a CSC matrix: dense[col * vox + indices[j]] = values[j]
 * (float) for j in [indptr[col], indptr[col + 1]); the rest of dense must be
 * zeroed by the caller.  Also colmax[col] = max of the column's values
 * (colmax zeroed by the caller).  n_cols <= 65535. */
int pmd_csc_to_dense(const int64_t* indptr, const int64_t* indices, const double* values,
                     int n_cols, int64_t vox, float* dense, float* colmax, void* stream);

/* The same into float64 (no maximum): for the dense mean and sigma that the
 * truncation + CSC compaction (pmc_dij_compact_static) consumes. */
int pmd_csc_to_dense_f64(const int64_t* indptr, const int64_t* indices, const double* values,
                         int n_cols, int64_t vox, double* dense, void* stream);

/* Windows of a stack of nx*ny*nz volumes (x-major, z fastest): out[c] is the
 * wx*wy*wz window of volume c (src + c * src_stride; src_stride 0 reads one
 * shared volume) whose first voxel is (ox, oy, oz) = origins[3c .. 3c+2]
 * (int32, may lie partly outside; outside reads as zero). */
int pmd_gather_windows(const float* src, int64_t src_stride, int nx, int ny, int nz,
                       const int32_t* origins, int n_windows, int wx, int wy, int wz, float* out,
                       void* stream);

/* The reverse, in dose units: dst[c * dst_stride + voxel] = max(win, 0) *
 * scale[c] (float64; scale NULL or zero: 1) for every window voxel inside the
 * volume; voxels outside every window keep their value. */
int pmd_scatter_windows(const float* win, const float* scale, int nx, int ny, int nz,
                        const int32_t* origins, int n_windows, int wx, int wy, int wz, double* dst,
                        int64_t dst_stride, void* stream);

/* Oriented windows (beamlets along any direction).  Window w is
 * win[7w .. 7w+6] = (ox, oy, oz, orient, col, shear1, shear2), int32: orient =
 * 2 * d + f names the depth axis d (0 x, 1 y, 2 z), read from its high end
 * when f = 1; the two other axes, in increasing order, are the window's first
 * two dimensions, shifted by s1(k) = round(k * shear1 / 65536) and s2(k)
 * voxels at window depth k (an oblique beamlet stays centred).  Window voxel
 * (a, b, k) of the wa*wb*wd window is voxel g of volume col with g[first] =
 * o[first] + a + s1(k), g[second] = o[second] + b + s2(k), g[d] = o[d] + k
 * (f = 0) or o[d] + wd - 1 - k (f = 1).  Gather: out[w][a][b][k] (zero outside
 * the grid).  Scatter: dst[col * dst_stride + g] = max(data, 0) * scale[w]
 * (float64; scale NULL or zero: 1) for window voxels inside the grid; windows
 * of one column must not overlap.  orient = 4, col = w and no shear is the
 * window of pmd_gather_windows / pmd_scatter_windows. */
int pmd_gather_windows_oriented(const float* src, int64_t src_stride, int nx, int ny, int nz,
                                const int32_t* win, int n_windows, int wa, int wb, int wd, float* out,
                                void* stream);
int pmd_scatter_windows_oriented(const float* data, const float* scale, int nx, int ny, int nz,
                                 const int32_t* win, int n_windows, int wa, int wb, int wd, double* dst,
                                 int64_t dst_stride, void* stream);

/* Back to dose units: mean[m] = max(out[m], 0) * colmax[m / vox] (float64). */
int pmd_unscale(const float* out, const float* colmax, int64_t vox, double* mean, int64_t m,
                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PYRADMC_B200_DENOISE_H */
