// denoise.cu — the 3D U-Net denoiser's kernels (no counterpart in pyRadMC).
//
// Activations are bf16 in NDHWC (channels innermost); weights bf16 as
// [Cout][Kpad] with K = tap * Cin + ci over the 27 taps of a 3x3x3 kernel
// (zero padded to a multiple of 64); every product accumulates in fp32.
//
// Convolution is an implicit GEMM on the tensor cores (mma.sync m16n8k16
// bf16 -> fp32): M = voxels, N = output channels, K = 27 * Cin.  The A tile is
// gathered straight from the activation with 16-byte cp.async copies whose
// zero-fill form supplies the convolution's zero padding, double-buffered
// against the MMAs.  The same kernel runs the data gradient (with flipped,
// transposed weights); the weight gradient is a second implicit GEMM that
// reduces over voxels and adds its fp32 partial into the gradient buffer.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "pyradmc_b200_denoise.h"

namespace pmd {

constexpr int kBM = 64;      // voxels per CTA tile
constexpr int kBK = 32;      // K per pipeline stage
constexpr int kPadK = 8;     // smem row padding (elements) against ldmatrix bank conflicts
constexpr int kRowK = kBK + kPadK;
constexpr int kThreads = 128;

struct ConvShape {
    int n, d, h, w;     // batch and spatial size (stride 1, padding 1)
    int cin, cout;      // cin % 8 == 0, cout % 8 == 0
    int kpad;           // 27 * cin rounded up to a multiple of 64
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;  // src-size 0: the 16 destination bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3,
                                            const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldmatrix_x2(uint32_t& r0, uint32_t& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r0), "=r"(r1)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldmatrix_x2_t(uint32_t& r0, uint32_t& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r0), "=r"(r1)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldmatrix_x4_t(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3,
                                              const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void mma_bf16(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Source of one 8-channel chunk of the implicit A matrix: voxel m's neighbour
// at tap (k / cin) and channels (k % cin) .. +7; null when it lies in the
// zero padding or past K.
__device__ __forceinline__ const __nv_bfloat16* a_chunk(const __nv_bfloat16* x, const ConvShape& s,
                                                        int nz, int zz, int yy, int xx, int k) {
    if (k >= 27 * s.cin) return nullptr;
    const int tap = k / s.cin;
    const int ci = k - tap * s.cin;
    const int z = zz + tap / 9 - 1;
    const int y = yy + (tap / 3) % 3 - 1;
    const int xq = xx + tap % 3 - 1;
    if ((unsigned)z >= (unsigned)s.d || (unsigned)y >= (unsigned)s.h || (unsigned)xq >= (unsigned)s.w)
        return nullptr;
    return x + ((((long long)nz * s.d + z) * s.h + y) * s.w + xq) * s.cin + ci;
}

// ---- forward / data-gradient convolution ------------------------------------------
// Y[m][co] = act(bias[co] + sum_k A[m][k] W[co][k]).  BN = cout (a multiple of 8).
// Four warps; warp w owns tile rows 16w .. 16w+15 and every output channel.
template <int BN>
__global__ void __launch_bounds__(kThreads)
conv3d_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wt,
              const float* __restrict__ bias, __nv_bfloat16* __restrict__ y, ConvShape s, int relu) {
    __shared__ __align__(16) __nv_bfloat16 As[2][kBM][kRowK];
    __shared__ __align__(16) __nv_bfloat16 Bs[2][BN][kRowK];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const long long m_total = (long long)s.n * s.d * s.h * s.w;
    const long long m0 = (long long)blockIdx.x * kBM;

    // each thread gathers rows tid / 4 and tid / 4 + 32, 8-element chunk tid % 4
    const int chunk = tid & 3;
    int rz[2], ry[2], rx[2], rn[2];
    bool rvalid[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const long long m = m0 + (tid >> 2) + 32 * i;
        rvalid[i] = m < m_total;
        long long t = rvalid[i] ? m : 0;
        rx[i] = (int)(t % s.w);
        t /= s.w;
        ry[i] = (int)(t % s.h);
        t /= s.h;
        rz[i] = (int)(t % s.d);
        rn[i] = (int)(t / s.d);
    }

    auto load_stage = [&](int stage, int kb) {
        const int k = kb * kBK + chunk * 8;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const __nv_bfloat16* src = rvalid[i] ? a_chunk(x, s, rn[i], rz[i], ry[i], rx[i], k) : nullptr;
            cp_async16(&As[stage][(tid >> 2) + 32 * i][chunk * 8], src ? src : x, src != nullptr);
        }
        for (int c = tid; c < BN * 4; c += kThreads) {
            const int row = c >> 2, cc = c & 3;
            cp_async16(&Bs[stage][row][cc * 8], wt + (long long)row * s.kpad + kb * kBK + cc * 8, true);
        }
        cp_async_commit();
    };

    float acc[BN / 8][4];
#pragma unroll
    for (int j = 0; j < BN / 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;

    const int n_kb = s.kpad / kBK;
    load_stage(0, 0);
    for (int kb = 0; kb < n_kb; ++kb) {
        const int cur = kb & 1;
        if (kb + 1 < n_kb) {
            load_stage(cur ^ 1, kb + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < kBK / 16; ++ks) {
            uint32_t a0, a1, a2, a3;
            ldmatrix_x4(a0, a1, a2, a3, &As[cur][warp * 16 + (lane & 15)][ks * 16 + (lane >> 4) * 8]);
#pragma unroll
            for (int j = 0; j < BN / 8; ++j) {
                uint32_t b0, b1;
                ldmatrix_x2(b0, b1, &Bs[cur][j * 8 + (lane & 7)][ks * 16 + ((lane >> 3) & 1) * 8]);
                mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
            }
        }
        __syncthreads();
    }

    // epilogue: bias, ReLU, bf16, NDHWC store
    const int r_lo = warp * 16 + (lane >> 2);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const long long m = m0 + r_lo + 8 * half;
        if (m >= m_total) continue;
        __nv_bfloat16* out = y + m * s.cout;
#pragma unroll
        for (int j = 0; j < BN / 8; ++j) {
            const int co = j * 8 + (lane & 3) * 2;
            float v0 = acc[j][2 * half], v1 = acc[j][2 * half + 1];
            if (bias) {
                v0 += bias[co];
                v1 += bias[co + 1];
            }
            if (relu) {
                v0 = fmaxf(v0, 0.0f);
                v1 = fmaxf(v1, 0.0f);
            }
            *reinterpret_cast<__nv_bfloat162*>(out + co) = __floats2bfloat162_rn(v0, v1);
        }
    }
}

// ---- weight gradient ----------------------------------------------------------------
// dW[co][k] += sum_m G[m][co] A[m][k] over this CTA's voxel range.  Grid: x =
// 64-wide k tiles, y = voxel splits.  MMA rows = co (BC = cout), cols = k,
// reduction = voxels; both operands come from voxel-major smem tiles through
// transposing ldmatrix loads.
constexpr int kWK = 64;   // k columns per CTA
constexpr int kWM = 32;   // voxels per pipeline stage
template <int BC>
__global__ void __launch_bounds__(kThreads)
conv3d_wgrad_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ g,
                    float* __restrict__ dw, float* __restrict__ dbias, ConvShape s,
                    long long voxels_per_split) {
    __shared__ __align__(16) __nv_bfloat16 Gs[2][kWM][BC + 8];
    __shared__ __align__(16) __nv_bfloat16 Xs[2][kWM][kWK + 8];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const long long m_total = (long long)s.n * s.d * s.h * s.w;
    const long long v_begin = (long long)blockIdx.y * voxels_per_split;
    const long long v_end = min(v_begin + voxels_per_split, m_total);
    const int k0 = blockIdx.x * kWK;
    // warp tiling of the (BC x 64) output: BC/16 row tiles x 8 col tiles over 4 warps
    constexpr int kRowTiles = BC / 16;
    constexpr int kTiles = kRowTiles * (kWK / 8);
    constexpr int kPerWarp = (kTiles + 3) / 4;
    float acc[kPerWarp][4];
#pragma unroll
    for (int t = 0; t < kPerWarp; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0f;
    float bacc = 0.0f;  // bias gradient: thread tid < BC sums column tid of G

    auto load_stage = [&](int stage, long long v0) {
        // G tile: kWM voxels x BC channels
        for (int c = tid; c < kWM * (BC / 8); c += kThreads) {
            const int row = c / (BC / 8), cc = c % (BC / 8);
            const long long v = v0 + row;
            const bool ok = v < v_end;
            cp_async16(&Gs[stage][row][cc * 8], ok ? g + v * s.cout + cc * 8 : g, ok);
        }
        // im2col tile: kWM voxels x kWK k
        for (int c = tid; c < kWM * (kWK / 8); c += kThreads) {
            const int row = c / (kWK / 8), cc = c % (kWK / 8);
            const long long v = v0 + row;
            const __nv_bfloat16* src = nullptr;
            if (v < v_end) {
                long long t = v;
                const int xx = (int)(t % s.w);
                t /= s.w;
                const int yy = (int)(t % s.h);
                t /= s.h;
                const int zz = (int)(t % s.d);
                const int nz = (int)(t / s.d);
                src = a_chunk(x, s, nz, zz, yy, xx, k0 + cc * 8);
            }
            cp_async16(&Xs[stage][row][cc * 8], src ? src : x, src != nullptr);
        }
        cp_async_commit();
    };

    const long long n_steps = (v_end - v_begin + kWM - 1) / kWM;
    if (n_steps <= 0) return;
    load_stage(0, v_begin);
    for (long long st = 0; st < n_steps; ++st) {
        const int cur = (int)(st & 1);
        if (st + 1 < n_steps) {
            load_stage(cur ^ 1, v_begin + (st + 1) * kWM);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (dbias != nullptr && blockIdx.x == 0 && tid < BC) {
#pragma unroll 4
            for (int r = 0; r < kWM; ++r) bacc += __bfloat162float(Gs[cur][r][tid]);
        }
#pragma unroll
        for (int ks = 0; ks < kWM / 16; ++ks) {
#pragma unroll
            for (int t = 0; t < kPerWarp; ++t) {
                const int tile = warp * kPerWarp + t;
                if (tile >= kTiles) break;
                const int rt = tile / (kWK / 8), ct = tile % (kWK / 8);
                uint32_t a0, a1, a2, a3, b0, b1;
                // A = G^T: rows co (16), cols voxels (16)
                {
                    const int q = lane >> 3, r = lane & 7;
                    const int vrow = ks * 16 + (q >> 1) * 8 + r;
                    const int col = rt * 16 + (q & 1) * 8;
                    ldmatrix_x4_t(a0, a1, a2, a3, &Gs[cur][vrow][col]);
                }
                // B = im2col: K = voxels (16), N = k (8); lanes 0-15 address its two 8x8 halves
                {
                    const int vrow = ks * 16 + (lane & 15);
                    ldmatrix_x2_t(b0, b1, &Xs[cur][vrow][ct * 8]);
                }
                mma_bf16(acc[t], a0, a1, a2, a3, b0, b1);
            }
        }
        __syncthreads();
    }
    // add this split's partial into dW (fp32)
#pragma unroll
    for (int t = 0; t < kPerWarp; ++t) {
        const int tile = warp * kPerWarp + t;
        if (tile >= kTiles) break;
        const int rt = tile / (kWK / 8), ct = tile % (kWK / 8);
        const int co = rt * 16 + (lane >> 2);
        const int k = k0 + ct * 8 + (lane & 3) * 2;
        atomicAdd(dw + (long long)co * s.kpad + k, acc[t][0]);
        atomicAdd(dw + (long long)co * s.kpad + k + 1, acc[t][1]);
        atomicAdd(dw + (long long)(co + 8) * s.kpad + k, acc[t][2]);
        atomicAdd(dw + (long long)(co + 8) * s.kpad + k + 1, acc[t][3]);
    }
    if (dbias != nullptr && blockIdx.x == 0 && tid < BC) atomicAdd(dbias + tid, bacc);
}

// ---- element-wise and data-movement kernels -------------------------------------------
// 16-byte vectors of 8 bf16 channels.
union Pack8 {
    uint4 u;
    __nv_bfloat162 h[4];
};
__device__ __forceinline__ void unpack8(uint4 v, float* f) {
    Pack8 p;
    p.u = v;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 t = __bfloat1622float2(p.h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
    Pack8 p;
#pragma unroll
    for (int i = 0; i < 4; ++i) p.h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    return p.u;
}

// ReLU backward in place: g <- g * (y > 0), 8 channels per thread (n8 vectors).
__global__ void relu_mask_kernel(uint4* g, const uint4* y, long long n8) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n8; i += stride) {
        float gv[8], yv[8];
        unpack8(g[i], gv);
        unpack8(__ldg(y + i), yv);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (!(yv[k] > 0.0f)) gv[k] = 0.0f;
        g[i] = pack8(gv);
    }
}

// Weights for the data gradient: Wd[ci][tap' * cout + co] = W[co][(26 - tap') * cin + ci].
__global__ void flip_weights_kernel(const __nv_bfloat16* w, __nv_bfloat16* wd, int cin, int cout,
                                    int kpad, int kpad_d) {
    const long long n = (long long)cin * kpad_d;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int ci = (int)(i / kpad_d), k = (int)(i % kpad_d);
        __nv_bfloat16 v = __float2bfloat16(0.0f);
        if (k < 27 * cout) {
            const int tap = k / cout, co = k % cout;
            v = w[(long long)co * kpad + (26 - tap) * cin + ci];
        }
        wd[i] = v;
    }
}

// 2x2x2 average pooling, NDHWC, one 8-channel vector per thread (c8 = c / 8
// vectors per voxel; 32-bit indices: the host bounds the element counts).
__global__ void avgpool_kernel(const uint4* x, uint4* y, int n, int d, int h, int w, int c8) {
    const int d2 = d / 2, h2 = h / 2, w2 = w / 2;
    const int total = n * d2 * h2 * w2 * c8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int t = i;
        const int cc = t % c8; t /= c8;
        const int xx = t % w2; t /= w2;
        const int yy = t % h2; t /= h2;
        const int zz = t % d2;
        const int nn = t / d2;
        const int v0 = ((nn * d + 2 * zz) * h + 2 * yy) * w + 2 * xx;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            float f[8];
            unpack8(__ldg(x + (size_t)(v0 + (o >> 2) * h * w + ((o >> 1) & 1) * w + (o & 1)) * c8 + cc), f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] *= 0.125f;
        y[i] = pack8(acc);
    }
}

__global__ void avgpool_grad_kernel(const uint4* gy, uint4* gx, int n, int d, int h, int w, int c8,
                                    int accumulate) {
    const int total = n * d * h * w * c8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int t = i;
        const int cc = t % c8; t /= c8;
        const int xx = t % w; t /= w;
        const int yy = t % h; t /= h;
        const int zz = t % d;
        const int nn = t / d;
        float v[8];
        unpack8(__ldg(gy + (size_t)(((nn * (d / 2) + zz / 2) * (h / 2) + yy / 2) * (w / 2) + xx / 2) * c8 + cc), v);
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] *= 0.125f;
        if (accumulate) {
            float o[8];
            unpack8(gx[i], o);
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] += o[k];
        }
        gx[i] = pack8(v);
    }
}

// Nearest 2x upsampling of `up` (cu8 vectors per voxel) into the first
// vectors of a concatenated tensor whose remaining cs8 vectors copy `skip`.
__global__ void upcat_kernel(const uint4* up, const uint4* skip, uint4* out, int n, int d, int h, int w,
                             int cu8, int cs8) {
    const int c8 = cu8 + cs8;
    const int total = n * d * h * w * c8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int cc = i % c8;
        const int vox = i / c8;
        uint4 v;
        if (cc < cu8) {
            int t = vox;
            const int xx = t % w; t /= w;
            const int yy = t % h; t /= h;
            const int zz = t % d;
            const int nn = t / d;
            v = __ldg(up + (size_t)(((nn * (d / 2) + zz / 2) * (h / 2) + yy / 2) * (w / 2) + xx / 2) * cu8 + cc);
        } else {
            v = __ldg(skip + (size_t)vox * cs8 + (cc - cu8));
        }
        out[i] = v;
    }
}

// Gradient of upcat: the up part sums its 8 children; the skip part is copied
// (added onto an existing skip gradient when `accumulate`).
__global__ void upcat_grad_kernel(const uint4* gout, uint4* gup, uint4* gskip, int n, int d, int h,
                                  int w, int cu8, int cs8, int accumulate) {
    const int c8 = cu8 + cs8;
    const int d2 = d / 2, h2 = h / 2, w2 = w / 2;
    const int n_up = n * d2 * h2 * w2 * cu8;
    const int n_skip = n * d * h * w * cs8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_up + n_skip; i += gridDim.x * blockDim.x) {
        if (i < n_up) {
            int t = i;
            const int cc = t % cu8; t /= cu8;
            const int xx = t % w2; t /= w2;
            const int yy = t % h2; t /= h2;
            const int zz = t % d2;
            const int nn = t / d2;
            const int v0 = ((nn * d + 2 * zz) * h + 2 * yy) * w + 2 * xx;
            float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                float f[8];
                unpack8(__ldg(gout + (size_t)(v0 + (o >> 2) * h * w + ((o >> 1) & 1) * w + (o & 1)) * c8 + cc), f);
#pragma unroll
                for (int k = 0; k < 8; ++k) acc[k] += f[k];
            }
            gup[i] = pack8(acc);
        } else {
            const int j = i - n_up;
            const int vox = j / cs8, cc = j % cs8;
            uint4 v = __ldg(gout + (size_t)vox * c8 + cu8 + cc);
            if (accumulate) {
                float a[8], b[8];
                unpack8(v, a);
                unpack8(gskip[j], b);
#pragma unroll
                for (int k = 0; k < 8; ++k) a[k] += b[k];
                v = pack8(a);
            }
            gskip[j] = v;
        }
    }
}

// Head: out[m] = base[m] + b + sum_c w[c] f[m][c] (a 1x1x1 conv to one channel,
// added to the noisy input dose: the network predicts a correction).
template <int C>
__global__ void head_kernel(const uint4* f, const float* w, const float* b, const float* base,
                            float* out, long long m_total) {
    float wl[C];
#pragma unroll
    for (int k = 0; k < C; ++k) wl[k] = __ldg(w + k);
    const float bias = __ldg(b);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < m_total; m += stride) {
        float acc = bias + (base ? base[m] : 0.0f);
#pragma unroll
        for (int c = 0; c < C / 8; ++c) {
            float v[8];
            unpack8(__ldg(f + m * (C / 8) + c), v);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc += wl[c * 8 + k] * v[k];
        }
        out[m] = acc;
    }
}

// Loss (L1 plus an L1 weighted by the target's precision) and its gradient with
// respect to the prediction:
//   l = |p - t| * (1 + lambda * weight),  dl/dp = sign(p - t) * (1 + lambda * weight),
// both divided by the voxel count.  Partial sums accumulate into loss[0].
__global__ void loss_kernel(const float* pred, const float* target, const float* weight,
                            float lambda, float* grad, float* loss, long long m_total) {
    float local = 0.0f;
    const float inv_n = 1.0f / (float)m_total;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < m_total; m += stride) {
        const float diff = pred[m] - target[m];
        const float wgt = 1.0f + lambda * (weight ? weight[m] : 0.0f);
        local += fabsf(diff) * wgt;
        grad[m] = (diff > 0.0f ? wgt : (diff < 0.0f ? -wgt : 0.0f)) * inv_n;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) local += __shfl_xor_sync(0xffffffffu, local, off);
    __shared__ float part[8];  // one sum per warp of the 256-thread block, one atomic per block
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.0f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += part[i];
        atomicAdd(loss, v * inv_n);
    }
}

// Head backward: dF[m][c] = g[m] w[c] (bf16), dW[c] += sum_m g[m] f[m][c], db += sum_m g[m].
template <int C>
__global__ void head_grad_kernel(const uint4* f, const float* w, const float* g, uint4* df,
                                 float* dw, float* db, long long m_total) {
    float wl[C], lw[C];
#pragma unroll
    for (int k = 0; k < C; ++k) {
        wl[k] = __ldg(w + k);
        lw[k] = 0.0f;
    }
    float lb = 0.0f;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < m_total; m += stride) {
        const float gm = g[m];
        lb += gm;
#pragma unroll
        for (int c = 0; c < C / 8; ++c) {
            float v[8], o[8];
            unpack8(__ldg(f + m * (C / 8) + c), v);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                lw[c * 8 + k] += gm * v[k];
                o[k] = gm * wl[c * 8 + k];
            }
            df[m * (C / 8) + c] = pack8(o);
        }
    }
    // warp sums, then block sums: one atomic per block and parameter (the
    // launch keeps the grid at a few blocks per SM, so each of the C + 1
    // addresses sees a few hundred atomics, not one per warp)
    __shared__ float part[C + 1][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < C; ++k) {
        float v = lw[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) part[k][warp] = v;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lb += __shfl_xor_sync(0xffffffffu, lb, off);
    if (lane == 0) part[C][warp] = lb;
    __syncthreads();
    if (threadIdx.x <= C) {
        float v = 0.0f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += part[threadIdx.x][i];
        atomicAdd(threadIdx.x < C ? dw + threadIdx.x : db, v);
    }
}

// Adam on fp32 master parameters; refreshes the bf16 working copy (when given)
// at the same flat index.
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, __nv_bfloat16* p16,
                            long long n, float lr, float beta1, float beta2, float eps, float bc1,
                            float bc2) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float gi = g[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        p[i] = pi;
        if (p16) p16[i] = __float2bfloat16(pi);
    }
}

// Network input: channel 0 the column-normalized dose, channel 1 the density,
// channel 2 the dose's Monte Carlo sigma on the same scale, 3..7 zero; one
// 16-byte store per voxel.
__global__ void pack_input_kernel(const float* dose, const float* density, const float* sigma,
                                  const float* colmax, long long vox, int density_shared,
                                  __nv_bfloat16* x, float* base, long long m_total) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < m_total; m += stride) {
        float scale = 1.0f;
        if (colmax) {
            const float c = colmax[m / vox];
            scale = c > 0.0f ? 1.0f / c : 1.0f;
        }
        const float v = dose[m] * scale;
        const float rho = density[density_shared ? m % vox : m];
        const float sg = sigma ? sigma[m] * scale : 0.0f;
        if (base) base[m] = v;
        union {
            uint4 u;
            __nv_bfloat162 h[4];
        } pk;
        pk.h[0] = __floats2bfloat162_rn(v, rho);
        pk.h[1] = __floats2bfloat162_rn(sg, 0.0f);
        pk.h[2] = pk.h[3] = __floats2bfloat162_rn(0.0f, 0.0f);
        *reinterpret_cast<uint4*>(x + m * 8) = pk.u;
    }
}

// CSC -> dense columns, with each column's maximum (values are non-negative, so
// the float bit patterns order like the values).
__global__ void csc_to_dense_kernel(const int64_t* indptr, const int64_t* indices,
                                    const double* values, long long vox, float* dense,
                                    float* colmax) {
    const int col = blockIdx.y;
    const long long begin = indptr[col], end = indptr[col + 1];
    float local = 0.0f;
    for (long long j = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x; j < end;
         j += (long long)gridDim.x * blockDim.x) {
        const float v = (float)values[j];
        dense[(long long)col * vox + indices[j]] = v;
        local = fmaxf(local, v);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, off));
    if ((threadIdx.x & 31) == 0 && local > 0.0f)
        atomicMax(reinterpret_cast<int*>(colmax + col), __float_as_int(local));
}

__global__ void unscale_kernel(const float* out, const float* colmax, long long vox, double* mean,
                               long long m_total) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < m_total; m += stride) {
        const float c = colmax[m / vox];
        mean[m] = (double)fmaxf(out[m], 0.0f) * (double)(c > 0.0f ? c : 1.0f);
    }
}

// Windows of a stack of volumes (x-major, z fastest): window c of size
// wx*wy*wz at origin (ox, oy, oz)[c]; voxels outside the volume read as zero.
__global__ void gather_windows_kernel(const float* src, long long src_stride, int nx, int ny,
                                      int nz, const int* origins, int wx, int wy, int wz,
                                      float* out, long long total) {
    const long long per = (long long)wx * wy * wz;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int c = (int)(i / per);
        long long r = i - (long long)c * per;
        const int k = (int)(r % wz); r /= wz;
        const int j = (int)(r % wy);
        const int ii = (int)(r / wy);
        const int x = origins[3 * c] + ii, y = origins[3 * c + 1] + j, z = origins[3 * c + 2] + k;
        float v = 0.0f;
        if ((unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz)
            v = src[(long long)c * src_stride + ((long long)x * ny + y) * nz + z];
        out[i] = v;
    }
}

__global__ void scatter_windows_kernel(const float* win, const float* scale, int nx, int ny, int nz,
                                       const int* origins, int wx, int wy, int wz, double* dst,
                                       long long dst_stride, long long total) {
    const long long per = (long long)wx * wy * wz;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int c = (int)(i / per);
        long long r = i - (long long)c * per;
        const int k = (int)(r % wz); r /= wz;
        const int j = (int)(r % wy);
        const int ii = (int)(r / wy);
        const int x = origins[3 * c] + ii, y = origins[3 * c + 1] + j, z = origins[3 * c + 2] + k;
        if ((unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz) {
            const float sc = scale ? scale[c] : 1.0f;
            dst[(long long)c * dst_stride + ((long long)x * ny + y) * nz + z] =
                (double)fmaxf(win[i], 0.0f) * (double)(sc > 0.0f ? sc : 1.0f);
        }
    }
}

// Oriented windows.  Window w is win[7w..7w+6] = (ox, oy, oz, orient, col,
// shear1, shear2): orient = 2 * d + f names the depth axis d (0 x, 1 y, 2 z),
// read from its high end when f = 1; the two other axes, in increasing order,
// are the window's first two dimensions; shear1/2 move them by
// round(k * shear / 65536) voxels at window depth k, so that a window can
// follow an oblique beamlet.  Window voxel (a, b, k) is grid voxel g with
// g[first] = o[first] + a + s1(k), g[second] = o[second] + b + s2(k) and
// g[d] = o[d] + k (f = 0) or o[d] + wd - 1 - k (f = 1), of volume col.  For a
// fixed k the shift is the same for every (a, b), so the map is one to one.
constexpr int kWinInts = 7;

__device__ __forceinline__ bool oriented_voxel(const int* wdesc, int a, int b, int k, int wd, int nx,
                                               int ny, int nz, long long& flat) {
    const int d = wdesc[3] >> 1, f = wdesc[3] & 1;
    const int l1 = d == 0 ? 1 : 0, l2 = d == 2 ? 1 : 2;
    const int s1 = (int)(((long long)k * wdesc[5] + 32768) >> 16);
    const int s2 = (int)(((long long)k * wdesc[6] + 32768) >> 16);
    int g[3];
    g[l1] = wdesc[l1] + a + s1;
    g[l2] = wdesc[l2] + b + s2;
    g[d] = wdesc[d] + (f ? wd - 1 - k : k);
    if ((unsigned)g[0] >= (unsigned)nx || (unsigned)g[1] >= (unsigned)ny || (unsigned)g[2] >= (unsigned)nz)
        return false;
    flat = ((long long)g[0] * ny + g[1]) * nz + g[2];
    return true;
}

__global__ void gather_oriented_kernel(const float* src, long long src_stride, int nx, int ny, int nz,
                                       const int* win, int wa, int wb, int wd, float* out,
                                       long long total) {
    const long long per = (long long)wa * wb * wd;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int w = (int)(i / per);
        long long r = i - (long long)w * per;
        const int k = (int)(r % wd); r /= wd;
        const int b = (int)(r % wb);
        const int a = (int)(r / wb);
        const int* wdesc = win + kWinInts * w;
        long long flat;
        float v = 0.0f;
        if (oriented_voxel(wdesc, a, b, k, wd, nx, ny, nz, flat))
            v = src[(long long)wdesc[4] * src_stride + flat];
        out[i] = v;
    }
}

__global__ void scatter_oriented_kernel(const float* data, const float* scale, int nx, int ny, int nz,
                                        const int* win, int wa, int wb, int wd, double* dst,
                                        long long dst_stride, long long total) {
    const long long per = (long long)wa * wb * wd;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int w = (int)(i / per);
        long long r = i - (long long)w * per;
        const int k = (int)(r % wd); r /= wd;
        const int b = (int)(r % wb);
        const int a = (int)(r / wb);
        const int* wdesc = win + kWinInts * w;
        long long flat;
        if (oriented_voxel(wdesc, a, b, k, wd, nx, ny, nz, flat)) {
            const float sc = scale ? scale[w] : 1.0f;
            dst[(long long)wdesc[4] * dst_stride + flat] =
                (double)fmaxf(data[i], 0.0f) * (double)(sc > 0.0f ? sc : 1.0f);
        }
    }
}

// CSC -> dense float64 columns (the caller zeroes dense).
__global__ void csc_to_dense_f64_kernel(const int64_t* indptr, const int64_t* indices,
                                        const double* values, long long vox, double* dense) {
    const int col = blockIdx.y;
    const long long begin = indptr[col], end = indptr[col + 1];
    for (long long j = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x; j < end;
         j += (long long)gridDim.x * blockDim.x)
        dense[(long long)col * vox + indices[j]] = values[j];
}

}  // namespace pmd

#include "denoise_umma.cuh"
#include "denoise_ws.cuh"
#include "denoise_wgrad.cuh"

using namespace pmd;

namespace {

int grid_for(long long n, int block = 256) {
    long long b = (n + block - 1) / block;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)(b < 1 ? 1 : b);
}

template <int BN>
void launch_conv(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* y,
                 ConvShape s, int relu, cudaStream_t st) {
    const long long m = (long long)s.n * s.d * s.h * s.w;
    conv3d_kernel<BN><<<(unsigned)((m + kBM - 1) / kBM), kThreads, 0, st>>>(x, w, bias, y, s, relu);
}

template <int BC>
void launch_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* g, float* dw, float* db, ConvShape s,
                  cudaStream_t st) {
    const long long m = (long long)s.n * s.d * s.h * s.w;
    const int kt = s.kpad / kWK;
    // enough voxel splits for ~4 CTAs per SM over all k tiles
    long long splits = (148LL * 4 + kt - 1) / kt;
    long long per = (m + splits - 1) / splits;
    per = ((per + kWM - 1) / kWM) * kWM;
    splits = (m + per - 1) / per;
    conv3d_wgrad_kernel<BC><<<dim3(kt, (unsigned)splits), kThreads, 0, st>>>(x, g, dw, db, s, per);
}

int launched() { return cudaGetLastError() == cudaSuccess ? 0 : -2; }

// The vectorized element-wise kernels index with 32-bit integers.
bool fits32(long long elements) { return elements < (1LL << 31); }

// Convolution path: 0 = the warp-specialized kernel (cin != 8), else the
// single-buffered tensor-memory kernel where its weights are staged in at most
// two passes, else the mma.sync kernel; 1 = mma.sync only;
// 2 = single-buffered tensor-memory kernel only; 3 = pipelined only; 4 = warp-specialized
// (TMA-fed) only.
int g_conv_impl = 0;

constexpr int kSmemPerSM = 233472;      // bytes of shared memory per SM
constexpr int kSmemPerBlockMax = 232448;
constexpr int kSmemReserved = 1024;     // per resident block

// Tile plan of the UMMA kernel; false when the shape is outside it (cout a
// multiple of 16 up to 192, cin 8 or a multiple of 16 up to 96).
bool umma_plan(const ConvShape& s, UmmaConv& u, int& smem, int& ctas_per_sm) {
    if (s.cout % 16 || s.cout < 16 || s.cout > 192) return false;
    if (!(s.cin == 8 || (s.cin % 16 == 0 && s.cin <= 96))) return false;
    const int cpt = s.cin / 8;
    u.s = s;
    // taller tiles amortize the halo over more MMAs where the halo is small
    // (measured: 12-18 % faster for cin <= 16, cout 16; slower at cout 32)
    u.tz = s.cin <= 16 && s.cout <= 16 ? 4 : (s.cin <= 48 ? 2 : 1);
    const int npos = (u.tz + 2) * kUHY * kUHX;
    u.plane_bytes = (unsigned)npos * 16;
    u.halo_bytes = u.plane_bytes * cpt;
    const int extra = 16;  // mbarrier + tensor-memory address
    const int all_chunks = 27 * cpt + (s.cin == 8 ? 1 : 0);
    const int base = (int)u.halo_bytes + kUSlack + extra;
    const int per_tap = cpt * s.cout * 16 + cpt * 8;  // weights + descriptor table entries
    if (base + all_chunks * (s.cout * 16 + 8) <= kSmemPerBlockMax) {
        u.taps_per_pass = 27;
        u.passes = 1;
        u.w_chunks = (unsigned)all_chunks;
    } else {
        if (s.cin == 8) return false;
        const int taps = (kSmemPerBlockMax - base) / per_tap;
        if (taps < 1) return false;
        u.taps_per_pass = taps;
        u.passes = (27 + taps - 1) / taps;
        u.w_chunks = (unsigned)(taps * cpt);
    }
    u.k_steps = (u.w_chunks + 1) / 2;
    u.ystride = s.cout;
    smem = base + (int)u.w_chunks * s.cout * 16 + (int)u.k_steps * 16;
    unsigned cols = 32;
    while (cols < (unsigned)(u.tz * s.cout)) cols <<= 1;
    u.tmem_cols = cols;
    u.tiles_d = (s.d + u.tz - 1) / u.tz;
    u.tiles_h = (s.h + kUTY - 1) / kUTY;
    u.tiles_w = (s.w + kUTX - 1) / kUTX;
    const long long tiles = (long long)s.n * u.tiles_d * u.tiles_h * u.tiles_w;
    if (tiles > (1LL << 30)) return false;
    u.n_tiles = (int)tiles;
    // resident blocks per SM: shared memory, and at most 512 tensor-memory
    // columns in all (enforced through the shared-memory request, so that an
    // allocation never waits on a block that holds its columns until it exits)
    int by_smem = kSmemPerSM / (smem + kSmemReserved);
    const int by_tmem = 512 / (int)cols;
    if (by_smem > by_tmem) {
        smem = kSmemPerSM / by_tmem - kSmemReserved;
        if (smem > kSmemPerBlockMax) smem = kSmemPerBlockMax;
        by_smem = kSmemPerSM / (smem + kSmemReserved);
    }
    ctas_per_sm = by_smem < 4 ? by_smem : 4;  // the kernel's launch bounds
    return ctas_per_sm >= 1;
}

// Plan of the pipelined variant: the single-pass plan with two halo buffers
// (each with its slack) and two accumulators; false when they do not fit.
bool umma_pipe_plan(const ConvShape& s, UmmaConv& u, int& smem, int& ctas_per_sm) {
    int base_smem = 0, base_per_sm = 0;
    if (!umma_plan(s, u, base_smem, base_per_sm) || u.passes != 1) return false;
    const int extra = 16;
    smem = 2 * ((int)u.halo_bytes + kUSlack) + (int)u.w_chunks * s.cout * 16 + (int)u.k_steps * 16 + extra;
    if (smem > kSmemPerBlockMax || 2 * u.tz * s.cout > 512) return false;
    unsigned cols = 32;
    while (cols < (unsigned)(2 * u.tz * s.cout)) cols <<= 1;
    u.tmem_cols = cols;
    int by_smem = kSmemPerSM / (smem + kSmemReserved);
    const int by_tmem = 512 / (int)cols;
    if (by_smem > by_tmem) {
        smem = kSmemPerSM / by_tmem - kSmemReserved;
        if (smem > kSmemPerBlockMax) smem = kSmemPerBlockMax;
        by_smem = kSmemPerSM / (smem + kSmemReserved);
    }
    ctas_per_sm = by_smem < 4 ? by_smem : 4;
    return ctas_per_sm >= 1;
}

template <int CPT>
int launch_umma_pipe(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias,
                     __nv_bfloat16* y, const UmmaConv& u, int smem, int per_sm, int relu,
                     cudaStream_t st) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -2;
    if (cudaFuncSetAttribute(conv3d_umma_pipe_kernel<CPT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return -2;
    const int grid = u.n_tiles < sms * per_sm ? u.n_tiles : sms * per_sm;
    conv3d_umma_pipe_kernel<CPT><<<grid, 128, smem, st>>>(x, w, bias, y, u, relu);
    return launched();
}

int dispatch_umma_pipe(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias,
                       __nv_bfloat16* y, const UmmaConv& u, int smem, int per_sm, int relu,
                       cudaStream_t st) {
    switch (u.s.cin / 8) {
        case 1: return launch_umma_pipe<1>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 2: return launch_umma_pipe<2>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 4: return launch_umma_pipe<4>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 6: return launch_umma_pipe<6>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 8: return launch_umma_pipe<8>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 12: return launch_umma_pipe<12>(x, w, bias, y, u, smem, per_sm, relu, st);
        default: return -1;
    }
}

// ---- warp-specialized tensor-memory kernel ---------------------------------

// Plan of conv3d_ws_kernel; false when the shape is outside it (cout a multiple
// of 16 up to 256, cin 8 or a multiple of 16) or nothing fits shared memory.
// Weights stay resident where all 27 taps fit beside at least two halo stages;
// the halo of a tile is then split into even channel groups only as far as it
// takes to hold two blocks (two MMA-issuing threads) per SM: one thread issues
// an MMA every ~50 cycles at best, two keep an SM's tensor cores busier
// (decoder level 0, 48 -> 16: 0.89 ms in three groups at two blocks per SM,
// 1.22 ms whole at one).  Otherwise the
// weights are streamed with the stages, in channel groups as large as three
// stages allow (two where three never fit).
bool ws_plan(const ConvShape& s, WsConv& p, int& smem, int& ctas_per_sm) {
    if (s.cout % 16 || s.cout < 16 || s.cout > 256) return false;
    if (!(s.cin == 8 || s.cin % 16 == 0)) return false;
    const int cpt = s.cin / 8, N = s.cout;
    p = WsConv{};
    p.s = s;
    p.tz = s.cin <= 16 && s.cout <= 16 ? 4 : (s.cin <= 48 ? 2 : 1);
    while (p.tz > 1 && 2 * p.tz * N > 512) --p.tz;
    if (2 * p.tz * N > 512) return false;
    p.box_bytes = (unsigned)((p.tz + 2) * kUHY * kUHX * 16);
    p.plane_bytes = (p.box_bytes + 127u) & ~127u;
    auto round128 = [](unsigned v) { return (v + 127u) & ~127u; };
    const int bars = 8 * (2 * kWsMaxStages + 4) + 16;  // mbarriers, TMEM address, flag
    const int pair_smem = kSmemPerSM / 2 - kSmemReserved;
    // resident weights: all channels in one stage if that fits, then smaller
    // groups (three stages) until two blocks fit an SM
    for (int cg = cpt; cg >= 1; --cg) {
        // even groups only (cg = 1 pairs taps, one K step in 28 on a zero chunk,
        // and measured slower than one block per SM with the whole halo)
        if (cpt % cg || (cg % 2 && cg != cpt)) continue;
        const unsigned chunks = 27u * cg + (cg == 1 ? 1u : 0u);  // per group (cg = 1: zero partner)
        const unsigned stage = round128((unsigned)cg * p.plane_bytes + kUSlack);
        const int n_st = cg == cpt ? 2 : 3;
        const long long need = (long long)n_st * stage + (long long)(cpt / cg) * chunks * N * 16 + bars;
        if (need > kSmemPerBlockMax) continue;
        if (p.cg != 0 && need > pair_smem) continue;  // a smaller group only to reach two blocks per SM
        p.cg = cg;
        p.groups = cpt / cg;
        p.stages = n_st;
        p.streamed = 0;
        p.halo_part = (unsigned)cg * p.plane_bytes + kUSlack;
        p.stage_bytes = stage;
        p.w_chunks = chunks;
        p.tx_bytes = (unsigned)cg * p.box_bytes;
        smem = (int)need;
        if (need <= pair_smem) break;
    }
    if (p.cg == 0) {  // streamed weights: the largest channel group with 3 stages, else 2
        for (int want = 3; want >= 2 && p.cg == 0; --want)
            for (int cg = cpt; cg >= 1; --cg) {
                if (cpt % cg || (cg > 1 && cg % 2)) continue;
                const unsigned chunks = 27u * cg + (cg == 1 ? 1u : 0u);
                const unsigned halo = (unsigned)cg * p.plane_bytes + kUSlack;
                const unsigned stage = round128(halo + chunks * N * 16);
                const int fixed = bars;
                int n_st = (kSmemPerBlockMax - fixed) / (int)stage;
                if (n_st > kWsMaxStages) n_st = kWsMaxStages;
                if (n_st < want) continue;
                p.cg = cg;
                p.groups = cpt / cg;
                p.stages = n_st;
                p.streamed = 1;
                p.halo_part = halo;
                p.stage_bytes = stage;
                p.w_chunks = chunks;
                p.tx_bytes = (unsigned)cg * p.box_bytes + 27u * cg * N * 16;
                smem = n_st * (int)stage + fixed;
                break;
            }
        if (p.cg == 0) return false;
    }
    p.acc_cols = (unsigned)(p.tz * N);
    unsigned cols = 32;
    while (cols < 2 * p.acc_cols) cols <<= 1;
    p.tmem_cols = cols;
    p.ystride = N;
    p.tiles_d = (s.d + p.tz - 1) / p.tz;
    p.tiles_h = (s.h + kUTY - 1) / kUTY;
    p.tiles_w = (s.w + kUTX - 1) / kUTX;
    const long long tiles = (long long)s.n * p.tiles_d * p.tiles_h * p.tiles_w;
    if (tiles > (1LL << 30)) return false;
    p.n_tiles = (int)tiles;
    // at most two blocks per SM, and never more than fit 512 tensor-memory
    // columns (enforced through the shared-memory request)
    int by_smem = kSmemPerSM / (smem + kSmemReserved);
    const int by_tmem = 512 / (int)cols;
    int per_sm = by_smem < by_tmem ? by_smem : by_tmem;
    if (per_sm > 2) per_sm = 2;
    if (per_sm < 1) return false;
    if (by_smem > per_sm) {
        smem = kSmemPerSM / per_sm - kSmemReserved;
        if (smem > kSmemPerBlockMax) smem = kSmemPerBlockMax;
    }
    ctas_per_sm = per_sm;
    return true;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, found once through the runtime (no link
// against the driver library); null when the driver does not offer it.
EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// Tensor maps of one launch: the NDHWC bf16 activation (box 8 channels x 10 x
// 18 x (tz + 2) x 1, zero fill outside) and the [cout][kpad] weights (box 8 x
// cout).  False when the driver refuses them (the caller then takes another
// kernel).
// The halo map alone: the NDHWC bf16 activation x of shape s, box 8 channels
// x 10 x 18 x (tz + 2) x 1, zero fill outside.
bool halo_tensor_map(const __nv_bfloat16* x, const ConvShape& s, int tz, CUtensorMap& xm) {
    const EncodeTiledFn enc = encode_tiled();
    if (!enc || reinterpret_cast<uintptr_t>(x) % 16) return false;
    const cuuint64_t e = sizeof(__nv_bfloat16);
    const cuuint64_t xdim[5] = {(cuuint64_t)s.cin, (cuuint64_t)s.w, (cuuint64_t)s.h, (cuuint64_t)s.d,
                                (cuuint64_t)s.n};
    const cuuint64_t xstride[4] = {xdim[0] * e, xdim[0] * xdim[1] * e, xdim[0] * xdim[1] * xdim[2] * e,
                                   xdim[0] * xdim[1] * xdim[2] * xdim[3] * e};
    const cuuint32_t xbox[5] = {8, (cuuint32_t)kUHX, (cuuint32_t)kUHY, (cuuint32_t)(tz + 2), 1};
    const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
    return enc(&xm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(x), xdim, xstride, xbox,
               ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool ws_tensor_maps(const __nv_bfloat16* x, const __nv_bfloat16* w, const WsConv& p, CUtensorMap& xm,
                    CUtensorMap& wm) {
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    if (reinterpret_cast<uintptr_t>(x) % 16 || reinterpret_cast<uintptr_t>(w) % 16) return false;
    const ConvShape& s = p.s;
    const cuuint64_t e = sizeof(__nv_bfloat16);
    const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
    if (!halo_tensor_map(x, s, p.tz, xm)) return false;
    const cuuint64_t wdim[2] = {(cuuint64_t)s.kpad, (cuuint64_t)s.cout};
    const cuuint64_t wstride[1] = {(cuuint64_t)s.kpad * e};
    const cuuint32_t wbox[2] = {8, (cuuint32_t)s.cout};
    return enc(&wm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(w), wdim, wstride, wbox,
               ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CG>
int launch_ws(const CUtensorMap& xm, const CUtensorMap& wm, const __nv_bfloat16* w, const float* bias,
              __nv_bfloat16* y, const WsConv& p, int smem, int per_sm, int relu, cudaStream_t st,
              const WsHead& head) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(conv3d_ws_kernel<CG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
            cudaSuccess)
        return -2;
    const int grid = p.n_tiles < sms * per_sm ? p.n_tiles : sms * per_sm;
    conv3d_ws_kernel<CG><<<grid, kWsThreads, smem, st>>>(xm, wm, w, bias, y, p, relu, head);
    return launched();
}

// 1 launched (code: 0, or -2 from launched()), -1 when the plan or the tensor
// maps do not cover the call.
int try_ws(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* y,
           const ConvShape& s, int relu, cudaStream_t st, int& code, const WsHead& head = WsHead{}) {
    WsConv p{};
    int smem = 0, per_sm = 0;
    CUtensorMap xm, wm;
    if (!ws_plan(s, p, smem, per_sm) || !ws_tensor_maps(x, w, p, xm, wm)) return -1;
    switch (p.cg) {
        case 1: code = launch_ws<1>(xm, wm, w, bias, y, p, smem, per_sm, relu, st, head); return 1;
        case 2: code = launch_ws<2>(xm, wm, w, bias, y, p, smem, per_sm, relu, st, head); return 1;
        case 4: code = launch_ws<4>(xm, wm, w, bias, y, p, smem, per_sm, relu, st, head); return 1;
        case 6: code = launch_ws<6>(xm, wm, w, bias, y, p, smem, per_sm, relu, st, head); return 1;
        case 8: code = launch_ws<8>(xm, wm, w, bias, y, p, smem, per_sm, relu, st, head); return 1;
        case 12: code = launch_ws<12>(xm, wm, w, bias, y, p, smem, per_sm, relu, st, head); return 1;
        default: return -1;
    }
}

// ---- weight gradient on the tensor cores ---------------------------------------------
// The plan of conv3d_wgrad_umma_kernel: the largest tile depth (2, else 1) and
// halo channel group (all chunks, else fewer, an even count) for which two or
// three stages fit shared memory; groups of accumulator units (taps, or with
// cin = 8 rows of three taps) as large as 512 tensor-memory columns allow.  False outside the kernel: cout not 16/32/64/128, cin not 8
// or a multiple of 16.
bool wg_plan(const ConvShape& s, WgConv& p, int& smem) {
    if (s.cout != 16 && s.cout != 32 && s.cout != 64 && s.cout != 128) return false;
    if (s.cin != 8 && (s.cin % 16 || s.cin > 256)) return false;
    const int cpt = s.cin / 8;
    p = WgConv{};
    p.s = s;
    p.dx_fold = s.cin == 8 ? 1 : 0;
    p.m64 = s.cout <= 64 ? 1 : 0;
    p.n_units = p.dx_fold ? 9 : 27;
    p.cols_per_unit = p.dx_fold ? 32u : (unsigned)s.cin;
    p.units = 512 / (int)p.cols_per_unit < p.n_units ? 512 / (int)p.cols_per_unit : p.n_units;
    p.unit_groups = (p.n_units + p.units - 1) / p.units;
    unsigned cols = 32;
    while (cols < (unsigned)p.units * p.cols_per_unit) cols *= 2;
    p.tmem_cols = cols;
    p.dy_lbo = (unsigned)(s.cout / 8) * 128u;
    for (int tz = 2; tz >= 1; --tz) {
        const unsigned box = (unsigned)((tz + 2) * kUHY * kUHX * 16);
        const unsigned plane = (box + 127u) / 128u * 128u;
        for (int ncg = cpt; ncg >= 1; --ncg) {
            if (cpt % ncg || (ncg % 2 && !(ncg == 1 && cpt == 1)) || 8 * ncg > 256) continue;
            const unsigned halo = (unsigned)(ncg == 1 ? 2 : ncg) * plane;
            const unsigned dyb = (unsigned)(tz * kUTY) * p.dy_lbo + 2048u;
            const unsigned stage = (halo + dyb + 1023u) / 1024u * 1024u;
            int stages = (kSmemPerBlockMax - 1024) / (int)stage;
            if (stages > 3) stages = 3;
            if (stages < 2) continue;
            p.tz = tz;
            p.tiles_d = (s.d + tz - 1) / tz;
            p.tiles_h = (s.h + kUTY - 1) / kUTY;
            p.tiles_w = (s.w + kUTX - 1) / kUTX;
            p.n_tiles = s.n * p.tiles_d * p.tiles_h * p.tiles_w;
            p.ncg = ncg;
            p.chunk_groups = cpt / ncg;
            p.n_mma = p.dx_fold ? 32 : 8 * ncg;
            p.b_sbo = p.dx_fold ? 16u : plane;
            p.stages = stages;
            p.plane_bytes = plane;
            p.box_bytes = box;
            p.halo_bytes = halo;
            p.dy_bytes = dyb;
            p.stage_bytes = stage;
            p.tx_bytes = (unsigned)ncg * box;
            smem = stages * (int)stage + 1024;
            // one block per SM: its accumulators take all 512 tensor-memory columns
            if (smem < kSmemPerSM / 2 + 1024) smem = kSmemPerSM / 2 + 1024;
            return true;
        }
    }
    return false;
}

// 1 launched (code: 0 or -2), -1 when the plan or the tensor map does not cover the call.
int try_wgrad_umma(const __nv_bfloat16* x, const __nv_bfloat16* g, float* dw, float* db,
                   const ConvShape& s, cudaStream_t st, int& code) {
    WgConv p;
    int smem = 0;
    CUtensorMap xm;
    if (!wg_plan(s, p, smem) || !halo_tensor_map(x, s, p.tz, xm)) return -1;
    if (reinterpret_cast<uintptr_t>(g) % 16 || reinterpret_cast<uintptr_t>(dw) % 16) return -1;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(conv3d_wgrad_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
            cudaSuccess) {
        code = -2;
        return 1;
    }
    int per_group = sms / p.unit_groups;
    if (per_group > p.n_tiles) per_group = p.n_tiles;
    if (per_group < 1) per_group = 1;
    conv3d_wgrad_umma_kernel<<<per_group * p.unit_groups, kWgThreads, smem, st>>>(xm, g, dw, db, p);
    code = launched();
    return 1;
}

template <int CPT>
int launch_umma(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* y,
                const UmmaConv& u, int smem, int per_sm, int relu, cudaStream_t st) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -2;
    if (cudaFuncSetAttribute(conv3d_umma_kernel<CPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
        return -2;
    const int grid = u.n_tiles < sms * per_sm ? u.n_tiles : sms * per_sm;
    conv3d_umma_kernel<CPT><<<grid, 128, smem, st>>>(x, w, bias, y, u, relu);
    return launched();
}

int dispatch_umma(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias,
                  __nv_bfloat16* y, const UmmaConv& u, int smem, int per_sm, int relu,
                  cudaStream_t st) {
    switch (u.s.cin / 8) {
        case 1: return launch_umma<1>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 2: return launch_umma<2>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 4: return launch_umma<4>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 6: return launch_umma<6>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 8: return launch_umma<8>(x, w, bias, y, u, smem, per_sm, relu, st);
        case 12: return launch_umma<12>(x, w, bias, y, u, smem, per_sm, relu, st);
        default: return -1;
    }
}

}  // namespace

extern "C" {

int pmd_conv3d(const void* x, const void* w, const float* bias, void* y, int n, int d, int h, int wd,
               int cin, int cout, int kpad, int relu, void* stream) {
    ConvShape s{n, d, h, wd, cin, cout, kpad};
    if (n < 1 || d < 1 || h < 1 || wd < 1 || cin < 8 || cin % 8 || kpad % 64 || kpad < 27 * cin)
        return -1;
    auto X = (const __nv_bfloat16*)x;
    auto W = (const __nv_bfloat16*)w;
    auto Y = (__nv_bfloat16*)y;
    cudaStream_t st = (cudaStream_t)stream;
    if (g_conv_impl == 4 || (g_conv_impl == 0 && cin != 8)) {
        // the warp-specialized tensor-memory kernel (by default everywhere but
        // the 8-channel input layer, where the single-buffered kernel measured
        // faster)
        int code = 0;
        if (try_ws(X, W, bias, Y, s, relu, st, code) == 1) return code;
        if (g_conv_impl == 4) return -1;
    }
    if (g_conv_impl == 3) {
        // the pipelined tensor-memory kernel (opt-in: measured slower than two
        // single-buffered CTAs per SM on the network's layers)
        UmmaConv u{};
        int smem = 0, per_sm = 0;
        if (umma_pipe_plan(s, u, smem, per_sm))
            return dispatch_umma_pipe(X, W, bias, Y, u, smem, per_sm, relu, st);
        if (g_conv_impl == 3) return -1;
    }
    if (g_conv_impl == 0 || g_conv_impl == 2) {
        // the tensor-memory kernel where its weights are staged in at most two
        // passes (measured: beyond that, and for output-channel slices, the
        // mma.sync kernel is faster)
        UmmaConv u{};
        int smem = 0, per_sm = 0;
        if (umma_plan(s, u, smem, per_sm) && (g_conv_impl == 2 || u.passes <= 2))
            return dispatch_umma(X, W, bias, Y, u, smem, per_sm, relu, st);
        if (g_conv_impl == 2) return -1;
    }
    switch (cout) {
        case 8: launch_conv<8>(X, W, bias, Y, s, relu, st); break;
        case 16: launch_conv<16>(X, W, bias, Y, s, relu, st); break;
        case 32: launch_conv<32>(X, W, bias, Y, s, relu, st); break;
        case 48: launch_conv<48>(X, W, bias, Y, s, relu, st); break;
        case 64: launch_conv<64>(X, W, bias, Y, s, relu, st); break;
        case 96: launch_conv<96>(X, W, bias, Y, s, relu, st); break;
        case 128: launch_conv<128>(X, W, bias, Y, s, relu, st); break;
        case 192: launch_conv<192>(X, W, bias, Y, s, relu, st); break;
        default: return -1;
    }
    return launched();
}

int pmd_conv3d_head(const void* x, const void* w, const float* bias, const float* head_w,
                    const float* head_b, const float* base, float* out, int n, int d, int h, int wd,
                    int cin, int cout, int kpad, int relu, void* stream) {
    ConvShape s{n, d, h, wd, cin, cout, kpad};
    if (n < 1 || d < 1 || h < 1 || wd < 1 || cin < 8 || cin % 8 || kpad % 64 || kpad < 27 * cin ||
        !head_w || !head_b || !out)
        return -1;
    if (g_conv_impl != 0 && g_conv_impl != 4) return -1;
    WsHead head;
    head.w = head_w;
    head.b = head_b;
    head.base = base;
    head.out = out;
    int code = 0;
    if (try_ws((const __nv_bfloat16*)x, (const __nv_bfloat16*)w, bias, nullptr, s, relu,
               (cudaStream_t)stream, code, head) == 1)
        return code;
    return -1;
}

int pmd_conv3d_wgrad_plan(int n, int d, int h, int wd, int cin, int cout, int* info) {
    if (!info || n < 1 || d < 1 || h < 1 || wd < 1 || cin < 8 || cin % 8) return -1;
    ConvShape s{n, d, h, wd, cin, cout, (27 * cin + 63) / 64 * 64};
    WgConv p;
    int smem = 0;
    if (!wg_plan(s, p, smem)) return -1;
    const int v[8] = {p.tz, p.ncg, p.chunk_groups, p.units, p.unit_groups, p.stages, (int)p.stage_bytes,
                      (int)p.tmem_cols};
    for (int i = 0; i < 8; ++i) info[i] = v[i];
    return 0;
}

int pmd_conv3d_plan(int n, int d, int h, int wd, int cin, int cout, int* info) {
    if (!info || n < 1 || d < 1 || h < 1 || wd < 1 || cin < 8 || cin % 8) return -1;
    for (int i = 0; i < 8; ++i) info[i] = 0;
    info[0] = -1;
    ConvShape s{n, d, h, wd, cin, cout, (27 * cin + 63) / 64 * 64};
    WsConv p{};
    UmmaConv u{};
    int smem = 0, per_sm = 0;
    if ((g_conv_impl == 4 || (g_conv_impl == 0 && cin != 8)) && ws_plan(s, p, smem, per_sm)) {
        info[0] = 4;
        info[1] = p.cg;
        info[2] = p.groups;
        info[3] = p.stages;
        info[4] = p.streamed;
        info[5] = p.tz;
        info[6] = per_sm;
        info[7] = smem;
        return 0;
    }
    if (g_conv_impl == 4) return 0;
    if (g_conv_impl == 3) {
        if (umma_pipe_plan(s, u, smem, per_sm)) info[0] = 3;
        return 0;
    }
    if ((g_conv_impl == 0 || g_conv_impl == 2) && umma_plan(s, u, smem, per_sm) &&
        (g_conv_impl == 2 || u.passes <= 2)) {
        info[0] = 2;
        info[5] = u.tz;
        info[6] = per_sm;
        info[7] = smem;
        return 0;
    }
    if (g_conv_impl == 2) return 0;
    switch (cout) {
        case 8: case 16: case 32: case 48: case 64: case 96: case 128: case 192: info[0] = 1; break;
        default: break;
    }
    return 0;
}

int pmd_conv3d_impl(int impl) {
    const int previous = g_conv_impl;
    if (impl >= 0 && impl <= 4) g_conv_impl = impl;
    return previous;
}

int pmd_conv3d_failures(void) {
    int n = 0;
    if (cudaMemcpyFromSymbol(&n, g_umma_failures, sizeof(int)) != cudaSuccess) return -2;
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_umma_failures, &zero, sizeof(int)) != cudaSuccess) return -2;
    return n;
}

int pmd_conv3d_wgrad(const void* x, const void* g, float* dw, float* dbias, int n, int d, int h,
                     int wd, int cin, int cout, int kpad, void* stream) {
    ConvShape s{n, d, h, wd, cin, cout, kpad};
    if (n < 1 || d < 1 || h < 1 || wd < 1 || cin < 8 || cin % 8 || kpad % kWK || kpad < 27 * cin)
        return -1;
    auto X = (const __nv_bfloat16*)x;
    auto G = (const __nv_bfloat16*)g;
    cudaStream_t st = (cudaStream_t)stream;
    if (g_conv_impl != 1) {  // the tensor-core kernel unless mma.sync is selected
        int code = 0;
        if (try_wgrad_umma(X, G, dw, dbias, s, st, code) == 1) return code;
    }
    switch (cout) {
        case 16: launch_wgrad<16>(X, G, dw, dbias, s, st); break;
        case 32: launch_wgrad<32>(X, G, dw, dbias, s, st); break;
        case 64: launch_wgrad<64>(X, G, dw, dbias, s, st); break;
        case 128: launch_wgrad<128>(X, G, dw, dbias, s, st); break;
        default: return -1;
    }
    return launched();
}

int pmd_flip_weights(const void* w, void* wd, int cin, int cout, int kpad, int kpad_d, void* stream) {
    if (cin < 1 || cout < 1 || kpad < 27 * cin || kpad_d < 27 * cout) return -1;
    flip_weights_kernel<<<grid_for((long long)cin * kpad_d), 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)w, (__nv_bfloat16*)wd, cin, cout, kpad, kpad_d);
    return launched();
}

int pmd_relu_mask(void* g, const void* y, int64_t n, void* stream) {
    if (n % 8) return -1;
    relu_mask_kernel<<<grid_for(n / 8), 256, 0, (cudaStream_t)stream>>>((uint4*)g, (const uint4*)y,
                                                                        n / 8);
    return launched();
}

int pmd_avgpool(const void* x, void* y, int n, int d, int h, int w, int c, void* stream) {
    if (d % 2 || h % 2 || w % 2 || c % 8 || !fits32((long long)n * d * h * w * c)) return -1;
    avgpool_kernel<<<grid_for((long long)n * d * h * w * c / 64), 256, 0, (cudaStream_t)stream>>>(
        (const uint4*)x, (uint4*)y, n, d, h, w, c / 8);
    return launched();
}

int pmd_avgpool_grad(const void* gy, void* gx, int n, int d, int h, int w, int c, int accumulate,
                     void* stream) {
    if (d % 2 || h % 2 || w % 2 || c % 8 || !fits32((long long)n * d * h * w * c)) return -1;
    avgpool_grad_kernel<<<grid_for((long long)n * d * h * w * c / 8), 256, 0, (cudaStream_t)stream>>>(
        (const uint4*)gy, (uint4*)gx, n, d, h, w, c / 8, accumulate);
    return launched();
}

int pmd_upcat(const void* up, const void* skip, void* out, int n, int d, int h, int w, int c_up,
              int c_skip, void* stream) {
    if (d % 2 || h % 2 || w % 2 || c_skip < 8 || c_up < 8 || c_up % 8 || c_skip % 8 ||
        !fits32((long long)n * d * h * w * (c_up + c_skip)))
        return -1;
    upcat_kernel<<<grid_for((long long)n * d * h * w * (c_up + c_skip) / 8), 256, 0,
                   (cudaStream_t)stream>>>((const uint4*)up, (const uint4*)skip, (uint4*)out, n, d,
                                           h, w, c_up / 8, c_skip / 8);
    return launched();
}

int pmd_upcat_grad(const void* gout, void* gup, void* gskip, int n, int d, int h, int w, int c_up,
                   int c_skip, int accumulate, void* stream) {
    if (d % 2 || h % 2 || w % 2 || c_skip < 8 || c_up < 8 || c_up % 8 || c_skip % 8 ||
        !fits32((long long)n * d * h * w * (c_up + c_skip)))
        return -1;
    const long long total = ((long long)n * d * h * w * c_skip + (long long)n * d * h * w * c_up / 8) / 8;
    upcat_grad_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        (const uint4*)gout, (uint4*)gup, (uint4*)gskip, n, d, h, w, c_up / 8, c_skip / 8, accumulate);
    return launched();
}

int pmd_head(const void* f, const float* w, const float* b, const float* base, float* out,
             int64_t m, int c, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    switch (c) {
        case 8: head_kernel<8><<<grid_for(m), 256, 0, st>>>((const uint4*)f, w, b, base, out, m); break;
        case 16: head_kernel<16><<<grid_for(m), 256, 0, st>>>((const uint4*)f, w, b, base, out, m); break;
        case 32: head_kernel<32><<<grid_for(m), 256, 0, st>>>((const uint4*)f, w, b, base, out, m); break;
        case 64: head_kernel<64><<<grid_for(m), 256, 0, st>>>((const uint4*)f, w, b, base, out, m); break;
        default: return -1;
    }
    return launched();
}

int pmd_head_grad(const void* f, const float* w, const float* g, void* df, float* dw, float* db,
                  int64_t m, int c, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    auto F = (const uint4*)f;
    auto DF = (uint4*)df;
    const int head_grid = grid_for(m) < 148 * 4 ? grid_for(m) : 148 * 4;  // 256 threads = 8 warps
    switch (c) {
        case 8: head_grad_kernel<8><<<head_grid, 256, 0, st>>>(F, w, g, DF, dw, db, m); break;
        case 16: head_grad_kernel<16><<<head_grid, 256, 0, st>>>(F, w, g, DF, dw, db, m); break;
        case 32: head_grad_kernel<32><<<head_grid, 256, 0, st>>>(F, w, g, DF, dw, db, m); break;
        case 64: head_grad_kernel<64><<<head_grid, 256, 0, st>>>(F, w, g, DF, dw, db, m); break;
        default: return -1;
    }
    return launched();
}

int pmd_loss(const float* pred, const float* target, const float* weight, float lambda,
             float* grad, float* loss, int64_t m, void* stream) {
    const int grid = grid_for(m) < 148 * 4 ? grid_for(m) : 148 * 4;
    loss_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(pred, target, weight, lambda, grad, loss, m);
    return launched();
}

int pmd_adam(float* p, const float* g, float* m, float* v, void* p16, int64_t n, float lr,
             float beta1, float beta2, float eps, int step, void* stream) {
    if (step < 1) return -1;
    const float bc1 = 1.0f - powf(beta1, (float)step);
    const float bc2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, (__nv_bfloat16*)p16, n, lr,
                                                                beta1, beta2, eps, bc1, bc2);
    return launched();
}

int pmd_pack_input(const float* dose, const float* density, const float* sigma,
                   const float* colmax, int64_t vox, int density_shared, void* x, float* base,
                   int64_t m, void* stream) {
    if (vox < 1) return -1;
    pack_input_kernel<<<grid_for(m), 256, 0, (cudaStream_t)stream>>>(
        dose, density, sigma, colmax, vox, density_shared, (__nv_bfloat16*)x, base, m);
    return launched();
}

int pmd_csc_to_dense(const int64_t* indptr, const int64_t* indices, const double* values,
                     int n_cols, int64_t vox, float* dense, float* colmax, void* stream) {
    if (n_cols < 0 || n_cols > 65535 || vox < 1) return -1;
    if (n_cols == 0) return 0;
    csc_to_dense_kernel<<<dim3(64, n_cols), 256, 0, (cudaStream_t)stream>>>(indptr, indices, values,
                                                                            vox, dense, colmax);
    return launched();
}

int pmd_unscale(const float* out, const float* colmax, int64_t vox, double* mean, int64_t m,
                void* stream) {
    if (vox < 1) return -1;
    unscale_kernel<<<grid_for(m), 256, 0, (cudaStream_t)stream>>>(out, colmax, vox, mean, m);
    return launched();
}

int pmd_csc_to_dense_f64(const int64_t* indptr, const int64_t* indices, const double* values,
                         int n_cols, int64_t vox, double* dense, void* stream) {
    if (n_cols < 0 || n_cols > 65535 || vox < 1) return -1;
    if (n_cols == 0) return 0;
    csc_to_dense_f64_kernel<<<dim3(64, n_cols), 256, 0, (cudaStream_t)stream>>>(indptr, indices,
                                                                                values, vox, dense);
    return launched();
}

int pmd_gather_windows(const float* src, int64_t src_stride, int nx, int ny, int nz,
                       const int32_t* origins, int n_windows, int wx, int wy, int wz, float* out,
                       void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || wx < 1 || wy < 1 || wz < 1 || n_windows < 0 || src_stride < 0)
        return -1;
    const long long total = (long long)n_windows * wx * wy * wz;
    if (total == 0) return 0;
    gather_windows_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        src, src_stride, nx, ny, nz, origins, wx, wy, wz, out, total);
    return launched();
}

int pmd_scatter_windows(const float* win, const float* scale, int nx, int ny, int nz,
                        const int32_t* origins, int n_windows, int wx, int wy, int wz, double* dst,
                        int64_t dst_stride, void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || wx < 1 || wy < 1 || wz < 1 || n_windows < 0 || dst_stride < 0)
        return -1;
    const long long total = (long long)n_windows * wx * wy * wz;
    if (total == 0) return 0;
    scatter_windows_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        win, scale, nx, ny, nz, origins, wx, wy, wz, dst, dst_stride, total);
    return launched();
}

int pmd_gather_windows_oriented(const float* src, int64_t src_stride, int nx, int ny, int nz,
                                const int32_t* win, int n_windows, int wa, int wb, int wd, float* out,
                                void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || wa < 1 || wb < 1 || wd < 1 || n_windows < 0 || src_stride < 0)
        return -1;
    const long long total = (long long)n_windows * wa * wb * wd;
    if (total == 0) return 0;
    gather_oriented_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        src, src_stride, nx, ny, nz, win, wa, wb, wd, out, total);
    return launched();
}

int pmd_scatter_windows_oriented(const float* data, const float* scale, int nx, int ny, int nz,
                                 const int32_t* win, int n_windows, int wa, int wb, int wd, double* dst,
                                 int64_t dst_stride, void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || wa < 1 || wb < 1 || wd < 1 || n_windows < 0 || dst_stride < 0)
        return -1;
    const long long total = (long long)n_windows * wa * wb * wd;
    if (total == 0) return 0;
    scatter_oriented_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        data, scale, nx, ny, nz, win, wa, wb, wd, dst, dst_stride, total);
    return launched();
}

}  // extern "C"
