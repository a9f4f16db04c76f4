// mlp.cu — the surrogate network's tensor-core kernels (sm_100a).
//
// D[M,N] = A[M,K] * B[N,K]^T with BF16 operands and FP32 accumulation on the
// 5th-generation tensor cores:
//   * one CTA per 128 x BN tile of D (BN = 64 or 256), 128 threads;
//   * A and B tiles (64 K-columns, 128-byte rows) move global -> shared by
//     TMA (cp.async.bulk.tensor.2d, 128-byte swizzle), two stages, completed
//     on mbarriers;
//   * one elected thread issues tcgen05.mma (kind::f16, M=128, N=BN, K=16
//     per instruction) into a TMEM accumulator and commits each stage to an
//     mbarrier, which frees the stage for the next TMA load;
//   * the four warps read the accumulator back with tcgen05.ld (warp w owns
//     TMEM lanes 32w..32w+31, i.e. rows of the tile) and run the fused
//     epilogue: bias + GELU (forward, also storing the pre-activation and
//     the transposed activation for the weight gradient), bias only (the
//     output layer), GELU' times the incoming gradient (backward), or plain
//     FP32 (weight gradients).
// Every operand is K-major; the backward pass gets its transposed operands
// from the transposed copies the epilogues and the optimiser write, so no
// MN-major descriptor is needed. All waits are bounded: a timeout sets *err,
// waits (bounded) for the copies and MMAs already issued, frees the TMEM and
// returns. No multicast load is used.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <string.h>

#include <mutex>

#include "engine.h"
#include "lcg.h"
#include "mlp_tc.cuh"
#include "tma.cuh"

namespace lcg {
namespace {

using namespace mlp;

struct GemmOut {
    const float *bias;   // [N] or NULL
    __nv_bfloat16 *z;    // forward GELU: pre-activation out; backward: pre-activation in
    __nv_bfloat16 *y;    // bf16 [M x N]
    __nv_bfloat16 *yt;   // bf16 [N x ldt], the transpose of y
    float *out;          // f32 [M x N]
    int32_t n, mvalid, ldt;
    int32_t *err;
};

template <int BN, int EPI>
__global__ void __launch_bounds__(128) k_gemm(const __grid_constant__ CUtensorMap ta,
                                              const __grid_constant__ CUtensorMap tb, int32_t k,
                                              GemmOut o) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2;
    __shared__ uint64_t full[2], done[2];
    __shared__ uint32_t tmem_base;
    __shared__ int ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
    unsigned char *sa0 = smem, *sb0 = smem + 2 * kABytes;
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(&done[0], 1);
        mbar_init(&done[1], 1);
        ok = 1;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base;
    const int nk = k / kBK;          // k: the K slice of this CTA
    const int k0 = blockIdx.z * k;   // split-K: slices along grid z
    if (tid == 0) {
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(kBM >> 4) << 24);
        int issued = 0, consumed = 0, committed = 0;
        auto load = [&](int kb) {
            const int s = kb & 1;
            mbar_arrive_expect_tx(&full[s], kABytes + kBBytes);
            tma_load_2d(sa0 + s * kABytes, &ta, k0 + kb * kBK, m0, &full[s]);
            tma_load_2d(sb0 + s * kBBytes, &tb, k0 + kb * kBK, n0, &full[s]);
            issued++;
        };
        load(0);
        if (nk > 1) load(1);
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb & 1;
            const uint32_t par = (kb >> 1) & 1;
            if (!mbar_wait_bounded(&full[s], par)) {
                ok = 0;
                break;
            }
            consumed++;
            fence_after_sync();
            const uint64_t ad = desc_sw128(smem_u32(sa0 + s * kABytes));
            const uint64_t bd = desc_sw128(smem_u32(sb0 + s * kBBytes));
#pragma unroll
            for (int kk = 0; kk < kBK / 16; kk++)  // +32 B per K16 slice
                mma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) ? 1u : 0u);
            mma_commit(&done[s]);
            committed++;
            if (kb + 2 < nk) {
                if (!mbar_wait_bounded(&done[s], par)) {
                    ok = 0;
                    break;
                }
                load(kb + 2);
            }
        }
        if (!ok) {
            // drain what is in flight before the TMEM and the barriers go away
            for (int kb = consumed; kb < issued; kb++)
                mbar_wait_bounded(&full[kb & 1], (kb >> 1) & 1);
            if (committed > 0)
                mbar_wait_bounded(&done[(committed - 1) & 1], ((committed - 1) >> 1) & 1);
            if (o.err) atomicExch(o.err, 1);
        }
    }
    __syncthreads();
    bool run = ok != 0;
    if (run) {
        const int last = nk - 1;
        if (!mbar_wait_bounded(&done[last & 1], (last >> 1) & 1)) {
            if (o.err) atomicExch(o.err, 2);
            run = false;
        }
    }
    fence_after_sync();
    if (run) {
        const int r = 32 * warp + lane, m = m0 + r;
        const bool store = m < o.mvalid;
        const int N = o.n;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            const int nb = n0 + c0;
            if (o.bias) {
#pragma unroll
                for (int i = 0; i < 16; i++) v[i] += o.bias[nb + i];
            }
            if (EPI == kEpiGelu) {
                __align__(16) __nv_bfloat16 zb[16], yb[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    zb[i] = __float2bfloat16_rn(v[i]);
                    yb[i] = __float2bfloat16_rn(gelu(v[i]));
                }
                if (store) {
                    uint4 *zp = reinterpret_cast<uint4 *>(o.z + (size_t)m * N + nb);
                    uint4 *yp = reinterpret_cast<uint4 *>(o.y + (size_t)m * N + nb);
                    zp[0] = reinterpret_cast<uint4 *>(zb)[0];
                    zp[1] = reinterpret_cast<uint4 *>(zb)[1];
                    yp[0] = reinterpret_cast<uint4 *>(yb)[0];
                    yp[1] = reinterpret_cast<uint4 *>(yb)[1];
                    if (o.yt) {
#pragma unroll
                        for (int i = 0; i < 16; i++) o.yt[(size_t)(nb + i) * o.ldt + m] = yb[i];
                    }
                }
            } else if (EPI == kEpiDGelu) {
                __align__(16) __nv_bfloat16 gb[16];
                if (store) {
                    const uint4 *zp = reinterpret_cast<const uint4 *>(o.z + (size_t)m * N + nb);
                    __align__(16) __nv_bfloat16 zz[16];
                    reinterpret_cast<uint4 *>(zz)[0] = zp[0];
                    reinterpret_cast<uint4 *>(zz)[1] = zp[1];
#pragma unroll
                    for (int i = 0; i < 16; i++)
                        gb[i] = __float2bfloat16_rn(v[i] * gelu_grad(__bfloat162float(zz[i])));
                    uint4 *yp = reinterpret_cast<uint4 *>(o.y + (size_t)m * N + nb);
                    yp[0] = reinterpret_cast<uint4 *>(gb)[0];
                    yp[1] = reinterpret_cast<uint4 *>(gb)[1];
                    if (o.yt) {
#pragma unroll
                        for (int i = 0; i < 16; i++) o.yt[(size_t)(nb + i) * o.ldt + m] = gb[i];
                    }
                }
            } else if (EPI == kEpiF32 && gridDim.z > 1) {
                // split-K: slices add into the output the launcher zeroed
                if (store) {
                    float *op = o.out + (size_t)m * N + nb;
#pragma unroll
                    for (int i = 0; i < 16; i++) atomicAdd(op + i, v[i]);
                }
            } else {  // kEpiLinear, kEpiF32
                if (store) {
                    float4 *op = reinterpret_cast<float4 *>(o.out + (size_t)m * N + nb);
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        op[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN)
                     : "memory");
    }
}

// ---- optimiser and small kernels ---------------------------------------------

// Adam on FP32 master weights [rows x cols]; writes the BF16 weights and
// their transpose.
__global__ void k_adam(float *w, float *m, float *v, const float *g, int32_t rows, int32_t cols,
                       float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16 *wb, __nv_bfloat16 *wt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)rows * cols) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    const __nv_bfloat16 b = __float2bfloat16_rn(wi);
    if (wb) wb[i] = b;
    if (wt) {
        const int64_t r = i / cols, c = i % cols;
        wt[c * rows + r] = b;
    }
}

// Column sums of a BF16 [rows x cols] matrix (bias gradients), FP32: a
// block of 32 columns x 32 row groups, each thread summing rows ty, ty + 32,
// ... in order, then a fixed-order tree over the groups (deterministic).
__global__ void k_colsum(const __nv_bfloat16 *g, int32_t rows, int32_t cols, int32_t rvalid,
                         float *out) {
    __shared__ float sh[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int c = blockIdx.x * 32 + tx;
    float s = 0.f;
    if (c < cols)
        for (int r = ty; r < rvalid; r += 32) s += __bfloat162float(g[(size_t)r * cols + c]);
    sh[ty][tx] = s;
    __syncthreads();
    for (int w = 16; w > 0; w >>= 1) {
        if (ty < w) sh[ty][tx] += sh[ty + w][tx];
        __syncthreads();
    }
    if (ty == 0 && c < cols) out[c] = sh[0][tx];
}

// One Adam step over up to kAdamMax tensors in one launch. The learning
// rate follows a cosine schedule read from device memory together with the
// number of steps taken, so a captured graph serves every step:
//   sched = {lr_max, lr_min, total_steps, beta1, beta2, eps}
//   lr(k) = lr_min + (lr_max - lr_min) (1 + cos(pi k / total)) / 2
//           (lr_max when total <= 0), bias corrections 1 - beta^(k + 1).
constexpr int kAdamMax = 16;
struct AdamSet {
    float *w[kAdamMax], *m1[kAdamMax], *m2[kAdamMax];
    const float *g[kAdamMax];
    __nv_bfloat16 *wb[kAdamMax], *wt[kAdamMax];
    int32_t rows[kAdamMax], cols[kAdamMax];
    int64_t start[kAdamMax + 1];
    int32_t n;
};

__global__ void k_adam_all(const __grid_constant__ AdamSet a, const float *sched,
                           const int32_t *step) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= a.start[a.n]) return;
    int j = 0;
    while (i >= a.start[j + 1]) j++;
    const int64_t e = i - a.start[j];
    const int k = *step;
    const float lr_max = sched[0], lr_min = sched[1], total = sched[2];
    const float b1 = sched[3], b2 = sched[4], eps = sched[5];
    const float lr = total > 0.f
                         ? lr_min + 0.5f * (lr_max - lr_min) *
                                        (1.f + cosf(3.14159265358979f * (float)k / total))
                         : lr_max;
    const float c1 = 1.f - powf(b1, (float)(k + 1)), c2 = 1.f - powf(b2, (float)(k + 1));
    const float gi = a.g[j][e];
    const float mi = b1 * a.m1[j][e] + (1.f - b1) * gi;
    const float vi = b2 * a.m2[j][e] + (1.f - b2) * gi * gi;
    a.m1[j][e] = mi;
    a.m2[j][e] = vi;
    const float wi = a.w[j][e] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    a.w[j][e] = wi;
    const __nv_bfloat16 b = __float2bfloat16_rn(wi);
    if (a.wb[j]) a.wb[j][e] = b;
    if (a.wt[j]) {
        const int64_t r = e / a.cols[j], c = e % a.cols[j];
        a.wt[j][c * a.rows[j] + r] = b;
    }
}

// Mean-squared-error gradient of out [rows x cols] against target, scaled by
// 2 / (rvalid * cols), as BF16 and transposed BF16 (ldt columns); also the
// per-row loss sums.
__global__ void k_mse_grad(const float *out, const float *target, int32_t rows, int32_t cols,
                           int32_t rvalid, int32_t ldt, __nv_bfloat16 *g, __nv_bfloat16 *gt,
                           float *loss_rows) {
    const int r = blockIdx.x;
    const int c = threadIdx.x;
    float d = 0.f;
    if (r < rvalid && c < cols) d = out[(size_t)r * cols + c] - target[(size_t)r * cols + c];
    if (c < cols) {
        const __nv_bfloat16 b = __float2bfloat16_rn(2.f * d / ((float)rvalid * cols));
        g[(size_t)r * cols + c] = b;
        gt[(size_t)c * ldt + r] = b;
    }
    __shared__ float sh[256];
    sh[c] = d * d;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (c < w) sh[c] += sh[c + w];
        __syncthreads();
    }
    if (c == 0 && loss_rows) loss_rows[r] = sh[0];
}

// Input layer in FP32 (kin <= 16 inputs): z = x W^T + b, y = GELU(z), one
// thread per (row, unit); stores z, y (BF16) and y^T (row stride ldt).
__global__ void k_input_fwd(const float *x, int32_t kin, const float *w, const float *b,
                            int32_t m, int32_t n, int32_t mvalid, __nv_bfloat16 *z,
                            __nv_bfloat16 *y, __nv_bfloat16 *yt, int32_t ldt) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;  // unit
    const int r = blockIdx.y;                             // row
    if (u >= n || r >= m) return;
    float acc = b ? b[u] : 0.f;
    if (r < mvalid)
        for (int k = 0; k < kin; k++) acc = fmaf(x[(size_t)r * kin + k], w[(size_t)u * kin + k], acc);
    else
        acc = 0.f;
    const __nv_bfloat16 zb = __float2bfloat16_rn(acc), yb = __float2bfloat16_rn(gelu(acc));
    if (z) z[(size_t)r * n + u] = zb;
    y[(size_t)r * n + u] = yb;
    if (yt) yt[(size_t)u * ldt + r] = yb;
}

// dW[u][k] = sum over the first mvalid rows of g[r][u] * x[r][k]: one block
// per unit, a fixed-order tree over the block.
__global__ void k_input_grad(const __nv_bfloat16 *g, const float *x, int32_t kin, int32_t m,
                             int32_t n, int32_t mvalid, float *dw) {
    __shared__ float sh[16][256];
    const int u = blockIdx.x, t = threadIdx.x;
    float acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.f;
    for (int r = t; r < mvalid; r += 256) {
        const float gv = __bfloat162float(g[(size_t)r * n + u]);
        for (int k = 0; k < kin; k++) acc[k] = fmaf(gv, x[(size_t)r * kin + k], acc[k]);
    }
    for (int k = 0; k < kin; k++) sh[k][t] = acc[k];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w)
            for (int k = 0; k < kin; k++) sh[k][t] += sh[k][t + w];
        __syncthreads();
    }
    if (t < kin) dw[(size_t)u * kin + t] = sh[t][0];
}

// Light curve from PCA coefficients and its chi**2 after the optimal scale
// (re_scale.cpp:16-42 and light_curve_comp.cpp:557-585):
//   s(c)[p] = mean[p] + sum_k c[k] * basis[k][p]
//   f[p]    = s(coef)[p], or anchor[p] * s(coef)[p] / s(coef_x)[p] when an
//             anchor curve (an exact curve at the point coef_x describes) is
//             given: the surrogate's relative change applied to it.
// One block per row, FP64 sums.
__device__ __forceinline__ double pca_curve(const float *sc, const float *sx, int32_t ncoef,
                                            const float *basis, const float *mean,
                                            int32_t npts, const double *anchor, int p) {
    float f = mean[p];
    for (int k = 0; k < ncoef; k++) f = fmaf(sc[k], basis[(size_t)k * npts + p], f);
    if (!anchor) return f;
    float g = mean[p];
    for (int k = 0; k < ncoef; k++) g = fmaf(sx[k], basis[(size_t)k * npts + p], g);
    return anchor[p] * ((double)f / (double)g);
}

__global__ void k_pca_chisq(const float *coef, int32_t ncoef, const float *basis,
                            const float *mean, int32_t npts, const double *flux,
                            const double *ferr, const double *weight, const float *coef_x,
                            const double *anchor, double *chisq, double *scale) {
    extern __shared__ float sc[];  // coef row, then the coef_x row
    __shared__ double red[3][256];
    const int r = blockIdx.x, t = threadIdx.x;
    float *sx = sc + ncoef;
    for (int k = t; k < ncoef; k += blockDim.x) {
        sc[k] = coef[(size_t)r * ncoef + k];
        if (anchor) sx[k] = coef_x[(size_t)r * ncoef + k];
    }
    const double *an = anchor ? anchor + (size_t)r * npts : nullptr;
    __syncthreads();
    double a = 0., bb = 0.;
    for (int p = t; p < npts; p += blockDim.x) {
        const double f = pca_curve(sc, sx, ncoef, basis, mean, npts, an, p);
        if (weight[p] > 0.) {
            const double wgt = weight[p] / (ferr[p] * ferr[p]);
            a += wgt * flux[p] * f;
            bb += wgt * (double)f * f;
        }
    }
    red[0][t] = a;
    red[1][t] = bb;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w) {
            red[0][t] += red[0][t + w];
            red[1][t] += red[1][t + w];
        }
        __syncthreads();
    }
    const double s = red[1][0] > 0. ? red[0][0] / red[1][0] : 1.;
    __syncthreads();
    double cs = 0.;
    for (int p = t; p < npts; p += blockDim.x) {
        const double f = pca_curve(sc, sx, ncoef, basis, mean, npts, an, p);
        if (weight[p] > 0.) {
            const double d = (flux[p] - s * f) / ferr[p];
            cs += weight[p] * d * d;
        }
    }
    red[2][t] = cs;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w) red[2][t] += red[2][t + w];
        __syncthreads();
    }
    if (t == 0) {
        chisq[r] = red[2][0];
        if (scale) scale[r] = s;
    }
}

}  // namespace

namespace mlp {
namespace {
using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                             cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}

}  // namespace

bool make_map(CUtensorMap *map, const void *base, int32_t rows, int32_t cols, int32_t box_rows) {
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace mlp

namespace {

template <int BN, int EPI>
cudaError_t launch_gemm_t(const CUtensorMap &ta, const CUtensorMap &tb, int m, int n, int k,
                          int splits, const GemmOut &o, cudaStream_t s) {
    const size_t smem = 2 * (size_t)(kBM + BN) * kBK * 2 + 1024;
    auto kern = k_gemm<BN, EPI>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    if (splits > 1) {
        e = cudaMemsetAsync(o.out, 0, (size_t)o.mvalid * n * sizeof(float), s);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((unsigned)(n / BN), (unsigned)(m / kBM), (unsigned)splits);
    kern<<<grid, 128, smem, s>>>(ta, tb, k / splits, o);
    count_launch();
    return cudaGetLastError();
}

}  // namespace
}  // namespace lcg

using namespace lcg;

extern "C" {

lcg_status lcg_mlp_gemm(void *stream, int32_t epi, int32_t m, int32_t n, int32_t k,
                        const void *a, const void *b, const float *bias, void *z, void *y,
                        void *yt, float *out, int32_t mvalid, int32_t ldt, int32_t *err) {
    if (!a || !b || m <= 0 || n <= 0 || k <= 0 || m % kBM || k % kBK || epi < 0 || epi > 3)
        return LCG_E_INVALID;
    if (n % 64) return LCG_E_INVALID;
    // 256-wide tiles unless that leaves most SMs idle; split K across CTAs for
    // the weight gradients (FP32 output, long K, few tiles)
    int nsm = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int bn = (n % 256 == 0 && (n / 256) * (m / kBM) >= nsm / 2) ? 256 : 64;
    int splits = 1;
    if (epi == kEpiF32) {
        const int tiles = (n / bn) * (m / kBM);
        while (tiles * splits * 2 <= 2 * nsm && (k / kBK) % (splits * 2) == 0 &&
               k / (splits * 2) >= 4 * kBK)
            splits *= 2;
    }
    if ((epi == kEpiGelu && (!z || !y)) || (epi == kEpiDGelu && (!z || !y)) ||
        ((epi == kEpiLinear || epi == kEpiF32) && !out) || ((yt != nullptr) && ldt < m))
        return LCG_E_INVALID;
    const uintptr_t al = (uintptr_t)a | (uintptr_t)b;
    if (al & 15) return LCG_E_INVALID;  // TMA wants 16-byte aligned bases
    CUtensorMap ta, tb;
    if (!make_map(&ta, a, m, k, kBM) || !make_map(&tb, b, n, k, bn)) return LCG_E_CUDA;
    GemmOut o{bias, (__nv_bfloat16 *)z, (__nv_bfloat16 *)y, (__nv_bfloat16 *)yt, out, n,
              mvalid, ldt, err};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (bn == 256) {
        switch (epi) {
        case kEpiGelu: e = launch_gemm_t<256, kEpiGelu>(ta, tb, m, n, k, splits, o, s); break;
        case kEpiLinear: e = launch_gemm_t<256, kEpiLinear>(ta, tb, m, n, k, splits, o, s); break;
        case kEpiDGelu: e = launch_gemm_t<256, kEpiDGelu>(ta, tb, m, n, k, splits, o, s); break;
        default: e = launch_gemm_t<256, kEpiF32>(ta, tb, m, n, k, splits, o, s); break;
        }
    } else {
        switch (epi) {
        case kEpiGelu: e = launch_gemm_t<64, kEpiGelu>(ta, tb, m, n, k, splits, o, s); break;
        case kEpiLinear: e = launch_gemm_t<64, kEpiLinear>(ta, tb, m, n, k, splits, o, s); break;
        case kEpiDGelu: e = launch_gemm_t<64, kEpiDGelu>(ta, tb, m, n, k, splits, o, s); break;
        default: e = launch_gemm_t<64, kEpiF32>(ta, tb, m, n, k, splits, o, s); break;
        }
    }
    return e == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_adam(void *stream, float *w, float *m1, float *m2, const float *g,
                        int32_t rows, int32_t cols, float lr, float beta1, float beta2, float eps,
                        int32_t step, void *w_bf16, void *wt_bf16) {
    if (!w || !m1 || !m2 || !g || rows <= 0 || cols <= 0 || step < 1) return LCG_E_INVALID;
    const int64_t n = (int64_t)rows * cols;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        w, m1, m2, g, rows, cols, lr, beta1, beta2, eps, c1, c2, (__nv_bfloat16 *)w_bf16,
        (__nv_bfloat16 *)wt_bf16);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_adam_all(void *stream, int32_t n, float *const *w, float *const *m1,
                            float *const *m2, const float *const *g, const int32_t *rows,
                            const int32_t *cols, void *const *w_bf16, void *const *wt_bf16,
                            const float *sched, const int32_t *step) {
    if (n <= 0 || n > kAdamMax || !w || !m1 || !m2 || !g || !rows || !cols || !sched || !step)
        return LCG_E_INVALID;
    AdamSet a;
    memset(&a, 0, sizeof(a));
    a.n = n;
    a.start[0] = 0;
    for (int j = 0; j < n; j++) {
        if (!w[j] || !m1[j] || !m2[j] || !g[j] || rows[j] <= 0 || cols[j] <= 0)
            return LCG_E_INVALID;
        a.w[j] = w[j];
        a.m1[j] = m1[j];
        a.m2[j] = m2[j];
        a.g[j] = g[j];
        a.wb[j] = w_bf16 ? (__nv_bfloat16 *)w_bf16[j] : nullptr;
        a.wt[j] = wt_bf16 ? (__nv_bfloat16 *)wt_bf16[j] : nullptr;
        a.rows[j] = rows[j];
        a.cols[j] = cols[j];
        a.start[j + 1] = a.start[j] + (int64_t)rows[j] * cols[j];
    }
    k_adam_all<<<(unsigned)((a.start[n] + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a, sched,
                                                                                       step);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_colsum(void *stream, const void *g_bf16, int32_t rows, int32_t cols,
                          int32_t rvalid, float *out) {
    if (!g_bf16 || !out || rows <= 0 || cols <= 0 || rvalid > rows) return LCG_E_INVALID;
    k_colsum<<<(unsigned)((cols + 31) / 32), dim3(32, 32), 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)g_bf16, rows, cols, rvalid, out);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_mse_grad(void *stream, const float *out, const float *target, int32_t rows,
                            int32_t cols, int32_t rvalid, int32_t ldt, void *g_bf16,
                            void *gt_bf16, float *loss_rows) {
    if (!out || !target || !g_bf16 || !gt_bf16 || cols <= 0 || cols > 256 || rows <= 0 ||
        rvalid > rows || ldt < rows)
        return LCG_E_INVALID;
    int t = 32;
    while (t < cols) t <<= 1;
    k_mse_grad<<<(unsigned)rows, t, 0, (cudaStream_t)stream>>>(
        out, target, rows, cols, rvalid, ldt, (__nv_bfloat16 *)g_bf16, (__nv_bfloat16 *)gt_bf16,
        loss_rows);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_input(void *stream, const float *x, int32_t kin, const float *w,
                         const float *b, int32_t m, int32_t n, int32_t mvalid, void *z, void *y,
                         void *yt, int32_t ldt) {
    if (!x || !w || !y || kin <= 0 || kin > 16 || m <= 0 || n <= 0 || mvalid > m ||
        (yt && ldt < m))
        return LCG_E_INVALID;
    dim3 grid((unsigned)((n + 127) / 128), (unsigned)m);
    k_input_fwd<<<grid, 128, 0, (cudaStream_t)stream>>>(x, kin, w, b, m, n, mvalid,
                                                         (__nv_bfloat16 *)z, (__nv_bfloat16 *)y,
                                                         (__nv_bfloat16 *)yt, ldt);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_input_grad(void *stream, const void *g_bf16, const float *x, int32_t kin,
                              int32_t m, int32_t n, int32_t mvalid, float *dw) {
    if (!g_bf16 || !x || !dw || kin <= 0 || kin > 16 || mvalid > m || n <= 0)
        return LCG_E_INVALID;
    k_input_grad<<<(unsigned)n, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)g_bf16, x,
                                                                 kin, m, n, mvalid, dw);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_pca_chisq(void *stream, const float *coef, int32_t m, int32_t ncoef,
                             const float *basis, const float *mean, int32_t npts,
                             const double *flux, const double *ferr, const double *weight,
                             const float *coef_x, const double *anchor, double *chisq,
                             double *scale) {
    if (!coef || !basis || !mean || !flux || !ferr || !weight || !chisq || m <= 0 ||
        ncoef <= 0 || ncoef > 4096 || npts <= 0 || (anchor && !coef_x))
        return LCG_E_INVALID;
    k_pca_chisq<<<(unsigned)m, 256, 2 * (size_t)ncoef * sizeof(float), (cudaStream_t)stream>>>(
        coef, ncoef, basis, mean, npts, flux, ferr, weight, coef_x, anchor, chisq, scale);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

}  // extern "C"
