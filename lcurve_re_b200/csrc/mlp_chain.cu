// mlp_chain.cu — every layer of the surrogate network for a 128-row tile in
// one launch (sm_100a).
//
// One CTA per 128 rows, 512 threads (16 warps). The tile's activations stay
// in shared memory between layers as the A operand of the next tcgen05.mma:
// four 16 KB K-blocks of [128 rows x 64] BF16 in the 128-byte-swizzled
// K-major layout TMA would write. Each layer:
//   * its weights (B operand, [n x K] BF16, K-major) arrive by TMA in up to
//     four 64-column K-blocks, issued while the previous layer's epilogue
//     runs;
//   * one elected thread issues the MMAs (kind::f16, M = 128, N = n, K = 16
//     each) into one TMEM accumulator of n columns and commits them to an
//     mbarrier;
//   * all sixteen warps read the accumulator back (warp w: TMEM lanes
//     32 (w % 4).. = rows, columns quarter w / 4) and run the epilogue, writing
//     the next A operand into shared memory (generic-proxy stores, then a
//     proxy fence before the next MMA reads them).
// Epilogues: bias + GELU (hidden layers; training also stores the
// pre-activation and the transposed activation for the weight gradients),
// bias only (output layer, FP32 out; training fuses the mean-squared-error
// gradient), and incoming gradient times GELU' of the stored pre-activation
// (the backward chain, storing each layer's gradient and its transpose).
// The forward chain starts from the FP32 input layer (nin <= 16) computed
// on the CUDA cores; the backward chain loads its first A operand (the
// output gradient) by TMA. No weight, activation or accumulator leaves the
// SM between layers; no TMEM is allocated or freed between layers.
//
// Every wait is bounded: a timeout sets *err, the CTA drains the copies and
// MMAs it issued (bounded), frees its TMEM and returns. No multicast load.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>

#include "engine.h"
#include "lcg.h"
#include "mlp_tc.cuh"
#include "tma.cuh"

namespace lcg {
namespace mlp {
namespace {

constexpr int kChainMax = 5;          // layers after the first A operand
constexpr int kChainThreads = 512;  // 128 x kGroups: warp w reads TMEM lanes 32 (w % 4)..
constexpr int kGroups = kChainThreads / 128;  // column groups of the epilogue
static_assert(kGroups == 2 || kGroups == 4, "64-column layers need 16-column groups");
constexpr int kSlots = 4;             // weight K-blocks of one layer
constexpr uint32_t kSlotBytes = 256u * kBK * 2;    // the largest B block, [256 x 64]
constexpr uint32_t kABlockBytes = (uint32_t)kBM * kBK * 2;
constexpr int kWidth = 256;           // activation width the tile holds
constexpr size_t kChainSmem = 4 * (size_t)kABlockBytes + kSlots * (size_t)kSlotBytes + 1024;

struct ChainLayer {
    int32_t n, kblocks, epi;
    const float *bias;
    const __nv_bfloat16 *zin;  // kEpiDGelu: pre-activation [m x n]
    __nv_bfloat16 *zout;       // kEpiGelu: pre-activation out [m x n]
    __nv_bfloat16 *y;          // BF16 result [m x n]
    __nv_bfloat16 *yt;         // its transpose [n x ldt]
    float *out;                // kEpiLinear: FP32 [m x n]
};

struct ChainArgs {
    CUtensorMap w[kChainMax];  // B operand of each layer, box 64 x n
    CUtensorMap a0;            // first A operand from global (no input layer), box 64 x 128
    ChainLayer layer[kChainMax];
    int32_t nlayers, a0_kblocks, input_layer;
    const float *x, *w0, *b0;  // FP32 input layer: 256 units, kin inputs
    int32_t kin;
    __nv_bfloat16 *z0, *yt0;
    const float *target;       // kEpiLinear last layer: mean-squared-error gradient
    __nv_bfloat16 *g, *gt;
    float *loss_rows;
    int32_t rvalid, m, mvalid, ldt;
    int32_t *err;
};

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive columns c0.. (c0 % 16 == 0) of one row into the swizzled
// activation tile.
__device__ __forceinline__ void act_store16(unsigned char *act, int row, int c0,
                                            const __nv_bfloat16 (&v)[16]) {
    const int j = (c0 & 63) >> 3, sw = row & 7;
    unsigned char *base = act + (c0 >> 6) * kABlockBytes + row * 128;
    *reinterpret_cast<uint4 *>(base + ((j ^ sw) << 4)) = reinterpret_cast<const uint4 *>(v)[0];
    *reinterpret_cast<uint4 *>(base + (((j + 1) ^ sw) << 4)) =
        reinterpret_cast<const uint4 *>(v)[1];
}

__device__ __forceinline__ void act_store1(unsigned char *act, int row, int c,
                                           __nv_bfloat16 v) {
    unsigned char *base = act + (c >> 6) * kABlockBytes + row * 128;
    *reinterpret_cast<__nv_bfloat16 *>(base + ((((c & 63) >> 3) ^ (row & 7)) << 4) +
                                       (c & 7) * 2) = v;
}

__device__ __forceinline__ void store16(__nv_bfloat16 *p, const __nv_bfloat16 (&v)[16]) {
    reinterpret_cast<uint4 *>(p)[0] = reinterpret_cast<const uint4 *>(v)[0];
    reinterpret_cast<uint4 *>(p)[1] = reinterpret_cast<const uint4 *>(v)[1];
}

__global__ void __launch_bounds__(kChainThreads, 1) k_mlp_chain(const __grid_constant__ ChainArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *act = smem;
    unsigned char *wslot = smem + 4 * kABlockBytes;
    __shared__ uint64_t full[kSlots], accb, abar;
    __shared__ uint32_t tmem_base;
    __shared__ int ok;
    __shared__ __align__(16) float xs[kBM * 16];
    __shared__ float lossp[kGroups][kBM];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + lane;
    const int m0 = blockIdx.x * kBM, m = m0 + row;
    // thread 0's record of the weight loads: parity of each slot's pending
    // load, and which slots have one in flight
    uint32_t uses[kSlots] = {0, 0, 0, 0}, ldpar[kSlots] = {0, 0, 0, 0}, pending = 0;
    bool a0_pending = false;

    if (tid == 0) {
        for (int s = 0; s < kSlots; s++) mbar_init(&full[s], 1);
        mbar_init(&accb, 1);
        mbar_init(&abar, 1);
        ok = 1;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(kWidth)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base;

    auto load_layer = [&](int l) {
        const ChainLayer &L = a.layer[l];
        const uint32_t bytes = (uint32_t)L.n * kBK * 2;
        for (int kb = 0; kb < L.kblocks; kb++) {
            ldpar[kb] = uses[kb] & 1u;
            uses[kb]++;
            pending |= 1u << kb;
            mbar_arrive_expect_tx(&full[kb], bytes);
            tma_load_2d(wslot + kb * kSlotBytes, &a.w[l], kb * kBK, 0, &full[kb]);
        }
    };
    if (tid == 0) {
        load_layer(0);
        if (!a.input_layer) {
            mbar_arrive_expect_tx(&abar, (uint32_t)a.a0_kblocks * kABlockBytes);
            for (int kb = 0; kb < a.a0_kblocks; kb++)
                tma_load_2d(act + kb * kABlockBytes, &a.a0, kb * kBK, m0, &abar);
            a0_pending = true;
        }
    }

    // ---- first A operand ----------------------------------------------------------------
    if (a.input_layer) {
        const int kin = a.kin;
        // the tile's inputs, zero past kin and for rows >= mvalid
        for (int i = tid; i < kBM * 16; i += kChainThreads) {
            const int r = i >> 4, k = i & 15;
            xs[i] = (k < kin && m0 + r < a.mvalid) ? a.x[(size_t)(m0 + r) * kin + k] : 0.f;
        }
        __syncthreads();
        const int u = tid & 255;  // unit
        constexpr int kRows = kBM * 256 / kChainThreads;  // rows per thread
        const int rbase = (tid >> 8) * kRows;
        float wr[16];
#pragma unroll
        for (int k = 0; k < 16; k++) wr[k] = k < kin ? a.w0[u * kin + k] : 0.f;
        const float bu = a.b0 ? a.b0[u] : 0.f;
        // eight rows at a time, FMA chains interleaved; the sums run in
        // k_input_fwd's order (the padded terms add exact zeros)
        for (int r0 = rbase; r0 < rbase + kRows; r0 += 8) {
            float acc[8];
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] = bu;
#pragma unroll
            for (int k4 = 0; k4 < 16; k4 += 4) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const float4 xv = *reinterpret_cast<const float4 *>(&xs[(r0 + j) * 16 + k4]);
                    acc[j] = fmaf(xv.x, wr[k4], acc[j]);
                    acc[j] = fmaf(xv.y, wr[k4 + 1], acc[j]);
                    acc[j] = fmaf(xv.z, wr[k4 + 2], acc[j]);
                    acc[j] = fmaf(xv.w, wr[k4 + 3], acc[j]);
                }
            }
            __align__(16) __nv_bfloat16 yb[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int r = r0 + j;
                const float z = m0 + r < a.mvalid ? acc[j] : 0.f;
                yb[j] = __float2bfloat16_rn(gelu(z));
                if (a.z0) a.z0[(size_t)(m0 + r) * kWidth + u] = __float2bfloat16_rn(z);
                act_store1(act, r, u, yb[j]);
            }
            if (a.yt0)
                *reinterpret_cast<uint4 *>(a.yt0 + (size_t)u * a.ldt + m0 + r0) =
                    *reinterpret_cast<const uint4 *>(yb);
        }
        fence_proxy_async_smem();
    } else if (!mbar_wait_bounded(&abar, 0)) {
        ok = 0;
    }
    __syncthreads();
    if (tid == 0 && a0_pending && ok) a0_pending = false;

    // ---- layers -------------------------------------------------------------------------
    int l = 0;
    for (; l < a.nlayers && ok; l++) {
        const ChainLayer &L = a.layer[l];
        if (tid == 0) {
            fence_after_sync();
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                   ((uint32_t)(L.n >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
            for (int kb = 0; kb < L.kblocks; kb++) {
                if (!mbar_wait_bounded(&full[kb], ldpar[kb])) {
                    ok = 0;
                    break;
                }
                pending &= ~(1u << kb);
                fence_after_sync();
                const uint64_t ad = desc_sw128(smem_u32(act + kb * kABlockBytes));
                const uint64_t bd = desc_sw128(smem_u32(wslot + kb * kSlotBytes));
#pragma unroll
                for (int kk = 0; kk < kBK / 16; kk++)
                    mma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) ? 1u : 0u);
            }
            mma_commit(&accb);  // also when a wait failed: covers what was issued
        }
        __syncwarp();  // warp 0's other lanes wait here, not in the spin below
        const bool done = mbar_wait_bounded(&accb, (uint32_t)(l & 1));
        if (!done) ok = 0;
        __syncthreads();
        if (!ok) break;
        fence_after_sync();
        // the next layer's weights load while this epilogue runs
        if (tid == 0 && l + 1 < a.nlayers) load_layer(l + 1);

        const int part = L.n / kGroups;
        float lsum = 0.f;
#pragma unroll 1
        for (int c0 = h * part; c0 < (h + 1) * part; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
            if (L.bias) {
#pragma unroll
                for (int i = 0; i < 16; i++) v[i] += L.bias[c0 + i];
            }
            if (L.epi == kEpiGelu) {
                __align__(16) __nv_bfloat16 zb[16], yb[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    zb[i] = __float2bfloat16_rn(v[i]);
                    yb[i] = __float2bfloat16_rn(gelu(v[i]));
                }
                act_store16(act, row, c0, yb);
                if (L.zout) store16(L.zout + (size_t)m * L.n + c0, zb);
                if (L.y) store16(L.y + (size_t)m * L.n + c0, yb);
                if (L.yt) {
#pragma unroll
                    for (int i = 0; i < 16; i++) L.yt[(size_t)(c0 + i) * a.ldt + m] = yb[i];
                }
            } else if (L.epi == kEpiDGelu) {
                __align__(16) __nv_bfloat16 zz[16], gb[16];
                const uint4 *zp = reinterpret_cast<const uint4 *>(L.zin + (size_t)m * L.n + c0);
                reinterpret_cast<uint4 *>(zz)[0] = zp[0];
                reinterpret_cast<uint4 *>(zz)[1] = zp[1];
#pragma unroll
                for (int i = 0; i < 16; i++)
                    gb[i] = __float2bfloat16_rn(v[i] * gelu_grad(__bfloat162float(zz[i])));
                act_store16(act, row, c0, gb);
                if (L.y) store16(L.y + (size_t)m * L.n + c0, gb);
                if (L.yt) {
#pragma unroll
                    for (int i = 0; i < 16; i++) L.yt[(size_t)(c0 + i) * a.ldt + m] = gb[i];
                }
            } else {  // kEpiLinear
                if (m < a.mvalid) {
                    float4 *op = reinterpret_cast<float4 *>(L.out + (size_t)m * L.n + c0);
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        op[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
                if (a.target) {
                    __align__(16) __nv_bfloat16 gb[16];
                    const float den = (float)a.rvalid * L.n;
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const float d =
                            m < a.rvalid ? v[i] - a.target[(size_t)m * L.n + c0 + i] : 0.f;
                        lsum = fmaf(d, d, lsum);
                        gb[i] = __float2bfloat16_rn(2.f * d / den);
                    }
                    store16(a.g + (size_t)m * L.n + c0, gb);
#pragma unroll
                    for (int i = 0; i < 16; i++) a.gt[(size_t)(c0 + i) * a.ldt + m] = gb[i];
                }
            }
        }
        if (L.epi == kEpiLinear && a.target) lossp[h][row] = lsum;
        fence_proxy_async_smem();
        fence_before_sync();
        __syncthreads();
    }
    if (ok && a.target && a.loss_rows && h == 0 && l == a.nlayers) {
        float sum = lossp[0][row];
        for (int g = 1; g < kGroups; g++) sum += lossp[g][row];
        a.loss_rows[m] = sum;
    }

    if (!ok && tid == 0) {
        // drain what is in flight before the shared memory and TMEM go away
        for (int s = 0; s < kSlots; s++)
            if (pending & (1u << s)) mbar_wait_bounded(&full[s], ldpar[s]);
        if (a0_pending) mbar_wait_bounded(&abar, 0);
        if (a.err) atomicExch(a.err, 1);
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kWidth)
                     : "memory");
    }
}

cudaError_t launch_chain(const ChainArgs &a, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_chain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kChainSmem);
    if (e != cudaSuccess) return e;
    k_mlp_chain<<<(unsigned)(a.m / kBM), kChainThreads, kChainSmem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace
}  // namespace mlp
}  // namespace lcg

using namespace lcg;
using namespace lcg::mlp;

extern "C" {

lcg_status lcg_mlp_forward(void *stream, const float *x, int32_t kin, int32_t m, int32_t mvalid,
                           const float *w0, const float *b0, int32_t depth, int32_t nout,
                           const void *const *w_bf16, const float *const *bias, float *out,
                           void *const *z, void *const *yt, int32_t ldt, const float *target,
                           void *g, void *gt, float *loss_rows, int32_t *err) {
    if (!x || !w0 || !w_bf16 || !bias || !out || kin <= 0 || kin > 16 || m <= 0 || m % kBM ||
        mvalid < 0 || mvalid > m || depth < 1 || depth > kChainMax || nout <= 0 || nout > 256 ||
        nout % 64)
        return LCG_E_INVALID;
    const bool train = z != nullptr;
    if (train && (!yt || ldt < m || ldt % 8)) return LCG_E_INVALID;
    if (target && (!g || !gt || ldt < m || ldt % 8 || !aligned16(g))) return LCG_E_INVALID;
    if (!aligned16(out)) return LCG_E_INVALID;
    ChainArgs a;
    memset(&a, 0, sizeof(a));
    for (int l = 0; l < depth; l++) {
        const bool last = l == depth - 1;
        ChainLayer &L = a.layer[l];
        L.n = last ? nout : kWidth;
        L.kblocks = kWidth / kBK;
        L.epi = last ? kEpiLinear : kEpiGelu;
        L.bias = bias[l];
        if (!w_bf16[l] || !aligned16(w_bf16[l])) return LCG_E_INVALID;
        if (!make_map(&a.w[l], w_bf16[l], L.n, kWidth, L.n)) return LCG_E_CUDA;
        if (last) {
            L.out = out;
        } else if (train) {
            if (!z[l + 1] || !yt[l + 1] || !aligned16(z[l + 1])) return LCG_E_INVALID;
            L.zout = (__nv_bfloat16 *)z[l + 1];
            L.yt = (__nv_bfloat16 *)yt[l + 1];
        }
    }
    a.nlayers = depth;
    a.input_layer = 1;
    a.x = x;
    a.w0 = w0;
    a.b0 = b0;
    a.kin = kin;
    if (train) {
        if (!z[0] || !yt[0] || !aligned16(z[0]) || !aligned16(yt[0])) return LCG_E_INVALID;
        a.z0 = (__nv_bfloat16 *)z[0];
        a.yt0 = (__nv_bfloat16 *)yt[0];
    }
    a.target = target;
    a.g = (__nv_bfloat16 *)g;
    a.gt = (__nv_bfloat16 *)gt;
    a.loss_rows = loss_rows;
    a.rvalid = mvalid;
    a.m = m;
    a.mvalid = mvalid;
    a.ldt = ldt;
    a.err = err;
    return launch_chain(a, (cudaStream_t)stream) == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_mlp_backward_data(void *stream, int32_t m, int32_t depth, int32_t nout,
                                 const void *g_out, const void *const *wt_bf16,
                                 const void *const *z, void *const *g, void *const *gt,
                                 int32_t ldt, int32_t *err) {
    if (!g_out || !wt_bf16 || !z || !g || m <= 0 || m % kBM || depth < 1 || depth > kChainMax ||
        nout <= 0 || nout > 256 || nout % 64 || !aligned16(g_out))
        return LCG_E_INVALID;
    if (gt && (ldt < m || ldt % 8)) return LCG_E_INVALID;
    ChainArgs a;
    memset(&a, 0, sizeof(a));
    // layer j maps the gradient of layer (depth - j) to that of layer (depth - 1 - j)
    for (int j = 0; j < depth; j++) {
        ChainLayer &L = a.layer[j];
        const int kdim = j == 0 ? nout : kWidth;
        L.n = kWidth;
        L.kblocks = kdim / kBK;
        L.epi = kEpiDGelu;
        if (!wt_bf16[j] || !z[j] || !g[j] || !aligned16(wt_bf16[j]) || !aligned16(z[j]) ||
            !aligned16(g[j]))
            return LCG_E_INVALID;
        if (!make_map(&a.w[j], wt_bf16[j], kWidth, kdim, kWidth)) return LCG_E_CUDA;
        L.zin = (const __nv_bfloat16 *)z[j];
        L.y = (__nv_bfloat16 *)g[j];
        L.yt = gt ? (__nv_bfloat16 *)gt[j] : nullptr;
    }
    if (!make_map(&a.a0, g_out, m, nout, kBM)) return LCG_E_CUDA;
    a.nlayers = depth;
    a.a0_kblocks = nout / kBK;
    a.input_layer = 0;
    a.m = m;
    a.mvalid = m;
    a.ldt = ldt;
    a.err = err;
    return launch_chain(a, (cudaStream_t)stream) == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

}  // extern "C"
