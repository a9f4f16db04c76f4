// walk.cu — the inner steps of the sampler's surrogate transitions on the
// device: one thread per chain forms a random-walk proposal through a
// triangular quadratic map (u_1 = z_1, u_k = z_k - P_k(z_<k), z the
// standardised parameters; unit Jacobian, so the proposal
// T^-1(T(y) + L n) is symmetric), tests the prior box, writes the
// network's input coordinates, and after the network and the chi**2 head
// have run, takes the Metropolis decision on the surrogate's chi**2.
//
// Layout of a walk's parameters (par, doubles, d the dimension):
//   m[d] s[d]          standardisation z = (y - m) / s
//   c0[d] B[d*d]       constant and linear terms: P_k = c0[k] + sum_i<k z_i B[i*d+k] + ...
//   A[d*d*d]           quadratic terms A[(k*d + i)*d + j] z_i z_j, i <= j < k
//   chol[d*d]          step covariance factor (row-major, lower triangular)
//   mid[d] half[d]     network input (y - mid) / half
//   lo[d] hi[d]        the prior box
//
// Random numbers: Philox4x32-10 (cuRAND's counter-based generator), one
// subsequence per chain, the offset set by the step (a device counter plus
// the step's index), so that a CUDA graph of several steps can be replayed
// without reseeding. Test callers pass the normals and uniforms instead.

#include <curand_kernel.h>
#include <stdint.h>

#include "engine.h"
#include "lcg.h"

namespace {

constexpr int kMaxDim = 16;
constexpr int kThreads = 128;

struct WalkPar {
    const double *m, *s, *c0, *B, *A, *chol, *mid, *half, *lo, *hi;
};

__device__ __forceinline__ WalkPar walk_par(const double *p, int d) {
    WalkPar w;
    w.m = p;
    w.s = w.m + d;
    w.c0 = w.s + d;
    w.B = w.c0 + d;
    w.A = w.B + d * d;
    w.chol = w.A + d * d * d;
    w.mid = w.chol + d * d;
    w.half = w.mid + d;
    w.lo = w.half + d;
    w.hi = w.lo + d;
    return w;
}

// P_k(z_<k) = c0[k] + sum_i<k z_i (B[i][k] + sum_{i<=j<k} A_k[i][j] z_j)
__device__ __forceinline__ double poly(const WalkPar &w, int d, int k, const double *z) {
    double r = w.c0[k];
    for (int i = 0; i < k; i++) {
        const double *a = w.A + ((size_t)k * d + i) * d;
        double t = w.B[i * d + k];
        for (int j = i; j < k; j++) t += a[j] * z[j];
        r += t * z[i];
    }
    return r;
}

// Philox offsets (in 32-bit outputs) of one chain's step: the proposal's
// normals take the first 32, the decision's uniform the next 32.
__device__ __forceinline__ unsigned long long rng_offset(const int64_t *ctr, int32_t step,
                                                        int purpose) {
    return ((unsigned long long)(*ctr + step)) * 64ull + (purpose ? 32ull : 0ull);
}

__global__ void __launch_bounds__(kThreads) k_walk_propose(int32_t nc, int32_t d,
                                                           const double *__restrict__ par,
                                                           const double *__restrict__ y,
                                                           unsigned long long seed,
                                                           const int64_t *__restrict__ ctr,
                                                           int32_t step,
                                                           const double *__restrict__ noise,
                                                           double *__restrict__ prop,
                                                           float *__restrict__ xunit,
                                                           uint8_t *__restrict__ ok) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const WalkPar w = walk_par(par, d);
    double z[kMaxDim], v[kMaxDim], n[kMaxDim];
    for (int k = 0; k < d; k++) z[k] = (y[(size_t)i * d + k] - w.m[k]) / w.s[k];
    if (noise) {
        for (int k = 0; k < d; k++) n[k] = noise[(size_t)i * d + k];
    } else {
        curandStatePhilox4_32_10_t st;
        curand_init(seed, (unsigned long long)i, rng_offset(ctr, step, 0), &st);
        for (int k = 0; k < d; k += 2) {
            const double2 g = curand_normal2_double(&st);
            n[k] = g.x;
            if (k + 1 < d) n[k + 1] = g.y;
        }
    }
    // u = T(z) + L n, then z' = T^-1(u) coordinate by coordinate
    for (int k = 0; k < d; k++) {
        double dl = 0.;
        for (int j = 0; j <= k; j++) dl += w.chol[k * d + j] * n[j];
        v[k] = z[k] - poly(w, d, k, z) + dl;
    }
    bool inside = true;
    for (int k = 0; k < d; k++) {
        v[k] = v[k] + poly(w, d, k, v);  // v[<k] already hold z'
        const double p = w.m[k] + v[k] * w.s[k];
        prop[(size_t)i * d + k] = p;
        xunit[(size_t)i * d + k] = (float)((p - w.mid[k]) / w.half[k]);
        inside = inside && p >= w.lo[k] && p <= w.hi[k];
    }
    ok[i] = inside ? 1 : 0;
}

__global__ void __launch_bounds__(kThreads) k_walk_accept(
    int32_t nc, int32_t d, const double *__restrict__ prop, const uint8_t *__restrict__ ok,
    const double *__restrict__ chi, double *__restrict__ y, double *__restrict__ chis,
    int32_t *__restrict__ moves, unsigned long long seed, const int64_t *__restrict__ ctr,
    int32_t step, const double *__restrict__ unif) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    double u;
    if (unif) {
        u = unif[i];
    } else {
        curandStatePhilox4_32_10_t st;
        curand_init(seed, (unsigned long long)i, rng_offset(ctr, step, 1), &st);
        u = curand_uniform_double(&st);  // (0, 1]
    }
    const double c = chi[i];
    // NaN and +inf chi**2 (failed or outside) compare false: rejected
    if (ok[i] && log(u) < -(c - chis[i]) / 2) {
        for (int k = 0; k < d; k++) y[(size_t)i * d + k] = prop[(size_t)i * d + k];
        chis[i] = c;
        if (moves) moves[i] += 1;
    }
}

__global__ void k_walk_advance(int64_t *ctr, int64_t inc) { *ctr += inc; }

unsigned blocks(int32_t nc) { return (unsigned)((nc + kThreads - 1) / kThreads); }

}  // namespace

extern "C" {

lcg_status lcg_walk_propose(void *stream, int32_t nc, int32_t d, const double *par,
                            const double *y, uint64_t seed, const int64_t *ctr, int32_t step,
                            const double *noise, double *prop, float *xunit, uint8_t *ok) {
    if (nc <= 0 || d <= 0 || d > kMaxDim || !par || !y || !prop || !xunit || !ok ||
        (!noise && !ctr) || step < 0)
        return LCG_E_INVALID;
    k_walk_propose<<<blocks(nc), kThreads, 0, (cudaStream_t)stream>>>(
        nc, d, par, y, (unsigned long long)seed, ctr, step, noise, prop, xunit, ok);
    lcg::count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_walk_accept(void *stream, int32_t nc, int32_t d, const double *prop,
                           const uint8_t *ok, const double *chi, double *y, double *chis,
                           int32_t *moves, uint64_t seed, const int64_t *ctr, int32_t step,
                           const double *unif) {
    if (nc <= 0 || d <= 0 || d > kMaxDim || !prop || !ok || !chi || !y || !chis ||
        (!unif && !ctr) || step < 0)
        return LCG_E_INVALID;
    k_walk_accept<<<blocks(nc), kThreads, 0, (cudaStream_t)stream>>>(
        nc, d, prop, ok, chi, y, chis, moves, (unsigned long long)seed, ctr, step, unif);
    lcg::count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

lcg_status lcg_walk_advance(void *stream, int64_t *ctr, int64_t inc) {
    if (!ctr) return LCG_E_INVALID;
    k_walk_advance<<<1, 1, 0, (cudaStream_t)stream>>>(ctr, inc);
    lcg::count_launch();
    return cudaGetLastError() == cudaSuccess ? LCG_OK : LCG_E_CUDA;
}

}  // extern "C"
