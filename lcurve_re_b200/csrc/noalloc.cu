// noalloc.cu — the FP64 flux sweep for callers that cannot allocate.
//
// lcg_sum_star_multi_noalloc is for programs in which this library must not
// call cudaMalloc: applications whose device memory is already claimed by
// another framework's pooling allocator (frameworks that reserve nearly all
// device memory at start-up, so an allocation from here would fail), and
// latency-critical loops in which an allocation or a free would synchronise
// the device. The caller owns every input and output array; the only
// scratch, the per-block partial sums, lives in g_sweep_scratch below: a
// file-scope device array of kScratchDoubles doubles (16 MiB) that every GPU
// which loads this library holds until the process exits.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current) and keeps it; a host-side
// use of the symbol itself would not be a device address. That first call
// should come before any stream capture on the device.
//
// Sharing: every call on a device uses the same array, and the array keeps
// the last call's contents. Each call writes every partial it reads before
// reading it, in stream order, so nothing has to start at zero; but calls
// whose executions overlap on the GPU (different streams, no ordering) race
// on the array and must be serialised by the caller.
//
// The arithmetic is that of the FP64 sweep (flux64.cu; comp_light_flat.cpp
// :80-372): 1024-face blocks in FlatGrid order, per entry the faces added in
// ascending order, blocks merged in order. Beaming and lensing are not part
// of this variant.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "lcg.h"

namespace {

constexpr int64_t kScratchDoubles = 2 * 1024 * 1024;  // 16 MiB
constexpr int kBlock = 1024;
constexpr int kThreads = 128;
constexpr int kPPT = 2;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_sweep_scratch[kScratchDoubles];

struct Limb {
    double c1, c2, c3, c4, base, mucrit;
    int32_t ltype;
};

// imu_bl and the non-beaming, non-lensing element of s1_elem / s2_elem
// (comp_light_flat.cpp:80-127, 150-167); star 2's factor magn = 1 leaves the
// product unchanged.
__device__ __forceinline__ double element(double ex, double ey, double ez, double dx, double dy,
                                          double dz, double flux, const Limb &L) {
    const double mu = ex * dx + ey * dy + ez * dz;
    const double m = (1.0 < mu) ? 1.0 : mu;
    double im;
    if (L.ltype == LCG_LIMB_POLY) {
        const double om = 1.0 - m;
        im = 1.0 - om * (L.c1 + om * (L.c2 + om * (L.c3 + om * L.c4)));
    } else {
        const double msq = sqrt((m < 0.0) ? 0.0 : m);
        im = L.base + msq * (L.c1 + msq * (L.c2 + msq * (L.c3 + msq * L.c4)));
    }
    const double val = mu * flux * ((double)(mu > 0.0) * im);
    return (double)(mu > L.mucrit) * val;
}

// One CTA: one 1024-face block x kThreads*kPPT phase entries. Columns are read
// with bounds-checked coalesced loads (the caller's arrays carry no padding).
__global__ void __launch_bounds__(kThreads)
    k_sweep_noalloc(int64_t n, int64_t n0, const double *__restrict__ dx,
                    const double *__restrict__ dy, const double *__restrict__ dz,
                    const double *__restrict__ flux, const double *__restrict__ in1,
                    const double *__restrict__ out1, int32_t nent, const double *__restrict__ ex,
                    const double *__restrict__ ey, const double *__restrict__ ez,
                    const double *__restrict__ phin, Limb L, double *scratch) {
    __shared__ double s_dx[kBlock], s_dy[kBlock], s_dz[kBlock], s_fl[kBlock];
    __shared__ double s_in[kBlock / 2], s_out[kBlock / 2];  // staged in two halves
    const int64_t lo = (int64_t)blockIdx.y * kBlock;
    const int64_t hi = (lo + kBlock < n) ? lo + kBlock : n;
    for (int t = threadIdx.x; t < hi - lo; t += kThreads) {
        s_dx[t] = dx[lo + t];
        s_dy[t] = dy[lo + t];
        s_dz[t] = dz[lo + t];
        s_fl[t] = flux[lo + t];
    }
    double qx[kPPT], qy[kPPT], qz[kPPT], pn[kPPT], br[kPPT];
    const int64_t ebase = (int64_t)blockIdx.x * kThreads * kPPT + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kPPT; j++) {
        const int64_t e = ebase + (int64_t)j * kThreads;
        const bool ok = e < nent;
        qx[j] = ok ? ex[e] : 0.;
        qy[j] = ok ? ey[e] : 0.;
        qz[j] = ok ? ez[e] : 0.;
        pn[j] = ok ? phin[e] : 0.;
        br[j] = 0.0;
    }
    __syncthreads();
    const int64_t a1 = hi < n0 ? hi : n0;
    for (int64_t i = lo; i < a1; i++) {
        const int t = (int)(i - lo);
#pragma unroll
        for (int j = 0; j < kPPT; j++)
            br[j] += element(qx[j], qy[j], qz[j], s_dx[t], s_dy[t], s_dz[t], s_fl[t], L);
    }
    // one-range faces, their eclipse ranges staged half a block at a time
    const int64_t b0 = lo > n0 ? lo : n0;
    for (int64_t h0 = b0; h0 < hi; h0 += kBlock / 2) {
        const int64_t h1 = (h0 + kBlock / 2 < hi) ? h0 + kBlock / 2 : hi;
        __syncthreads();
        for (int64_t i = h0 + threadIdx.x; i < h1; i += kThreads) {
            s_in[i - h0] = in1[i - n0];
            s_out[i - h0] = out1[i - n0];
        }
        __syncthreads();
        for (int64_t i = h0; i < h1; i++) {
            const int t = (int)(i - lo), u = (int)(i - h0);
            const double ein = s_in[u], eout = s_out[u];
#pragma unroll
            for (int j = 0; j < kPPT; j++) {
                const double v = element(qx[j], qy[j], qz[j], s_dx[t], s_dy[t], s_dz[t], s_fl[t], L);
                const bool ecl = (pn[j] >= ein && pn[j] <= eout) || pn[j] <= eout - 1.0;
                br[j] += ecl ? 0.0 : v;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kPPT; j++) {
        const int64_t e = ebase + (int64_t)j * kThreads;
        if (e < nent) scratch[(int64_t)blockIdx.y * nent + e] = br[j];
    }
}

__global__ void k_merge_noalloc(const double *__restrict__ scratch, int64_t nblk, int32_t nent,
                                double *out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nent) return;
    double o = 0.0;
    for (int64_t b = 0; b < nblk; b++) o += scratch[b * nent + e];
    out[e] = o;
}

std::mutex g_setup_mutex;
double *g_scratch_addr[kMaxDevices] = {};

// Puts the caller's current device back on every return path: this entry point
// runs inside other programs, whose later runtime calls must not land on the
// device that owned `out`.
struct CurrentDeviceGuard {
    int saved = -1;
    CurrentDeviceGuard() {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            saved = -1;
            cudaGetLastError();
        }
    }
    ~CurrentDeviceGuard() {
        if (saved >= 0 && cudaSetDevice(saved) != cudaSuccess) cudaGetLastError();
    }
};

// A failure this call caused: consume the runtime's record of it, so that the
// caller's next cudaGetLastError does not report it a second time.
lcg_status own_cuda_failure() {
    cudaGetLastError();
    return LCG_E_CUDA;
}

}  // namespace

extern "C" lcg_status lcg_sum_star_multi_noalloc(
    void *stream, int32_t star, int64_t n, int64_t n0, const double *dx, const double *dy,
    const double *dz, const double *flux, const double *in1, const double *out1, int32_t nent,
    const double *ex, const double *ey, const double *ez, const double *phin, const double *ldc,
    int32_t ltype, double mucrit, double *out) {
    if ((star != LCG_STAR1 && star != LCG_STAR2) || n < 0 || n0 < 0 || n0 > n || nent < 0 ||
        !ldc || !out || (ltype != LCG_LIMB_POLY && ltype != LCG_LIMB_CLARET))
        return LCG_E_INVALID;
    if (n > 0 && (!dx || !dy || !dz || !flux)) return LCG_E_INVALID;
    if (n > n0 && (!in1 || !out1)) return LCG_E_INVALID;
    if (nent > 0 && (!ex || !ey || !ez || !phin)) return LCG_E_INVALID;
    const int64_t nblk = (n + kBlock - 1) / kBlock;
    if (nent > 0 && nblk > kScratchDoubles / nent) return LCG_E_CAPACITY;
    if (nblk > 65535) return LCG_E_CAPACITY;  // grid.y limit
    if (nent == 0) return LCG_OK;

    // the device that owns the output array
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, out) != cudaSuccess ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) ||
        attr.device < 0 || attr.device >= kMaxDevices) {
        cudaGetLastError();
        return LCG_E_INVALID;
    }
    CurrentDeviceGuard keep_callers_device;
    if (cudaSetDevice(attr.device) != cudaSuccess) return own_cuda_failure();
    double *scratch;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[attr.device]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_sweep_scratch) != cudaSuccess || !p)
                return own_cuda_failure();
            g_scratch_addr[attr.device] = static_cast<double *>(p);
        }
        scratch = g_scratch_addr[attr.device];
    }
    Limb L{ldc[0], ldc[1], ldc[2], ldc[3], 1.0 - (ldc[0] + ldc[1] + ldc[2] + ldc[3]), mucrit,
           ltype};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // cudaLaunchKernel reports this launch's own status; an error left by the
    // caller's earlier work is neither consumed nor blamed on this call unless
    // it is a sticky one that also fails these launches.
    if (nblk > 0) {
        dim3 grid((unsigned)((nent + kThreads * kPPT - 1) / (kThreads * kPPT)), (unsigned)nblk);
        void *args[] = {&n,  &n0, &dx, &dy, &dz, &flux, &in1, &out1, &nent,
                        &ex, &ey, &ez, &phin, &L, &scratch};
        if (cudaLaunchKernel((const void *)k_sweep_noalloc, grid, dim3(kThreads), args, 0, s) !=
            cudaSuccess)
            return own_cuda_failure();
    }
    const double *partials = scratch;
    int64_t nb = nblk;
    void *margs[] = {&partials, &nb, &nent, &out};
    if (cudaLaunchKernel((const void *)k_merge_noalloc, dim3((unsigned)((nent + 255) / 256)),
                         dim3(256), margs, 0, s) != cudaSuccess)
        return own_cuda_failure();
    return LCG_OK;
}
