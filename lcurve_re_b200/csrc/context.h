// context.h — host-side state of an engine context, shared by the
// single-model path (engine.cu) and the batched path (batch_host.cu).
#pragma once

#include <stdarg.h>
#include <stdio.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "engine.h"
#include "lcg.h"

namespace lcg {
namespace eng {

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n == 0) n = 1;
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc((void **)&p, n * sizeof(T));
        if (e != cudaSuccess) return e;
        cap = n;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct StarSetup {
    double r1, r2, rl1, rl2, ffac1, ffac2, rref1, pref1, rref2, pref2, gref;
    int infill, nlat, nlatfill, nlngfill, eclipse;
    double thelo, thehi;
    int nface;   // numface: the reference's face count
    int ntiled;  // faces of the ring tiling (may differ by one or two)
    int64_t nhalf;
    std::vector<RingRec> rings;
};

struct Fail {
    int code;
    std::string msg;
};

struct Grid {
    DBuf<double> px, py, pz, nx, ny, nz, ein, eout;
    DBuf<float> area, grav, flux;
    DBuf<uint8_t> necl;
    DBuf<RingRec> rings;
    DBuf<int32_t> queue, counters;  // eclipse candidates of this grid
    DBuf<double4> es;               // and their state between the two passes
    DBuf<int32_t> hits;
    // flat
    DBuf<int64_t> n0;
    DBuf<float4> geo, pos;
    DBuf<ulonglong2> ecl;
    DBuf<double> fdx, fdy, fdz, fpx, fpy, fpz, fflux, fin, fout;
    DBuf<float> fp;
    DBuf<float4> runb;
    DBuf<ulonglong2> runh;
    // opaque disc: per-face disc ranges, and the flat grid's several-range faces
    DBuf<uint8_t> ndx, rn;
    DBuf<double2> xr, rr;
    DBuf<int32_t> ridx;
    bool disc = false;  // ndx / xr hold this grid's disc ranges
    int64_t n = 0, npad = 0, ntiled = 0;
    int fast = 0;  // flat records built for the fast mixed sweep
    StarSetup setup;

    cudaError_t alloc_points(int64_t nf) {
        n = nf;
        ntiled = nf;
        cudaError_t e = cudaSuccess;
        DBuf<double> *d[] = {&px, &py, &pz, &nx, &ny, &nz, &ein, &eout};
        for (auto *b : d)
            if ((e = b->ensure(nf)) != cudaSuccess) return e;
        if ((e = area.ensure(nf)) || (e = grav.ensure(nf)) || (e = flux.ensure(nf)) ||
            (e = necl.ensure(nf)))
            return e;
        return cudaSuccess;
    }
    cudaError_t alloc_flat(int mixed, int need_pos, int fast_on) {
        npad = ((n + 4095) / 4096) * 4096;
        if (npad == 0) npad = 4096;
        cudaError_t e = n0.ensure(2);  // n0, n1
        if (e) return e;
        if (disc && ((e = ridx.ensure(n)) || (e = rn.ensure(n)) || (e = rr.ensure(kRagRanges * n))))
            return e;
        if (mixed) {
            if ((e = ecl.ensure(npad))) return e;
            if (fast_on) {
                if ((e = fp.ensure(8 * npad)) || (e = runb.ensure(npad / 64)) ||
                    (e = runh.ensure(npad / 64)))
                    return e;
            } else if ((e = geo.ensure(npad))) {
                return e;
            }
            if (need_pos && (e = pos.ensure(npad))) return e;
        } else {
            DBuf<double> *d[] = {&fdx, &fdy, &fdz, &fpx, &fpy, &fpz, &fflux, &fin, &fout};
            for (auto *b : d)
                if ((e = b->ensure(npad)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    GridDev dev() const {
        return GridDev{px.p, py.p, pz.p, nx.p, ny.p, nz.p, area.p, grav.p, flux.p,
                       necl.p, ein.p, eout.p, n, ntiled, disc ? ndx.p : nullptr,
                       disc ? xr.p : nullptr};
    }
    FlatDev flat() const {
        return FlatDev{n, npad, n0.p, geo.p, ecl.p, pos.p, fdx.p, fdy.p, fdz.p,
                       fpx.p, fpy.p, fpz.p, fflux.p, fin.p, fout.p, fp.p, runb.p, runh.p,
                       n0.p ? n0.p + 1 : nullptr, ridx.p, rr.p, rn.p};
    }
    void release() {
        DBuf<double> *d[] = {&px, &py, &pz, &nx, &ny, &nz, &ein, &eout, &fdx, &fdy,
                             &fdz, &fpx, &fpy, &fpz, &fflux, &fin, &fout};
        for (auto *b : d) b->release();
        area.release(); grav.release(); flux.release(); necl.release(); rings.release();
        queue.release(); counters.release(); es.release(); hits.release();
        n0.release(); geo.release(); pos.release(); ecl.release(); fp.release();
        runb.release(); runh.release(); ndx.release(); rn.release(); xr.release(); rr.release(); ridx.release();
        disc = false;
    }
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};

struct BatchState;
void batch_release(BatchState *b);

}  // namespace eng
}  // namespace lcg

using lcg::DatumRec;
using lcg::DevStatus;
using lcg::Ginterp;
using lcg::eng::DBuf;
using lcg::eng::Grid;
using lcg::eng::Timer;

struct lcg_ctx {
    int device = 0, precision = LCG_PREC_MIXED, verbose = 0, nsm = 148, eclipse_warp = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // exact-reuse cache
    bool has_geom = false, has_cont = false;
    lcg_model key{};
    int cached_mixed_pos = -1;
    bool copy1 = true, copy2 = true;
    Ginterp gi{};
    Grid g1f, g2f, g1c, g2c;
    // batched evaluation (batch.cu); NULL until the first batch
    lcg::eng::BatchState *batch = nullptr;
    // the models a batch call evaluates through the single-model path (every
    // model of an FP64 context; those outside the batched stages otherwise)
    // run on worker contexts, one host thread and one stream each, so that
    // their latency-bound pipelines overlap on the GPU; each worker holds a
    // copy of the resident points (h_data, from lcg_set_data)
    std::vector<lcg_ctx *> workers;
    std::vector<int64_t> worker_data_version;
    std::vector<DatumRec> h_data;
    // work buffers
    DBuf<DevStatus> status;
    DBuf<int32_t> queue, counters, blockcnt;
    DBuf<int32_t> blockcnt2;  // star 2's partition scratch when it flattens on side[0]
    DBuf<DatumRec> data;
    DBuf<int64_t> off;
    DBuf<double> pex, pey, pez, pphin, pw1, pw2, part1f, part1c, part2f, part2c, calc, scratch,
        sfac, out, diag, osum;
    DBuf<float4> pef;
    DBuf<unsigned long long> ppfx;
    DBuf<uint8_t> ptype;
    // disc, rim and bright spot of the last model; iscale components
    DBuf<lcg::ElemRec> elem;
    DBuf<double4> epos;
    DBuf<lcg::DiscRing> drings;
    DBuf<double> csum, fcomp, iwork;
    lcg::CompParams comp{};
    // side streams: star 2's grids (side[0]) and the component elements
    // (side[1]) run beside star 1's; their eclipse solves are latency-bound,
    // so they overlap well. Created by the first call.
    // With fine grids only (no coarse ones, no opaque disc), star 2's continuum,
    // partition and flux sweep also stay on side[0], which waits for the phase
    // entries (ev_phases) and joins before the scatter: star 1's sweep fills
    // the SMs that star 2's latency-bound geometry leaves idle.
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr}, ev_phases = nullptr;
    std::vector<int64_t> h_off;
    std::vector<double> h_diag;
    // resident light-curve points (lcg_set_data)
    // light_curve_comp_fast: all points, sample indices, interpolated curve
    DBuf<DatumRec> fdata;
    DBuf<int64_t> fidx;
    DBuf<double> fcalc, fout;
    int32_t data_n = 0;
    int64_t data_version = 0;  // bumped by every lcg_set_data
    int64_t data_nent = 0;
    double data_xmin = 0., data_xmax = 0.;
    // profiling
    bool profiling = false;
    std::vector<Timer> pending[LCG_NSTAGE];
    double stage_ms[LCG_NSTAGE] = {0};
    int64_t stage_n[LCG_NSTAGE] = {0};
    int64_t flux_elements = 0;

    lcg_status fail(int code, const char *fmt, ...) {
        char b[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(b, sizeof b, fmt, ap);
        va_end(ap);
        err = b;
        return (lcg_status)code;
    }
    lcg_status cuda_fail(cudaError_t e, const char *what) {
        return fail(e == cudaErrorMemoryAllocation ? LCG_E_NOMEM : LCG_E_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
    }
    void stage_begin(int s, Timer &t) {
        if (!profiling) return;
        cudaEventCreate(&t.a);
        cudaEventCreate(&t.b);
        cudaEventRecord(t.a, stream);
        (void)s;
    }
    void stage_end(int s, Timer &t) {
        if (!profiling) return;
        cudaEventRecord(t.b, stream);
        pending[s].push_back(t);
    }
    void collect_timers() {
        for (int s = 0; s < LCG_NSTAGE; s++) {
            for (auto &t : pending[s]) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, t.a, t.b);
                stage_ms[s] += ms;
                stage_n[s] += 1;
                cudaEventDestroy(t.a);
                cudaEventDestroy(t.b);
            }
            pending[s].clear();
        }
    }
};

namespace lcg {
namespace eng {

struct StageScope {
    lcg_ctx *c;
    int s;
    Timer t;
    StageScope(lcg_ctx *c_, int s_) : c(c_), s(s_) { c->stage_begin(s, t); }
    ~StageScope() { c->stage_end(s, t); }
};

// per-model host setup (engine.cu)
void get_r1r2(const lcg_model &m, double &rr1, double &rr2);
// Radii, lobe checks, reference spheres and gref of one star grid; with
// tiling, also the face count and the latitude-ring table.
bool prepare_star(const lcg_model &m, int star, int fine, StarSetup &s, Fail &f,
                  bool tiling = true);
// Face count and ring table of a grid without infill: they depend on nlat alone.
int numface(int nlat, bool infill, double thelo, double thehi, int nlatfill, int nlngfill);
bool add_rings(int star, StarSetup &s, int &nface, double tlo, double thi, double dtheta,
               int nlatfill, int nlngfill);
const char *status_text(int code);
bool same_geometry(const lcg_model &a, const lcg_model &b);
bool same_continuum(const lcg_model &a, const lcg_model &b);
ContParams continuum_params(const lcg_model &m, int star);
FluxConsts flux_consts(const lcg_model &m, int star, double spin, double rlens1);
FastCoef fast_coef(const lcg_model &m, int star, int mixed);
lcg_status check_model(lcg_ctx *c, const lcg_model *m);
// Disc, rim and spot of a model: counts, ring table and element constants
// (set_disc_grid.cpp, set_bright_spot_grid.cpp); false with f set on a
// reference error.
bool comp_setup(const lcg_model &m, CompParams &p, std::vector<DiscRing> &rings, Fail &f);
bool bright_spot_position(double q, double rad, double *pos, Fail &f);
lcg_status finish_status(lcg_ctx *c);

}  // namespace eng
}  // namespace lcg
