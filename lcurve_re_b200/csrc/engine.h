// engine.h — kernel parameter blocks and launchers shared by the host engine
// (engine.cpp) and the kernel files (geometry.cu, flux.cu, flux64.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "roche.cuh"
#include "disc.cuh"
#include "ecl_screen.cuh"

namespace lcg {

// Number of kernels this library has launched (all contexts); read by
// lcg_kernel_launches.
void count_launch();
void count_launches(int64_t k);

// One latitude ring of a star grid (set_star_grid.cpp:280-320), computed on
// the host with the reference's libm so ring sizes match exactly.
struct RingRec {
    double sint, cost, phi1, span, latspan;  // span = phi2 - phi1, latspan = thi - tlo
    int32_t nphi, nl, off, hoff;             // hoff: first half-face of the ring
};

// Point-order star grid on the device (the reference's vector<Point>).
// n is the reference's face count (numface, the length of its vector);
// faces [ntiled, n) are default Points (no tiled face lands there) and the
// tiling's faces past n are dropped, as the reference's vector holds them.
struct GridDev {
    double *px, *py, *pz, *nx, *ny, *nz;
    float *area, *grav, *flux;
    uint8_t *necl;
    double *ein, *eout;
    int64_t n, ntiled;
    // ranges an opaque disc adds to each face (light_curve_comp.cpp:288-323):
    // ndx[i] of them in xr[kDiscRanges i ...]; NULL when there is no opaque disc
    const uint8_t *ndx;
    const double2 *xr;
};
constexpr int kDiscRanges = 2;   // disc_eclipse gives at most two ranges
constexpr int kRagRanges = 1 + kDiscRanges;  // the companion's, then the disc's

struct GridParams {
    int32_t star, roche, npole, nrings;
    int64_t nhalf;  // total half-faces (sum over rings of (nphi+1)/2)
    double q, spin, rref, pref, acc, gref, rad_sphere;
};

// Eclipse of one star's faces by its companion (set_star_grid.cpp:372-386).
struct EclParams {
    int32_t comp_star;   // the eclipsing star
    int32_t comp_roche;  // Roche-distorted eclipser (else a sphere of radius comp_r)
    double q, comp_spin, comp_rref, comp_pref, comp_r, cosi, sini, delta;
    EclScreen scr;       // FP32 screen of the bisections' line-of-sight tests
};

// The FP32 screen runs in mixed contexts when neither the eclipsed star
// (radius r_face) nor the eclipser (reference sphere rref) is tiny: a white
// dwarf's own eclipse boundaries, and eclipses by one, stay with FP64 alone.
inline void set_ecl_screen(EclParams &ep, int mixed, double r_face) {
    ep.scr = make_ecl_screen(ep.comp_star, ep.q, ep.comp_spin, ep.comp_rref, ep.comp_pref);
    ep.scr.on = mixed && ep.comp_roche && r_face >= 0.01 && ep.comp_rref >= 0.05;
}

// Continuum of one star (set_star_continuum.cpp:26-297).
struct ContParams {
    int32_t star, mirror, nspot, uesp_on;
    double t_own, t_other;    // t1/t2 of this star and of the other (model values)
    double absorb, gdcbol, wavelength, rcomp, efac;
    double spot_dir[3][3], spot_fwhm[3], spot_tcen[3];
    double uesp_dir[3], uesp_longhw, uesp_lathw, uesp_taper, uesp_temp;
    // mixed contexts: the intensity (gravity darkening, irradiated temperature,
    // Planck) in FP32 from the FP64 geometry and temperature; irr32 = absorb
    // t_other^4, planck_c1 = 2e27 h c / wavelength^3 (the reference's FAC1 over
    // lambda^3), planck_c2 = 1e9 h c / k / wavelength
    int32_t fp32;
    float irr32, planck_c1, planck_c2;
};

// One light-curve point, the byte layout of lcg_datum / Lcurve::Datum.
struct DatumRec {
    double time, expose, flux, ferr, weight;
    int32_t ndiv, pad_;
};

// Device status word: the first failure wins.
struct DevStatus {
    int32_t code;
    int32_t face;
};

// Flattened grid for the flux sweep (FlatGrid, comp_light_flat.cpp:26-65).
// Faces [0,n0) are never eclipsed, [n0,n) have one eclipse range. The
// mixed-precision view packs (nx,ny,nz,flux) as float4 and the eclipse range
// as 64-bit fixed-point phase (ingress, width; ecl_fx64 in geometry.cu); the
// FP64 view keeps the reference's doubles. Arrays are padded with zero faces
// to npad.
struct FlatDev {
    int64_t n, npad;
    int64_t *n0;  // device scalar, written by the partition
    float4 *geo;  // mixed, general: (nx, ny, nz, flux)
    ulonglong2 *ecl;  // mixed: (ingress, width) as 64-bit fixed-point phase
    float4 *pos;  // (px,py,pz,0): beaming and lensing only
    double *dx, *dy, *dz, *px, *py, *pz, *flux, *in1, *out1;  // FP64
    // mixed, fast: per PAIR of faces (a, b) four float4
    //   (nx_a, nx_b, ny_a, ny_b) (cz_a, cz_b, f0_a, f0_b) (f1_a, f1_b, f2_a, f2_b) (f3_a, f3_b, f4_a, f4_b)
    // with cz = cos(i) nz and f_k = flux * p_k, so each float2 operand of the
    // packed FP32x2 arithmetic is an aligned register pair
    float *fp;
    // per run of 32 pairs (64 faces) of fp: (ax, ay, R, C) bounding
    // mu = ex nx + ey ny + cz <= ex ax + ey ay + |(ex, ey)| R + C for every face
    // of the run (C includes a margin over FP32 rounding), so a warp can skip
    // a run that faces away at all its phases
    float4 *runb;
    // per run: an arc (I, W) of fixed-point phase holding every eclipse range
    // of the run's faces (W = ~0: test each face; (0, 0): none has a range), so
    // a warp whose phases all lie outside it skips the run's eclipse tests
    ulonglong2 *runh;
    // faces with two or more eclipse ranges (opaque discs) sit last, in
    // [*n1, n): their records above are zero (they add nothing to the main
    // sweeps); ridx is each one's face index in the grid, rr its rn ranges
    int64_t *n1;
    int32_t *ridx;
    double2 *rr;  // kRagRanges per ragged face
    uint8_t *rn;
};

// Face records of the fast mixed sweep (no beaming, no lensing, mucrit <= 0):
// the constant z term of mu = e.n and the face flux times the intensity
// polynomial, so mu costs 2 FMA and Horner yields flux * I directly.
//   Claret: I = p0 + p1 t + p2 t^2 + p3 t^3 + p4 t^4, t = sqrt(mu), p = (1 - sum c, c1..c4)
//   poly:   I = 1 - sum_k c_k (1-mu)^k expanded in powers of t = mu
struct FastCoef {
    int32_t on, ltype;
    double cosi;
    double p[5];
};

// Sub-exposure phase entries of all data points (light_curve_comp.cpp:416-455).
struct PhaseDev {
    double *ex, *ey, *ez, *phin, *w1, *w2;
    float4 *ef;     // (ex, ey, ez, unused) for the mixed sweeps
    uint8_t *type;  // Ginterp::type
    int64_t nent;
    unsigned long long *pfx;  // phin as a 64-bit fixed-point fraction (mixed)
};

struct PhaseParams {
    double t0, period, pdot, deltat, slope, quad, cube, middle, range, cosi, sini;
    Ginterp gi;
};

// Limb darkening and beaming/lensing constants of one flux sweep.
struct FluxConsts {
    double c[4], base, mucrit;
    int32_t ltype, beam_on, glens;
    double beam, spin, vfac, xcofm, rlens1;
};

struct ScatterParams {
    int32_t copy1, copy2;
    double third;
    // disc / rim / spot: per-entry element sums (3 rows of ldc), added per
    // point as slfac * (disc + rim + spot) (light_curve_comp.cpp:476-490)
    const double *csum;
    int64_t ldc;
    PhaseParams pp;  // to recompute each point's slfac
    // iscale: write the per-point components [star 1, disc, rim, spot,
    // star 2] to fcomp (5 per point) instead of the light curve
    double *fcomp;
};

// The four sweeps' chunk partials (1f, 1c, 2f, 2c; NULL when a sweep did not
// run) and their per-entry sums.
struct ReduceParams {
    const double *part[4];
    int64_t nchunk[4], nent[4];
    int64_t ldp;  // row stride of the partials
    double *osum[4];
};

// ---- batched evaluation -----------------------------------------------------
// A batch evaluates many models over the same resident points. Each model has
// two star grids ("slots" 2m and 2m+1); the faces of all slots live in one set
// of point arrays, the flat records of slot s start at a multiple of 1024
// faces, and every stage walks a work list of slots instead of launching per
// grid. Only the fast mixed sweep is batched (no beaming, lensing, mucrit > 0,
// coarse grids or infill).
struct SlotDev {
    GridParams gp;
    EclParams ep;
    ContParams cp;
    FastCoef fc;
    int64_t face0;  // first face in the batch point arrays
    int64_t nface, ntiled;
    int64_t flat0;  // first face of the slot's flat records (a multiple of 1024)
    int64_t blk0;   // first 1024-face partition block
    int32_t ring0;  // first ring of the slot's table in the ring pool
    int32_t model, eclipse_on, live;
};

struct ModelDev {
    PhaseParams pp;
    double third;
    double sfac0;  // the scale when it is not fitted
    int32_t live;
    int32_t pad_;
};

struct BatchDev {
    const SlotDev *slots;
    const ModelDev *models;
    const int64_t *face0;      // nslots + 1 face offsets (candidate -> slot)
    const int64_t *chunk_pre;  // nslots + 1 flux-chunk offsets
    const RingRec *rings;
    int32_t nslots, nmodels;
    GridDev g;  // every face of the batch
    float *fp;  // fast sweep records (FlatDev::fp layout per slot)
    float4 *runb;  // FlatDev::runb per slot, from flat0 / 64
    ulonglong2 *runh;  // FlatDev::runh per slot, from flat0 / 64
    ulonglong2 *ecl;
    int64_t *n0;  // per slot
    // eclipse candidates: those whose bisections the FP32 screen serves go to
    // the front of queue, the others (FP64 alone) to the back, so that warps
    // do not mix the two; counters: [0] candidates, [1]-[3] work counters of
    // the passes, [4] back-of-queue candidates, [5] front-of-queue ones, [6]
    // candidates pot_min found eclipsed
    int32_t *blockcnt, *queue, *counters;
    int64_t qcap;  // queue capacity (faces of the batch)
    // eclipse candidates between the two passes of the thread mode: per queue
    // entry (phase of the potential minimum, phi1, phi2, ACC), and the list of
    // the entries pot_min found eclipsed (the bisections' work, compacted)
    double4 *es;
    int32_t *hits;
    DevStatus *st;  // per model
    // work lists: counts[0] geometry slots, counts[1] continuum slots; each
    // list has its slots and prefix sums (count + 1 entries) of its units
    const int32_t *counts;
    const int32_t *geo_slot;
    const int64_t *geo_half, *geo_face;
    const int32_t *cont_slot;
    const int64_t *cont_face, *cont_blk;
};

// k such that pre[k] <= u < pre[k + 1], over count entries.
__host__ __device__ __forceinline__ int find_seg(const int64_t *__restrict__ pre, int count,
                                                 int64_t u) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Per-model phase rows of a batch: entry e of model m at m * ldp + e.
struct BatchPhases {
    float4 *ef;
    double *w1, *w2;
    int64_t ldp, nent;
    unsigned long long *pfx;  // PhaseDev::pfx, ldp per model
};

// ---- launchers (geometry.cu) ------------------------------------------------
void launch_grid(const GridParams &p, const RingRec *rings, GridDev g, DevStatus *st,
                 cudaStream_t s);
// queue: one int per face; counters: 8 (candidates, work counters, hits);
// es / hits: per-candidate state between the thread mode's two passes and the
// compacted list of the eclipsed candidates (one per face each).
void launch_eclipse(const EclParams &p, int32_t eclipse_on, GridDev g, int32_t *queue,
                    int32_t *counters, double4 *es, int32_t *hits, DevStatus *st, int nsm,
                    int32_t warp_mode, cudaStream_t s);
void launch_continuum(const ContParams &p, GridDev g, cudaStream_t s);
void launch_flatten(GridDev g, FlatDev f, int32_t *blockcnt, int mixed, int need_pos,
                    const FastCoef &fc, DevStatus *st, cudaStream_t s);
void launch_phases(const PhaseParams &p, const DatumRec *data, const int64_t *off, int32_t n,
                   PhaseDev ph, cudaStream_t s);
void launch_scatter(const ScatterParams &p, const ReduceParams &r, const PhaseDev &ph,
                    const DatumRec *data, const int64_t *off, int32_t n, double *calc,
                    cudaStream_t s);
// finalize: scale / chi**2 (re_scale.cpp:16-42, light_curve_comp.cpp:557-585).
// out[0] = chisq, out[1] = wnok, out[2] = 1 when they were computed.
void launch_finalize(int32_t flags, const DatumRec *data, int32_t n, double *calc,
                     double *sfac_io, double *out, cudaStream_t s);
// flux-weighted gravity / volume-averaged radius sums (comp_gravity.cpp,
// comp_radius.cpp): out[0..3] = sum f*g, sum f, sum solid angle, sum volume
void launch_diagnostics(int star, GridDev g, double *out, cudaStream_t s);
// light_curve_comp_fast interpolation of the model at sampled points mc
// (sample indices idx, m of them) to all n points; chi**2, wnok -> out[0..1].
// dst row r = src row rows[r] (count rows of n doubles)
void launch_gather_rows(const double *src, int32_t n, const int32_t *rows, int32_t count,
                        double *dst, cudaStream_t s);
void launch_interp(const DatumRec *data, int32_t n, const int64_t *idx, int32_t m,
                   const double *mc, double *calc, int32_t rdata, double *out, cudaStream_t s);

void launch_pack_flat(FlatDev f, int64_t n0, int need_pos, cudaStream_t s);
// run bounds of fast records: npairs pairs from fp, one float4 per 32 pairs
void launch_run_bounds(const float *fp, const ulonglong2 *ecl, int64_t npairs, float4 *runb,
                       ulonglong2 *runh, cudaStream_t s);
void launch_batch_run_bounds(const BatchDev &b, int nsm, cudaStream_t s);
void launch_pack_phases(PhaseDev ph, cudaStream_t s);

// batched stages (geometry.cu): grid + eclipse of the geometry list;
// continuum + partition of the continuum list; phases; reduction, scatter and
// scale / chi**2 of every model. Grids are fixed by the layout (persistent
// loops over device-side counts), so a captured graph replays any work lists.
void launch_batch_grid(const BatchDev &b, int nsm, cudaStream_t s);
void launch_batch_eclipse(const BatchDev &b, int nsm, int32_t warp_mode, cudaStream_t s);
void launch_batch_continuum(const BatchDev &b, int nsm, cudaStream_t s);
void launch_batch_flatten(const BatchDev &b, int nsm, cudaStream_t s);
void launch_batch_phases(const BatchDev &b, const DatumRec *data, const int64_t *off, int32_t n,
                         const BatchPhases &ph, cudaStream_t s);
void launch_batch_reduce(const BatchDev &b, const BatchPhases &ph, const double *part,
                         int64_t ldp, double *osum, const DatumRec *data, const int64_t *off,
                         int32_t n, int32_t flags, double *calc, double *sfac, double *out,
                         cudaStream_t s);

// ---- launchers (flux.cu, flux64.cu) -----------------------------------------
struct FluxPlan {
    int fast;       // fast mixed sweep (FlatDev::fa/fb records)
    int ppt;        // phase entries per thread
    int threads;    // threads per CTA
    int64_t chunk;  // faces per CTA
    int64_t nchunk;
    int64_t ntile;  // phase tiles
};
FluxPlan plan_flux(int mixed, int fast, int64_t nface, int64_t nent, int nsm);
void launch_flux(int mixed, int star, const FluxConsts &k, const FlatDev &f,
                 const PhaseDev &ph, const FluxPlan &plan, double *part, int64_t ldp,
                 DevStatus *st, cudaStream_t s);
// Batched fast mixed sweep: one CTA per (flux chunk of any slot, phase tile);
// plan.chunk divides 1024, plan.nchunk is the batch's total chunk count.
void launch_batch_flux(const BatchDev &b, const BatchPhases &ph, const FluxPlan &plan,
                       double *part, int64_t ldp, cudaStream_t s);
// FP32 FMA throughput probe: fills *gflop with the FLOPs it executed.
void launch_fma_probe(float *sink, int blocks, int iters, double *gflop, cudaStream_t s);
void launch_dfma_probe(double *sink, int blocks, int iters, double *gflop, cudaStream_t s);
void launch_flux64(int star, const FluxConsts &k, const FlatDev &f, const PhaseDev &ph,
                   const FluxPlan &plan, double *part, int64_t ldp, DevStatus *st,
                   cudaStream_t s);
// Faces with several eclipse ranges, [*f.n1, f.n): each CTA row continues the
// partial sums of one face block of blk faces (1024 for the FP64 sweep: the
// reference's block order; plan.chunk for the mixed sweeps), in face order,
// after the main sweep has written them.
void launch_flux_ragged(int star, const FluxConsts &k, const FlatDev &f, const GridDev &g,
                        const PhaseDev &ph, int64_t blk, int64_t nblk, double *part,
                        int64_t ldp, cudaStream_t s);

// ---- accretion disc, disc rim and bright spot (components.cu) ----------------
// One component element: outward normal, flux (brightness x area, rounded to
// float as the reference's Point::flux) and up to kMaxRanges eclipse ranges in
// the order the reference pushes them (opaque disc, star 1, star 2).
constexpr int kMaxRanges = 4;
struct ElemRec {
    double dx, dy, dz;
    float flux;
    int32_t nr;
    double2 r[kMaxRanges];
};
// One ring of disc elements (set_disc_grid.cpp:79-96)
struct DiscRing {
    double rad, h, sinp, cosp, area;
    int32_t ntheta, off;
};
// Everything the element kernel needs, derived on the host per model. The
// elements are the disc [0, nd), its outer rim [nd, nd + ne) and the spot
// [nd + ne, nd + ne + ns), each in the reference's vector order.
struct CompParams {
    int32_t nd, ne, ns, nrad;
    const DiscRing *rings;
    double bright_disc, rdisc2, texp;                    // set_disc_continuum
    double rad_e, h_e, area_e;                           // set_disc_edge (outer)
    int32_t nout, ntheta_e;
    double tedge, t2, absorb_edge, wave;                 // set_edge_continuum
    double bspot[3], bvec[3], tvec[3];                   // set_bright_spot_grid
    double bmax, sfac, area_s, bright_s, expon, epow, cfrac, length;
    int32_t nspot;
    int32_t opaque, eclipse1, eclipse2, roche1, roche2;  // star_eclipse
    double q, spin1, spin2, cosi, sini, delta, r1, r2, rref1, pref1, rref2, pref2;
    DiscGeom dg;
};
// Elements into el (and (x, y, z, area) into pos); errors into *st.
void launch_components(const CompParams &p, ElemRec *el, double4 *pos, DevStatus *st,
                       cudaStream_t s);
// The ranges an opaque disc adds to each face of a star grid.
void launch_disc_faces(const DiscGeom &dg, const GridDev &g, uint8_t *ndx, double2 *xr,
                       DevStatus *st, cudaStream_t s);
// Per phase entry, the disc, rim and spot element sums (comp_light.cpp:323-408)
// into rows 0, 1, 2 of out (row stride ldc); part holds comp_sums_scratch
// doubles (per-chunk partial sums, added in chunk order).
int64_t comp_sums_scratch(int32_t n, int64_t ldc);
void launch_comp_sums(const ElemRec *el, int32_t nd, int32_t ne, int32_t n, double lin,
                      double quad, const PhaseDev &ph, double *part, double *out, int64_t ldc,
                      cudaStream_t s);
// iscale: per-component scale factors by least squares (svdfit.cpp:22-80) from
// fcomp (5 per point; nc = 5 with star 2's column, else 4), or the given sfac
// when scaling is off; then calc and, when scaled or rdata, chi**2 / wnok into
// out[0..1] with out[2] = 1. work holds 6 n doubles.
void launch_iscale(int32_t flags, int32_t nc, const DatumRec *data, int32_t n,
                   const double *fcomp, double *work, double *calc, double *sfac, double *out,
                   cudaStream_t s);

}  // namespace lcg
