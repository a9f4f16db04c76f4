// geometry.cu — the FP64 stages of one light curve, compiled with
// --fmad=false so that every product and sum rounds as in the reference:
//   k_grid       face radius solve, normal, gravity, area (set_star_grid.cpp:226-523)
//   k_ecl_pre    sphere pre-test + compaction of Roche eclipse candidates
//   k_ecl_roche  ingress/egress of the candidates from a work queue
//   k_continuum  gravity darkening, irradiation, black body (set_star_continuum.cpp)
//   k_flat_*     stable partition into FlatGrid order (comp_light_flat.cpp:26-65)
//   k_phases     per-point phase and sub-exposure entries (light_curve_comp.cpp:350-455)
//   k_scatter    merge of the flux partials into the light curve (:457-498)
//   k_finalize   scale factor and chi**2 (re_scale.cpp:16-42, light_curve_comp.cpp:557-585)
//   k_diag       sums behind logg and the volume-averaged radius (comp_gravity.cpp, comp_radius.cpp)
#include <stdlib.h>

#include "eclipse.cuh"
#include "engine.h"
#include "fixed_phase.cuh"

namespace lcg {

namespace {

__device__ __forceinline__ void set_status(DevStatus *st, int code, int64_t face) {
    if (atomicCAS(&st->code, 0, code) == 0) st->face = (int32_t)face;
}

// One half-face h of a grid and its mirror partner.
__device__ __forceinline__ void grid_half(const GridParams &p, const RingRec *__restrict__ rings,
                                          GridDev g, int64_t h, DevStatus *st) {
    int lo = 0, hi = p.nrings - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (rings[mid].hoff <= h) lo = mid;
        else hi = mid - 1;
    }
    const RingRec R = rings[lo];
    const int np = (int)(h - R.hoff);
    const double phi = R.phi1 + R.span * (np + 0.5) / R.nphi;
    const double sinp = sin(phi), cosp = cos(phi);
    const V3 dirn = p.npole ? v3(R.sint * cosp, R.sint * sinp, R.cost)
                            : v3(R.cost, R.sint * cosp, R.sint * sinp);
    const V3 cofm = p.star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    double rad, gravity;
    V3 posn, dvec;
    if (p.roche) {
        int fail = face_chop(p.star, p.q, p.spin, dirn.x, dirn.y, p.rref, p.pref, p.acc, rad);
        if (fail) {
            // the reference re-runs the scalar Roche::face on such lanes
            if (face_scalar(p.star, p.q, p.spin, dirn, p.rref, p.pref, p.acc, posn, dvec, rad,
                            gravity)) {
                set_status(st, 3, R.off + np);
                return;
            }
        } else {
            posn = add(cofm, scale(rad, dirn));
            dvec = drpot(p.star, p.q, p.spin, posn);
            gravity = len(dvec);
            dvec.x /= gravity;
            dvec.y /= gravity;
            dvec.z /= gravity;
        }
    } else {
        rad = p.rad_sphere;
        posn = add(cofm, scale(rad, dirn));
        dvec = dirn;
        gravity = 1.;
    }
    const double area = (R.span / R.nphi * rad * R.sint) * (R.latspan / R.nl * rad) / dot(dirn, dvec);
    const float af = (float)area, gf = (float)(gravity / p.gref);
    // a tiled face past the reference's face count is dropped (its vector
    // ends there, set_star_grid.cpp:162-166)
    int64_t i = R.off + np;
    if (i < g.n) {
        g.px[i] = posn.x; g.py[i] = posn.y; g.pz[i] = posn.z;
        g.nx[i] = dvec.x; g.ny[i] = dvec.y; g.nz[i] = dvec.z;
        g.area[i] = af;
        g.grav[i] = gf;
    }
    const int np2 = R.nphi - 1 - np;
    if (np2 != np && R.off + np2 < g.n) {
        i = R.off + np2;
        if (p.npole) {
            g.px[i] = posn.x; g.py[i] = -posn.y; g.pz[i] = posn.z;
            g.nx[i] = dvec.x; g.ny[i] = -dvec.y; g.nz[i] = dvec.z;
        } else {
            g.px[i] = posn.x; g.py[i] = posn.y; g.pz[i] = -posn.z;
            g.nx[i] = dvec.x; g.ny[i] = dvec.y; g.nz[i] = -dvec.z;
        }
        g.area[i] = af;
        g.grav[i] = gf;
    }
}

__global__ void k_grid(GridParams p, const RingRec *__restrict__ rings, GridDev g,
                       DevStatus *st) {
    const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (h < p.nhalf) grid_half(p, rings, g, h, st);
}

// Sphere test of face i: a spherical eclipser sets the range directly; a
// Roche eclipser makes the face a candidate.
__device__ __forceinline__ bool ecl_pre_face(const EclParams &p, int32_t eclipse_on, GridDev g,
                                             int64_t i) {
    bool cand = false;
    if (i >= g.ntiled) {
        // a default Point (lcurve.h:53-54): no face of the tiling lands here
        g.px[i] = g.py[i] = g.pz[i] = 0.;
        g.nx[i] = g.ny[i] = g.nz[i] = 0.;
        g.area[i] = 0.f;
        g.grav[i] = 1.f;
        g.necl[i] = 0;
        g.ein[i] = g.eout[i] = 0.;
    } else {
        g.necl[i] = 0;
        g.ein[i] = 0.;
        g.eout[i] = 0.;
        if (eclipse_on) {
            const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
            const V3 cofm = p.comp_star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
            double phi1, phi2, lam1, lam2;
            if (p.comp_roche) {
                cand = sphere_eclipse_ph(p.cosi, p.sini, pos, cofm, p.comp_rref, phi1, phi2,
                                         lam1, lam2);
            } else if (sphere_eclipse_ph(p.cosi, p.sini, pos, cofm, p.comp_r, phi1, phi2, lam1,
                                         lam2)) {
                g.necl[i] = 1;
                g.ein[i] = phi1;
                g.eout[i] = phi2;
            }
        }
    }
    return cand;
}

// Appends the candidates of a full warp to the queue (warp-aggregated).
__device__ __forceinline__ void queue_push(bool cand, int32_t item, int32_t *queue,
                                           int32_t *counters) {
    const unsigned mask = __ballot_sync(0xffffffffu, cand);
    if (mask) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(mask) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&counters[0], __popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (cand) queue[base + __popc(mask & ((1u << lane) - 1u))] = item;
    }
}

// Sphere test of every face; Roche eclipsers queue their candidates.
__global__ void k_ecl_pre(EclParams p, int32_t eclipse_on, GridDev g, int32_t *queue,
                          int32_t *counters) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool cand = i < g.n && ecl_pre_face(p, eclipse_on, g, i);
    queue_push(cand, (int32_t)i, queue, counters);
}

// Ingress/egress of the queued candidates. Up to warp_max candidates, one
// warp bisects each face (ingress_egress_warp): few candidates leave most of
// the GPU idle otherwise. Beyond that, k_ecl_potmin and k_ecl_bisect take
// over (one thread per candidate, each warp taking 32 consecutive candidates
// at a time so that neighbouring faces, with similar iteration counts, run in
// lockstep) and this kernel returns at once. The count is read on the device,
// so the choice needs no host round trip.
__global__ void __launch_bounds__(128, 4) k_ecl_roche(EclParams p, GridDev g,
                                                   const int32_t *__restrict__ queue,
                                                   int32_t *counters, DevStatus *st,
                                                   int32_t warp_max) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = counters[0];
    if (total <= warp_max) {
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&counters[1], 1);
            k = __shfl_sync(full, k, 0);
            if (k >= total) break;
            const int32_t i = queue[k];
            const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
            double ing = 0., egr = 0.;
            int s = 0;
            const bool ecl = ingress_egress_warp(p.comp_star, p.q, p.comp_spin, p.cosi, p.sini,
                                                 p.delta, pos, p.comp_rref, p.comp_pref, ing,
                                                 egr, s);
            if (lane == 0) {
                if (s) {
                    set_status(st, s, i);
                } else if (ecl) {
                    g.necl[i] = 1;
                    g.ein[i] = ing;
                    g.eout[i] = egr;
                }
            }
        }
        return;
    }
}

// Appends the eclipsed candidates k of a warp's 32 (lanes with hit) to the
// list the bisection pass walks, in lane order, so that warps bisect only
// faces pot_min found eclipsed (consecutive candidates stay together). All 32
// lanes call it.
__device__ __forceinline__ void push_hits(bool hit, int k, int32_t *hits, int32_t *count) {
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    int at = 0;
    if (lane == 0) at = atomicAdd(count, __popc(m));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (hit) hits[at + __popc(m & ((1u << lane) - 1u))] = k;
}

// One test of a bisection: the FP32 screen where p.scr allows it (it decides
// only where the FP64 test's answer is certain, so the bisection takes the
// same midpoints), else Roche::fblink in FP64. u0: the point relative to the
// eclipser's centre, in FP32.
__device__ __noinline__ int ecl_screen_test(const EclScreen scr, float cosi, float sini,
                                            double pmid, float u0x, float u0y, float u0z,
                                            float acc) {
    const double ph = pmid - rint(pmid);  // |ph| <= 1/2 keeps the FP32 angle fine
    float sn, cs;
    sincospif(2.f * (float)ph, &sn, &cs);
    return fblink_screen(scr, u0x, u0y, u0z, sini * cs, -sini * sn, cosi, acc);
}

// The bisection of ingress (side 0) or egress (side 1) of ingress_egress
// (ingress_egress.cpp:61-86) from the pot_min state, for every lane of a warp
// at once (all 32 lanes call it; lanes with live false only vote). Each lane
// screens its midpoints in FP32 until one is unsure; when no live lane can go
// on, the warp runs Roche::fblink in FP64 for all the lanes waiting on one, in
// a single pass, and the screening resumes. The FP64 passes are thus packed
// (one per test of the lane that needs the most, instead of one per step
// whenever any lane needs one), and the lanes take the FP64 decisions at the
// same midpoints as the plain loop. With the screen off it is the plain loop.
__device__ __forceinline__ double ecl_bisect_warp(const EclParams &p, bool live, double pin,
                                                  double pout, double acc, V3 pos, int &s) {
    // what the screening loop reads, in registers (p may be global memory;
    // the FP64 test, a third of the steps, reads the rest from it)
    const EclScreen scr = p.scr;
    const double delta = p.delta;
    const float cif = (float)p.cosi, sif = (float)p.sini, accf = (float)acc;
    const float u0x = (float)(pos.x - (p.comp_star == kStar1 ? 0. : 1.));
    const float u0y = (float)pos.y, u0z = (float)pos.z;
    bool done = !live;
    int guard = 0;
    double pmid = 0.;
    for (;;) {
        bool need = false;
        while (!done) {
            if (!(fabs(pin - pout) > delta)) { done = true; break; }
            if (++guard > 400) { s = kEclNoConverge; done = true; break; }
            pmid = (pin + pout) / 2.;
            if (!scr.on) { need = true; break; }
            const int d = ecl_screen_test(scr, cif, sif, pmid, u0x, u0y, u0z, accf);
            if (d == kScreenUnsure) { need = true; break; }
            if (d == kScreenTrue) pin = pmid;
            else pout = pmid;
        }
        if (!__any_sync(0xffffffffu, need)) break;
        if (need) {
            if (fblink(p.comp_star, p.q, p.comp_spin, acc, set_earth(p.cosi, p.sini, pmid), pos,
                       p.comp_rref, p.comp_pref, s))
                pin = pmid;
            else
                pout = pmid;
            if (s) done = true;
        }
    }
    return (pin + pout) / 2.;
}

// Thread mode (more candidates than warp_max), in two passes with a small code
// footprint each, as for the batch (k_ecl_potmin_b / k_ecl_bisect_b): the
// sphere test and pot_min per candidate, then ingress and egress on the two
// lanes of a pair. es holds each candidate's state between the passes, hits
// the candidates pot_min found eclipsed.
__global__ void __launch_bounds__(128, 4) k_ecl_potmin(EclParams p, GridDev g,
                                                    const int32_t *__restrict__ queue,
                                                    int32_t *counters, double4 *es, int32_t *hits,
                                                    DevStatus *st, int32_t warp_max) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = counters[0];
    if (total <= warp_max) return;
    const V3 cofm = p.comp_star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&counters[2], 32);
        base = __shfl_sync(full, base, 0);
        if (base >= total) break;
        const int k = base + lane;
        bool hit = false;
        if (k < total) {
            const int32_t i = queue[k];
            const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
            double phi1, phi2, lam1, lam2, phi = 0., lam = 0.;
            if (sphere_eclipse_ph(p.cosi, p.sini, pos, cofm, p.comp_rref, phi1, phi2, lam1,
                                  lam2)) {
                const double ACC = 2. * sqrt(2. * kTwoPi * (lam2 - lam1) * p.delta);
                int s = 0;
                hit = pot_min(p.comp_star, p.q, p.comp_spin, p.cosi, p.sini, pos, phi1, phi2,
                              lam1, lam2, p.comp_rref, p.comp_pref, ACC, phi, lam, s);
                if (s) {
                    set_status(st, s, i);
                    hit = false;
                }
                es[k] = make_double4(phi, phi1, phi2, ACC);
            }
        }
        push_hits(hit, k, hits, &counters[6]);
    }
}

template <int NB>
__global__ void __launch_bounds__(128, NB)
    k_ecl_bisect(__grid_constant__ const EclParams p, __grid_constant__ const GridDev g,
                 const int32_t *__restrict__ queue, int32_t *counters, const double4 *es,
                 const int32_t *__restrict__ hits, DevStatus *st, int32_t warp_max) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = counters[0];
    if (total <= warp_max) return;
    const int64_t n2 = 2 * (int64_t)counters[6];
    for (;;) {
        int64_t base = 0;
        if (lane == 0) base = atomicAdd(&counters[3], 32);
        base = __shfl_sync(full, base, 0);
        if (base >= n2) break;
        // every lane stays here (ecl_bisect_warp votes over the warp); both
        // lanes of a pair agree on live
        const int64_t u = base + lane;
        const int side = (int)(u & 1);
        const bool live = u < n2;
        const int k = live ? hits[u >> 1] : 0;
        const int32_t i = live ? queue[k] : 0;
        const double4 E = live ? es[k] : make_double4(0., 0., 0., 0.);
        const V3 pos = live ? v3(g.px[i], g.py[i], g.pz[i]) : v3(0., 0., 0.);
        int s = 0;
        double v = ecl_bisect_warp(p, live, E.x, side ? E.z : E.y, E.w, pos, s);
        v = v - floor(v);
        const double other = __shfl_xor_sync(full, v, 1);
        const int os = __shfl_xor_sync(full, s, 1);
        if (live && side == 0) {
            if (s || os) {
                set_status(st, s ? s : os, i);
            } else {
                double egr = other;
                if (egr < v) egr++;
                g.necl[i] = 1;
                g.ein[i] = v;
                g.eout[i] = egr;
            }
        }
    }
}

__device__ __forceinline__ void continuum_face(const ContParams &p, GridDev g, int64_t i) {
    if (i >= g.ntiled) {  // default Point: zero area, zero flux
        g.flux[i] = 0.f;
        return;
    }
    const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
    const V3 dir = v3(g.nx[i], g.ny[i], g.nz[i]);
    const V3 cofm_other = p.star == kStar1 ? v3(1., 0., 0.) : v3(0., 0., 0.);
    const V3 vec = sub(cofm_other, pos);
    const double r = len(vec);
    const double mu = dot(dir, vec) / r;
    const double EFAC = p.efac;
    double t;
    if (p.star == kStar1) {
        t = p.t_own;
        for (int k = 0; k < p.nspot; k++) {
            const V3 sd = v3(p.spot_dir[k][0], p.spot_dir[k][1], p.spot_dir[k][2]);
            double dist = rad2deg(acos(dot(pos, sd) / len(pos)));
            t += (p.spot_tcen[k] - p.t_own) * exp(-sq(dist / (p.spot_fwhm[k] / EFAC)) / 2.);
        }
        if (p.uesp_on) {
            const V3 evec = v3(pos.x, pos.y, 0);
            const double evecl = len(evec);
            if (evecl > 0.) {
                double rd = len(pos);
                double clat = dot(pos, evec) / evecl / rd;
                clat = dmin(1.0, dmax(-1., clat));
                double dlat = rad2deg(acos(clat));
                double clong = dot(v3(p.uesp_dir[0], p.uesp_dir[1], p.uesp_dir[2]), evec) / evecl;
                clong = dmin(1.0, dmax(-1., clong));
                double dlong = rad2deg(acos(clong));
                if (dlat <= p.uesp_lathw && dlong <= p.uesp_longhw) {
                    t = p.uesp_temp;
                } else if (dlat <= p.uesp_lathw) {
                    t += (p.uesp_temp - p.t_own) * exp(-(dlong - p.uesp_longhw) / p.uesp_taper);
                } else if (dlong <= p.uesp_longhw) {
                    t += (p.uesp_temp - p.t_own) * exp(-(dlat - p.uesp_lathw) / p.uesp_taper);
                } else {
                    t += (p.uesp_temp - p.t_own) * exp(-(dlat - p.uesp_lathw) / p.uesp_taper) *
                         exp(-(dlong - p.uesp_longhw) / p.uesp_taper);
                }
            }
        }
    } else {
        t = fabs(p.t_own);
        for (int k = 0; k < p.nspot; k++) {
            const V3 sd = v3(p.spot_dir[k][0], p.spot_dir[k][1], p.spot_dir[k][2]);
            const V3 off = sub(pos, v3(1., 0., 0.));
            double dist = rad2deg(acos(dot(off, sd) / len(off)));
            t += (p.spot_tcen[k] - t) * exp(-sq(dist / (p.spot_fwhm[k] / EFAC)) / 2.);
        }
    }
    if (p.fp32) {
        // the intensity in FP32 (the face's flux is stored as a float): the same
        // formulas as below; x^(1/4) as two square roots, Planck from its
        // constants over the wavelength, set on the host
        const float gd = powf(g.grav[i], (float)p.gdcbol);
        const float tg = (float)t * gd, tg2 = tg * tg;
        const double rc = p.rcomp;
        double geom = 0.;
        float temp = tg;
        if (mu > -rc) {
            if (mu >= rc) {
                geom = sq(rc / r) * mu;
            } else {
                double x0 = -mu / rc;
                geom = sq(rc / r) * rc *
                       (sqrt(1. - x0 * x0) * (2 + x0 * x0) / 3 - x0 * (kPi / 2 - asin(x0))) / kPi;
            }
            temp = sqrtf(sqrtf(fmaf(tg2, tg2, p.irr32 * (float)geom)));
        }
        const float area = g.area[i];
        float f = area * (p.planck_c1 / (expf(p.planck_c2 / temp) - 1.f));
        if (p.mirror) {
            const float tm = (float)(p.star == kStar1 ? fabs(p.t_other) : p.t_other);
            f = fmaf(area * (float)geom, p.planck_c1 / (expf(p.planck_c2 / tm) - 1.f), f);
        }
        g.flux[i] = f;
        return;
    }
    const double gd = pow((double)g.grav[i], p.gdcbol);
    const double rc = p.rcomp;
    // pow(t_other, 4) for star 1 and pow(t_other, 4.) for star 2 are the same call
    const double irr = p.absorb * pow(p.t_other, 4.);
    double temp, geom;
    if (mu >= rc) {
        geom = sq(rc / r) * mu;
        temp = pow(pow(t * gd, 4.0) + irr * geom, 0.25);
    } else if (mu > -rc) {
        double x0 = -mu / rc;
        geom = sq(rc / r) * rc * (sqrt(1. - x0 * x0) * (2 + x0 * x0) / 3 - x0 * (kPi / 2 - asin(x0))) /
               kPi;
        temp = pow(pow(t * gd, 4.0) + irr * geom, 0.25);
    } else {
        geom = 0.;
        temp = t * gd;
    }
    float f = (float)(g.area[i] * planck(p.wavelength, temp));
    if (p.mirror) {
        const double tm = p.star == kStar1 ? fabs(p.t_other) : p.t_other;
        f = (float)(f + g.area[i] * geom * planck(p.wavelength, tm));
    }
    g.flux[i] = f;
}

__global__ void k_continuum(ContParams p, GridDev g) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < g.n) continuum_face(p, g, i);
}

constexpr int kFlatBlock = 1024;

// Eclipse class of face i for the FlatGrid partition (comp_light_flat.cpp:26-65):
// 0 never eclipsed, 1 one range, 2 several (an opaque disc's ranges added to
// the companion's).
__device__ __forceinline__ int flat_class(const GridDev &g, int64_t i) {
    const int k = g.necl[i] + (g.ndx ? g.ndx[i] : 0);
    return k < 2 ? k : 2;
}

// Per 1024-face block: the one-range count in blockcnt[b], the several-range
// count in blockcnt[nb + b].
__global__ void k_flat_count(GridDev g, int32_t *blockcnt) {
    const int64_t i = blockIdx.x * (int64_t)kFlatBlock + threadIdx.x;
    const int cls = i < g.n ? flat_class(g, i) : 0;
    const int c1 = __syncthreads_count(cls == 1);
    const int c2 = g.ndx ? __syncthreads_count(cls == 2) : 0;
    if (threadIdx.x == 0) {
        blockcnt[blockIdx.x] = c1;
        blockcnt[gridDim.x + blockIdx.x] = c2;
    }
}

// Single block: exclusive scan of the per-block eclipse counts; n0 = faces
// never eclipsed.
__device__ __forceinline__ void scan_blocks(int32_t *blockcnt, int32_t nb, int64_t n,
                                            int64_t *n0) {
    __shared__ int32_t part[1024];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? blockcnt[i] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int t = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
            __syncthreads();
            part[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nb) blockcnt[i] = (int32_t)(carry + part[threadIdx.x] - v);
        __syncthreads();
        if (threadIdx.x == 1023) carry += part[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *n0 = n - carry;
    __syncthreads();
}

// Both counts scanned: n0 = faces never eclipsed, n1 = n0 + one-range faces
// (n0[0] and n0[1]).
__global__ void k_flat_scan(int32_t *blockcnt, int32_t nb, int64_t n, int64_t *n0) {
    __shared__ int64_t c2;
    int64_t t2 = 0;
    scan_blocks(blockcnt + nb, nb, n, n0);  // n0[0] = n - (several-range faces)
    if (threadIdx.x == 0) c2 = n - n0[0];
    __syncthreads();
    t2 = c2;
    scan_blocks(blockcnt, nb, n - t2, n0);  // n0[0] = n - several - one-range
    if (threadIdx.x == 0) n0[1] = n - t2;
}

// Face i's record of the fast mixed sweep at flat position dest (pairs of
// faces interleaved, FlatDev::fp).
__device__ __forceinline__ void fast_record(float *fp, int64_t dest, GridDev g, int64_t i,
                                            const FastCoef &fc) {
    const double fl = (double)g.flux[i];
    float *r = fp + 16 * (dest >> 1) + (dest & 1);
    r[0] = (float)g.nx[i];
    r[2] = (float)g.ny[i];
    r[4] = (float)(fc.cosi * g.nz[i]);
    r[6] = (float)(fl * fc.p[0]);
    r[8] = (float)(fl * fc.p[1]);
    r[10] = (float)(fl * fc.p[2]);
    r[12] = (float)(fl * fc.p[3]);
    r[14] = (float)(fl * fc.p[4]);
}

// Stable three-way partition [never | one range | several]. Several-range
// faces get all-zero records (they add exact zeros to the main sweeps) and
// their face index and ranges in FlatGrid order; k_flux_ragged adds them.
__global__ void k_flat_scatter(GridDev g, FlatDev f, const int32_t *__restrict__ blockoff,
                               int mixed, int need_pos, FastCoef fc) {
    __shared__ int32_t warp_tot[2][32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t i = blockIdx.x * (int64_t)kFlatBlock + t;
    const bool in = i < g.n;
    const int cls = in ? flat_class(g, i) : 0;
    const unsigned m1 = __ballot_sync(0xffffffffu, cls == 1);
    const unsigned m2 = __ballot_sync(0xffffffffu, cls == 2);
    if (lane == 0) {
        warp_tot[0][w] = __popc(m1);
        warp_tot[1][w] = __popc(m2);
    }
    __syncthreads();
    int b1 = 0, b2 = 0;
    for (int k = 0; k < w; k++) {
        b1 += warp_tot[0][k];
        b2 += warp_tot[1][k];
    }
    const unsigned below = (1u << lane) - 1u;
    const int rank1 = b1 + __popc(m1 & below), rank2 = b2 + __popc(m2 & below);
    if (!in) return;
    const int64_t n0 = f.n0[0], n1 = f.n0[1];
    const int64_t boff1 = blockoff[blockIdx.x], boff2 = blockoff[gridDim.x + blockIdx.x];
    const int64_t dest = cls == 1   ? n0 + boff1 + rank1
                         : cls == 2 ? n1 + boff2 + rank2
                                    : blockIdx.x * (int64_t)kFlatBlock - boff1 - boff2 +
                                          (t - rank1 - rank2);
    // a one-range face's range: the companion's, else the disc's first
    double ein = 0., eout = 0.;
    if (cls == 1) {
        if (g.necl[i]) { ein = g.ein[i]; eout = g.eout[i]; }
        else { ein = g.xr[kDiscRanges * i].x; eout = g.xr[kDiscRanges * i].y; }
    }
    const bool live = cls < 2;
    if (mixed) {
        if (fc.on) {
            if (live) {
                fast_record(f.fp, dest, g, i, fc);
            } else {
                float *r = f.fp + 16 * (dest >> 1) + (dest & 1);
                for (int q = 0; q < 16; q += 2) r[q] = 0.f;
            }
        } else {
            f.geo[dest] = live ? make_float4((float)g.nx[i], (float)g.ny[i], (float)g.nz[i],
                                             g.flux[i])
                               : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        f.ecl[dest] = cls == 1 ? ecl_fx64(ein, eout) : make_ulonglong2(0ull, 0ull);
        if (need_pos)
            f.pos[dest] = live ? make_float4((float)g.px[i], (float)g.py[i], (float)g.pz[i], 0.f)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
        const double z = 0.;
        f.dx[dest] = live ? g.nx[i] : z; f.dy[dest] = live ? g.ny[i] : z;
        f.dz[dest] = live ? g.nz[i] : z;
        f.px[dest] = live ? g.px[i] : z; f.py[dest] = live ? g.py[i] : z;
        f.pz[dest] = live ? g.pz[i] : z;
        f.flux[dest] = live ? (double)g.flux[i] : z;
        f.in1[dest] = ein;
        f.out1[dest] = eout;
    }
    if (cls == 2) {
        const int64_t r = dest - n1;
        int q = 0;
        if (g.necl[i]) f.rr[kRagRanges * r + q++] = make_double2(g.ein[i], g.eout[i]);
        for (int k = 0; k < g.ndx[i]; k++) f.rr[kRagRanges * r + q++] = g.xr[kDiscRanges * i + k];
        f.rn[r] = (uint8_t)q;
        f.ridx[r] = (int32_t)i;
    }
}

// Orbital phase of one point (4 Newton steps with pdot, the deltat shift)
// and its polynomial scale factor (light_curve_comp.cpp:358-376).
__device__ __forceinline__ void point_phase(const PhaseParams &p, const DatumRec &d,
                                            double &phase, double &slfac) {
    phase = (d.time - p.t0) / p.period;
    for (int it = 0; it < 4; it++)
        phase -= (p.t0 + phase * (p.period + p.pdot * phase) - d.time) /
                 (p.period + 2. * p.pdot * phase);
    phase += p.deltat / p.period / 2. * (cos(2. * kPi * phase) - 1.);
    const double frac = (d.time - p.middle) / p.range;
    slfac = 1. + frac * (p.slope + frac * (p.quad + frac * p.cube));
}

// Phase and trapezoid weight of sub-exposure nd (light_curve_comp.cpp:416-455).
__device__ __forceinline__ void sub_exposure(double phase, double expose, int ndiv, int nd,
                                             double &phi, double &wgt) {
    if (ndiv == 1) {
        phi = phase;
        wgt = 1.0;
    } else {
        phi = phase + expose * (nd - (ndiv - 1) / 2.0) / (ndiv - 1);
        wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
    }
}

__global__ void k_phases(PhaseParams p, const DatumRec *__restrict__ data,
                         const int64_t *__restrict__ off, int32_t n, PhaseDev ph) {
    const int np = blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= n) return;
    const DatumRec d = data[np];
    double phase, slfac;
    point_phase(p, d, phase, slfac);
    const double expose = d.expose / p.period;
    const int ndiv = d.ndiv;
    const double norm = (ndiv - 1 > 1) ? ndiv - 1 : 1;
    int64_t e = off[np];
    for (int nd = 0; nd < ndiv; ++nd, ++e) {
        double phi, wgt;
        sub_exposure(phase, expose, ndiv, nd, phi, wgt);
        const V3 earth = set_earth(p.cosi, p.sini, phi);
        const double phin = phi - floor(phi);
        ph.ex[e] = earth.x;
        ph.ey[e] = earth.y;
        ph.ez[e] = earth.z;
        ph.phin[e] = phin;
        ph.w1[e] = slfac * wgt * gi_scale1(p.gi, phi) / norm;
        ph.w2[e] = slfac * wgt * gi_scale2(p.gi, phi) / norm;
        ph.type[e] = (uint8_t)gi_type(p.gi, phi);
        ph.ef[e] = make_float4((float)earth.x, (float)earth.y, (float)earth.z, 0.f);
        ph.pfx[e] = phase_fx64(phin);
    }
}

// Sum of the chunk partials of every phase entry, chunks in order (for the
// FP64 sweep: the reference's block order). One thread per (sweep, entry);
// consecutive threads read consecutive entries of a chunk row.
__global__ void k_reduce_chunks(ReduceParams p) {
    const int s = blockIdx.y;
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const double *__restrict__ part = p.part[s];
    if (!part || e >= p.nent[s]) return;
    const int64_t nc = p.nchunk[s], ldp = p.ldp;
    double o = 0.0;
    int64_t c = 0;
    for (; c + 8 <= nc; c += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = part[(c + u) * ldp + e];
#pragma unroll
        for (int u = 0; u < 8; u++) o += v[u];
    }
    for (; c < nc; c++) o += part[c * ldp + e];
    p.osum[s][e] = o;
}

// Per data point: weighted sub-exposure sums of the four sweeps in the
// reference's order (pb1f, pb1c, pb2f, pb2c, light_curve_comp.cpp:476-480),
// then third light.
__global__ void k_scatter(ScatterParams p, const double *__restrict__ o1f,
                          const double *__restrict__ o1c, const double *__restrict__ o2f,
                          const double *__restrict__ o2c, PhaseDev ph,
                          const DatumRec *__restrict__ data, const int64_t *__restrict__ off,
                          int32_t n, double *calc) {
    const int np = blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= n) return;
    const int64_t e0 = off[np], e1 = e0 + (data[np].ndiv > 0 ? data[np].ndiv : 0);
    double c = 0.;
    for (int64_t e = e0; e < e1; e++)
        if (p.copy1 || ph.type[e] == 1) c += ph.w1[e] * o1f[e];
    if (!p.copy1)
        for (int64_t e = e0; e < e1; e++)
            if (ph.type[e] != 1) c += ph.w1[e] * o1c[e];
    double c2 = 0.;
    double *acc = p.fcomp ? &c2 : &c;  // iscale keeps the stars apart
    for (int64_t e = e0; e < e1; e++)
        if (p.copy2 || ph.type[e] == 3) *acc += ph.w2[e] * o2f[e];
    if (!p.copy2)
        for (int64_t e = e0; e < e1; e++)
            if (ph.type[e] != 3) *acc += ph.w2[e] * o2c[e];
    if (p.csum || p.fcomp) {
        // comp_disc / comp_edge / comp_spot of the point: sub-exposure sums
        // weighted and merged in order, over max(1, ndiv - 1)
        // (comp_light.cpp:323-408, light_curve_comp.cpp:476-490, 378-414)
        const DatumRec d = data[np];
        double phase, slfac;
        point_phase(p.pp, d, phase, slfac);
        const int ndiv = d.ndiv;
        double cd = 0.0, ce = 0.0, cs = 0.0;
        if (p.csum) {
            for (int nd = 0; nd < ndiv; nd++) {
                const int64_t e = e0 + nd;
                const double wgt = ndiv == 1 ? 1.0 : ((nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0);
                cd += wgt * p.csum[e];
                ce += wgt * p.csum[p.ldc + e];
                cs += wgt * p.csum[2 * p.ldc + e];
            }
            const int norm = (ndiv - 1 > 1) ? ndiv - 1 : 1;
            cd /= norm;
            ce /= norm;
            cs /= norm;
        }
        if (p.fcomp) {
            double *f = p.fcomp + 5 * (int64_t)np;
            f[0] = c;
            f[1] = slfac * cd;
            f[2] = slfac * ce;
            f[3] = slfac * cs;
            f[4] = c2;
            calc[np] = 0.;
            return;
        }
        c += slfac * (cd + ce + cs);
    }
    calc[np] = c + p.third;
}

// Fixed-shape tree over the 1024 threads of the block: deterministic.
__device__ __forceinline__ double block_sum(double v, double *sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// One block of 1024 threads: thread t takes points t, t+1024, ... in order,
// the block sums them in a fixed tree.
__device__ __forceinline__ void finalize_block(int32_t flags, const DatumRec *__restrict__ data,
                                               int32_t n, double *calc, double *sfac_io,
                                               double *out, double *sh) {
    const bool scale = flags & 1, rdata = flags & 2;
    const int t = threadIdx.x;
    if (scale) {
        double a = 0., b = 0., w = 0.;
        for (int i = t; i < n; i += 1024) {
            const DatumRec d = data[i];
            if (d.weight > 0.) {
                const double wgt = d.weight / sq(d.ferr);
                a += wgt * d.flux * calc[i];
                b += wgt * calc[i] * calc[i];
                w += d.weight;
            }
        }
        const double sdy = block_sum(a, sh), syy = block_sum(b, sh), wnok = block_sum(w, sh);
        const bool ok = wnok > 0.0;
        const double sc = ok ? sdy / syy : 1.;
        if (t == 0) {
            out[1] = wnok;
            for (int k = 0; k < 5; k++) sfac_io[k] = sc;
        }
        if (!ok) {
            if (t == 0) {
                out[0] = 0.;
                out[2] = 1.;
            }
            return;
        }
        for (int i = t; i < n; i += 1024) calc[i] = calc[i] * sc;
    } else {
        const double sc = sfac_io[0];
        for (int i = t; i < n; i += 1024) calc[i] *= sc;
        if (!rdata) {
            if (t == 0) out[2] = 0.;
            return;
        }
    }
    double cs = 0., w = 0.;
    for (int i = t; i < n; i += 1024) {
        const DatumRec d = data[i];
        if (d.weight > 0.) {
            cs += d.weight * sq((d.flux - calc[i]) / d.ferr);
            w += d.weight;
        }
    }
    const double chisq = block_sum(cs, sh), wnok = block_sum(w, sh);
    if (t == 0) {
        out[0] = chisq;
        if (!scale) out[1] = wnok;
        out[2] = 1.;
    }
}

__global__ void __launch_bounds__(1024) k_finalize(int32_t flags, const DatumRec *__restrict__ data,
                                                   int32_t n, double *calc, double *sfac_io,
                                                   double *out) {
    __shared__ double sh[1024];
    finalize_block(flags, data, n, calc, sfac_io, out, sh);
}

// light_curve_comp_fast's interpolation (light_curve_comp_fast.cpp:46-83):
// point i takes the model at the sampled points around it (sample indices
// idx[0..m), ascending), linearly in time; with rdata, chi**2 and wnok over
// all points (out[0], out[1]). One block of 1024 threads, fixed-order tree.
__global__ void __launch_bounds__(1024) k_interp(const DatumRec *__restrict__ data, int32_t n,
                                                 const int64_t *__restrict__ idx, int32_t m,
                                                 const double *__restrict__ mc, double *calc,
                                                 int32_t rdata, double *out) {
    __shared__ double sh[1024];
    const int t = threadIdx.x;
    double cs = 0., w = 0.;
    for (int i = t; i < n; i += 1024) {
        int lo = 0, hi = m;  // first sample index >= i
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (idx[mid] < i) lo = mid + 1;
            else hi = mid;
        }
        double c;
        if (lo == 0) {
            c = mc[0];
        } else if (lo == m) {
            c = mc[m - 1];
        } else {
            const int64_t i1 = idx[lo - 1], i2 = idx[lo];
            const double tt = (data[i].time - data[i1].time) / (data[i2].time - data[i1].time);
            c = mc[lo - 1] * (1.0 - tt) + mc[lo] * tt;
        }
        calc[i] = c;
        const DatumRec d = data[i];
        if (d.weight > 0.) {
            w += d.weight;
            cs += d.weight * sq((d.flux - c) / d.ferr);
        }
    }
    if (!rdata) return;
    const double chisq = block_sum(cs, sh), wnok = block_sum(w, sh);
    if (t == 0) {
        out[0] = chisq;
        out[1] = wnok;
    }
}

// Bound of mu over one run of 32 face pairs of the fast records, one warp per
// run (lane l reads pair l): with a = the mean of (nx, ny), R = the largest
// |(nx, ny) - a| and C = the largest cz of the run's faces,
//   mu = ex nx + ey ny + cz <= ex ax + ey ay + |(ex, ey)| R + C.
// R and C are widened well past FP32 rounding (1e-6, 1e-5), so when the bound
// is negative the computed mu of every face of the run is <= 0 and the run adds
// exactly zero. All-zero records (padding) are left out; a run of padding only
// gets C = -1.
// With ecl, also the run's eclipse-range hull: an arc [I, I + W) holding every
// nonempty range (I_f, W_f + 1) of the run's faces, as the record (I, W), or
// W = ~0 for "test every face" (ranges a quarter orbit long or spread over
// more than that), (0, 0) when no face of the run has a range.
__device__ __forceinline__ void run_bound(const float *__restrict__ fp,
                                          const ulonglong2 *__restrict__ ecl, int64_t npairs,
                                          int64_t run, float4 *out, ulonglong2 *hull) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t q = run * 32 + lane;
    float nx[2] = {0.f, 0.f}, ny[2] = {0.f, 0.f}, cz[2] = {0.f, 0.f};
    bool use[2] = {false, false};
    if (q < npairs) {
        const float4 P0 = reinterpret_cast<const float4 *>(fp)[4 * q];
        const float4 P1 = reinterpret_cast<const float4 *>(fp)[4 * q + 1];
        nx[0] = P0.x; nx[1] = P0.y; ny[0] = P0.z; ny[1] = P0.w; cz[0] = P1.x; cz[1] = P1.y;
        for (int k = 0; k < 2; k++) use[k] = nx[k] != 0.f || ny[k] != 0.f || cz[k] != 0.f;
    }
    float sx = 0.f, sy = 0.f, cnt = 0.f;
    for (int k = 0; k < 2; k++)
        if (use[k]) { sx += nx[k]; sy += ny[k]; cnt += 1.f; }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(full, sx, o);
        sy += __shfl_xor_sync(full, sy, o);
        cnt += __shfl_xor_sync(full, cnt, o);
    }
    const float ax = cnt > 0.f ? sx / cnt : 0.f, ay = cnt > 0.f ? sy / cnt : 0.f;
    float r = 0.f, c = -1.f;
    for (int k = 0; k < 2; k++)
        if (use[k]) {
            r = fmaxf(r, sqrtf((nx[k] - ax) * (nx[k] - ax) + (ny[k] - ay) * (ny[k] - ay)));
            c = fmaxf(c, cz[k]);
        }
    for (int o = 16; o > 0; o >>= 1) {
        r = fmaxf(r, __shfl_xor_sync(full, r, o));
        c = fmaxf(c, __shfl_xor_sync(full, c, o));
    }
    if (lane == 0)
        *out = cnt > 0.f ? make_float4(ax, ay, r * (1.f + 1e-6f) + 1e-6f, c + 1e-5f)
                         : make_float4(0.f, 0.f, 0.f, -1.f);
    if (!ecl) return;
    ulonglong2 E[2] = {make_ulonglong2(0ull, 0ull), make_ulonglong2(0ull, 0ull)};
    if (q < npairs) {
        E[0] = ecl[2 * q];
        E[1] = ecl[2 * q + 1];
    }
    const unsigned m = __ballot_sync(full, E[0].y != 0ull || E[1].y != 0ull);
    ulonglong2 H = make_ulonglong2(0ull, 0ull);
    if (m) {
        // offsets from one range's start, as signed 64-bit distances on the circle
        const unsigned long long mine = E[0].y != 0ull ? E[0].x : E[1].x;
        const unsigned long long ref = __shfl_sync(full, mine, __ffs(m) - 1);
        constexpr long long kQuarter = 1ll << 62;
        long long lo = LLONG_MAX, hi = LLONG_MIN;
        bool whole = false;
        for (int k = 0; k < 2; k++)
            if (E[k].y != 0ull) {
                const long long off = (long long)(E[k].x - ref);
                if (E[k].y >= (unsigned long long)kQuarter || off >= kQuarter || off <= -kQuarter) {
                    whole = true;
                } else {
                    lo = off < lo ? off : lo;
                    const long long end = off + (long long)E[k].y;
                    hi = end > hi ? end : hi;
                }
            }
        for (int o = 16; o > 0; o >>= 1) {
            const long long l2 = __shfl_xor_sync(full, lo, o), h2 = __shfl_xor_sync(full, hi, o);
            lo = l2 < lo ? l2 : lo;
            hi = h2 > hi ? h2 : hi;
        }
        whole = __any_sync(full, whole);
        H = whole ? make_ulonglong2(0ull, ~0ull)
                  : make_ulonglong2(ref + (unsigned long long)lo,
                                    (unsigned long long)hi - (unsigned long long)lo);
    }
    if (lane == 0) *hull = H;
}

__global__ void k_run_bounds(const float *__restrict__ fp, const ulonglong2 *__restrict__ ecl,
                             int64_t npairs, float4 *runb, ulonglong2 *runh) {
    const int64_t run = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (run >= (npairs + 31) / 32) return;  // whole warps
    run_bound(fp, ecl, npairs, run, runb + run, runh + run);
}

// Run bounds of the continuum list's slots (16 runs per 1024-face block).
__global__ void k_run_bounds_b(BatchDev b) {
    const int nk = b.counts[1];
    if (nk <= 0) return;
    const int64_t total = b.cont_blk[nk] * 16;
    const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < total;
         w += warps) {
        const int64_t B = w >> 4;
        const int k = find_seg(b.cont_blk, nk, B);
        const SlotDev &S = b.slots[b.cont_slot[k]];
        const int64_t run = (B - b.cont_blk[k]) * 16 + (w & 15);
        run_bound(b.fp + 8 * S.flat0, b.ecl + S.flat0, (S.nface + 1) / 2, run,
                  b.runb + S.flat0 / 64 + run, b.runh + S.flat0 / 64 + run);
    }
}

// dst row r = src row rows[r] (rows of n doubles).
__global__ void k_gather_rows(const double *__restrict__ src, int32_t n,
                              const int32_t *__restrict__ rows, double *dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[(int64_t)blockIdx.y * n + i] = src[(int64_t)rows[blockIdx.y] * n + i];
}

// comp_gravity / comp_radius blocked sums: one thread per 8192-point block,
// serial inside the block; the host merges the blocks in order.
__global__ void k_diag(int star, GridDev g, double *blk) {
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t BLK = 8192, nblk = (g.n + BLK - 1) / BLK;
    if (b >= nblk) return;
    const V3 cofm = star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    double bfg = 0., bf = 0., bsa = 0., bvol = 0.;
    const int64_t end = (g.n < b * BLK + BLK) ? g.n : b * BLK + BLK;
    for (int64_t i = b * BLK; i < end; i++) {
        const float fgv = g.flux[i] * g.grav[i];
        bfg += fgv;
        bf += g.flux[i];
        const V3 vec = sub(v3(g.px[i], g.py[i], g.pz[i]), cofm);
        const double r = len(vec);
        const double rcosa = dot(v3(g.nx[i], g.ny[i], g.nz[i]), vec);
        bsa += g.area[i] * rcosa / pow(r, 3.0);
        bvol += g.area[i] * rcosa;
    }
    blk[4 * b] = bfg;
    blk[4 * b + 1] = bf;
    blk[4 * b + 2] = bsa;
    blk[4 * b + 3] = bvol;
}

// FP64 FlatGrid columns -> the packed mixed-precision view (used when a
// caller hands in a host FlatGrid through lcg_sum_star_multi).
__global__ void k_pack_flat(FlatDev f, int64_t n0, int need_pos) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i == 0) *f.n0 = n0;
    if (i >= f.n) return;
    f.geo[i] = make_float4((float)f.dx[i], (float)f.dy[i], (float)f.dz[i], (float)f.flux[i]);
    f.ecl[i] = i >= n0 ? ecl_fx64(f.in1[i], f.out1[i]) : make_ulonglong2(0ull, 0ull);
    if (need_pos) f.pos[i] = make_float4((float)f.px[i], (float)f.py[i], (float)f.pz[i], 0.f);
}

__global__ void k_pack_phases(PhaseDev ph) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ph.nent) return;
    ph.ef[e] = make_float4((float)ph.ex[e], (float)ph.ey[e], (float)ph.ez[e], 0.f);
    ph.pfx[e] = phase_fx64(ph.phin[e]);
}

// ---- batched stages ---------------------------------------------------------

// The slot's view of the batch point arrays.
__device__ __forceinline__ GridDev slot_grid(const GridDev &g, int64_t face0, int64_t nface,
                                             int64_t ntiled) {
    return GridDev{g.px + face0, g.py + face0, g.pz + face0, g.nx + face0, g.ny + face0,
                   g.nz + face0, g.area + face0, g.grav + face0, g.flux + face0, g.necl + face0,
                   g.ein + face0, g.eout + face0, nface, ntiled};
}

__global__ void __launch_bounds__(128) k_grid_b(BatchDev b) {
    const int nk = b.counts[0];
    if (nk <= 0) return;
    const int64_t total = b.geo_half[nk];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < total; u += stride) {
        const int k = find_seg(b.geo_half, nk, u);
        const SlotDev &S = b.slots[b.geo_slot[k]];
        grid_half(S.gp, b.rings + S.ring0, slot_grid(b.g, S.face0, S.nface, S.ntiled), u - b.geo_half[k],
                  b.st + S.model);
    }
}

// Sphere pre-test of the geometry list's faces; candidates are queued by
// their batch face index. Whole warps step together (queue_push votes).
__global__ void k_ecl_pre_b(BatchDev b) {
    const int nk = b.counts[0];
    if (nk <= 0) return;
    const int64_t total = b.geo_face[nk];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (int64_t u0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); u0 < total;
         u0 += stride) {
        const int64_t u = u0 + lane;
        bool cand = false, scr = false;
        int32_t item = 0;
        if (u < total) {
            const int k = find_seg(b.geo_face, nk, u);
            const SlotDev &S = b.slots[b.geo_slot[k]];
            const int64_t i = u - b.geo_face[k];
            cand = ecl_pre_face(S.ep, S.eclipse_on, slot_grid(b.g, S.face0, S.nface, S.ntiled), i);
            item = (int32_t)(S.face0 + i);
            scr = S.ep.scr.on;
        }
        // screened candidates to the front of the queue, the others to the back
        const unsigned back = __ballot_sync(0xffffffffu, cand && !scr);
        queue_push(cand && scr, item, b.queue, b.counters);
        if (back) {
            const int leader = __ffs(back) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&b.counters[4], __popc(back));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (cand && !scr)
                b.queue[b.qcap - 1 - (base + __popc(back & ((1u << lane) - 1u)))] = item;
        }
    }
}

// After k_ecl_pre_b: the candidate count covers both ends of the queue;
// counters[5] keeps the front's.
__global__ void k_ecl_join_b(BatchDev b) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        b.counters[5] = b.counters[0];
        b.counters[0] += b.counters[4];
    }
}

// Candidate k of the batch queue (front, then back in push order).
__device__ __forceinline__ int32_t queue_at(const BatchDev &b, int k) {
    const int front = b.counters[5];
    return k < front ? b.queue[k] : b.queue[b.qcap - 1 - (k - front)];
}

// k_ecl_roche over the batch queue: each candidate finds its slot by its
// face index.
// Warp mode of the batched eclipse (few candidates): one warp per candidate.
// With more candidates than warp_max, k_ecl_potmin_b and k_ecl_bisect_b do
// the work and this kernel returns at once (the choice is made on the device).
// Warp mode for this call: at most warp_max candidates and, when the mode is
// chosen automatically, none that the FP32 screen serves (the front of the
// queue): thread mode with the screen has the shorter latency even for few.
__device__ __forceinline__ bool batch_warp_mode(const BatchDev &b, int32_t warp_max,
                                                int32_t auto_mode) {
    return b.counters[0] <= warp_max && !(auto_mode && b.counters[5] > 0);
}

__global__ void __launch_bounds__(128, 4) k_ecl_roche_b(BatchDev b, int32_t warp_max,
                                                     int32_t auto_mode) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = b.counters[0];
    const GridDev g = b.g;
    if (batch_warp_mode(b, warp_max, auto_mode)) {
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&b.counters[1], 1);
            k = __shfl_sync(full, k, 0);
            if (k >= total) break;
            const int32_t i = queue_at(b, k);
            const SlotDev &S = b.slots[find_seg(b.face0, b.nslots, i)];
            const EclParams &p = S.ep;
            const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
            double ing = 0., egr = 0.;
            int s = 0;
            const bool ecl = ingress_egress_warp(p.comp_star, p.q, p.comp_spin, p.cosi, p.sini,
                                                 p.delta, pos, p.comp_rref, p.comp_pref, ing,
                                                 egr, s);
            if (lane == 0) {
                if (s) {
                    set_status(b.st + S.model, s, i - S.face0);
                } else if (ecl) {
                    g.necl[i] = 1;
                    g.ein[i] = ing;
                    g.eout[i] = egr;
                }
            }
        }
        return;
    }
}

// Thread mode of the batched eclipse, in two passes whose code is small enough
// to stay in the instruction cache (the fused solve stalled on instruction
// fetch): the sphere test and pot_min per candidate, then the ingress and
// egress bisections (ingress_egress.cpp:61-86) on the two lanes of a pair.
// Warps take consecutive candidates (similar iteration counts run together).
// Same arithmetic and decisions as ingress_egress: identical results.
__global__ void __launch_bounds__(128, 4) k_ecl_potmin_b(BatchDev b, int32_t warp_max,
                                                      int32_t auto_mode) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = b.counters[0];
    if (batch_warp_mode(b, warp_max, auto_mode)) return;
    const GridDev g = b.g;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&b.counters[2], 32);
        base = __shfl_sync(full, base, 0);
        if (base >= total) break;
        const int k = base + lane;
        bool hit = false;
        if (k < total) {
            const int32_t i = queue_at(b, k);
            const SlotDev &S = b.slots[find_seg(b.face0, b.nslots, i)];
            const EclParams &p = S.ep;
            const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
            const V3 cofm = p.comp_star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
            double phi1, phi2, lam1, lam2, phi = 0., lam = 0.;
            if (sphere_eclipse_ph(p.cosi, p.sini, pos, cofm, p.comp_rref, phi1, phi2, lam1,
                                  lam2)) {
                const double ACC = 2. * sqrt(2. * kTwoPi * (lam2 - lam1) * p.delta);
                int s = 0;
                hit = pot_min(p.comp_star, p.q, p.comp_spin, p.cosi, p.sini, pos, phi1, phi2,
                              lam1, lam2, p.comp_rref, p.comp_pref, ACC, phi, lam, s);
                if (s) {
                    set_status(b.st + S.model, s, i - S.face0);
                    hit = false;
                }
                b.es[k] = make_double4(phi, phi1, phi2, ACC);
            }
        }
        push_hits(hit, k, b.hits, &b.counters[6]);
    }
}

// 6 blocks of 4 warps per SM (a sweep of 4, 5, 6 and 8 on B200 chose 6: more
// warps hide the FP64 latency, fewer registers spill more)
template <int NB>
__global__ void __launch_bounds__(128, NB)
    k_ecl_bisect_b(__grid_constant__ const BatchDev b, int32_t warp_max, int32_t auto_mode) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = b.counters[0];
    if (batch_warp_mode(b, warp_max, auto_mode)) return;
    const int64_t n2 = 2 * (int64_t)b.counters[6];
    for (;;) {
        int64_t base = 0;
        if (lane == 0) base = atomicAdd(&b.counters[3], 32);
        base = __shfl_sync(full, base, 0);
        if (base >= n2) break;
        const int64_t u = base + lane;
        const int side = (int)(u & 1);
        const bool live = u < n2;
        const int k = live ? b.hits[u >> 1] : 0;
        const int32_t i = live ? queue_at(b, k) : 0;
        const int sl = find_seg(b.face0, b.nslots, i);
        const double4 E = live ? b.es[k] : make_double4(0., 0., 0., 0.);
        const V3 pos = live ? v3(b.g.px[i], b.g.py[i], b.g.pz[i]) : v3(0., 0., 0.);
        int s = 0;
        double v = ecl_bisect_warp(b.slots[sl].ep, live, E.x, side ? E.z : E.y, E.w, pos, s);
        v = v - floor(v);
        const double other = __shfl_xor_sync(full, v, 1);
        const int os = __shfl_xor_sync(full, s, 1);
        if (live && side == 0) {
            const SlotDev &S = b.slots[sl];
            if (s || os) {
                set_status(b.st + S.model, s ? s : os, i - S.face0);
            } else {
                double egr = other;
                if (egr < v) egr++;
                b.g.necl[i] = 1;
                b.g.ein[i] = v;
                b.g.eout[i] = egr;
            }
        }
    }
}

__global__ void k_continuum_b(BatchDev b) {
    const int nk = b.counts[1];
    if (nk <= 0) return;
    const int64_t total = b.cont_face[nk];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < total; u += stride) {
        const int k = find_seg(b.cont_face, nk, u);
        const SlotDev &S = b.slots[b.cont_slot[k]];
        continuum_face(S.cp, slot_grid(b.g, S.face0, S.nface, S.ntiled), u - b.cont_face[k]);
    }
}

// Partition counts per 1024-face block of the continuum list's slots; a
// CTA takes whole blocks.
__global__ void __launch_bounds__(kFlatBlock) k_flat_count_b(BatchDev b) {
    const int nk = b.counts[1];
    if (nk <= 0) return;
    const int64_t total = b.cont_blk[nk];
    for (int64_t B = blockIdx.x; B < total; B += gridDim.x) {
        const int k = find_seg(b.cont_blk, nk, B);
        const SlotDev &S = b.slots[b.cont_slot[k]];
        const int64_t lb = B - b.cont_blk[k];
        const int64_t i = lb * kFlatBlock + threadIdx.x;
        const int flag = (i < S.nface) && b.g.necl[S.face0 + i] == 1;
        const int c = __syncthreads_count(flag);
        if (threadIdx.x == 0) b.blockcnt[S.blk0 + lb] = c;
    }
}

__global__ void __launch_bounds__(1024) k_flat_scan_b(BatchDev b) {
    const int nk = b.counts[1];
    for (int k = blockIdx.x; k < nk; k += gridDim.x) {
        const int s = b.cont_slot[k];
        const SlotDev &S = b.slots[s];
        const int32_t nb = (int32_t)((S.nface + kFlatBlock - 1) / kFlatBlock);
        scan_blocks(b.blockcnt + S.blk0, nb, S.nface, b.n0 + s);
    }
}

// Stable partition into fast sweep records; the record after an odd last
// face is zeroed (the sweep reads faces in pairs).
__global__ void __launch_bounds__(kFlatBlock) k_flat_scatter_b(BatchDev b) {
    __shared__ int32_t warp_tot[32];
    const int nk = b.counts[1];
    if (nk <= 0) return;
    const int64_t total = b.cont_blk[nk];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int64_t B = blockIdx.x; B < total; B += gridDim.x) {
        const int k = find_seg(b.cont_blk, nk, B);
        const int s = b.cont_slot[k];
        const SlotDev &S = b.slots[s];
        const int64_t lb = B - b.cont_blk[k];
        const int64_t i = lb * kFlatBlock + t, n = S.nface;
        const bool in = i < n;
        const int flag = in && b.g.necl[S.face0 + i] == 1;
        const unsigned m = __ballot_sync(0xffffffffu, flag);
        if (lane == 0) warp_tot[w] = __popc(m);
        __syncthreads();
        int before = 0;
        for (int q = 0; q < w; q++) before += warp_tot[q];
        __syncthreads();
        const int rank = before + __popc(m & ((1u << lane) - 1u));
        float *fp = b.fp + 8 * S.flat0;
        ulonglong2 *ecl = b.ecl + S.flat0;
        if (in) {
            const GridDev g = slot_grid(b.g, S.face0, n, S.ntiled);
            const int64_t n0 = b.n0[s];
            const int64_t boff = b.blockcnt[S.blk0 + lb];
            const int64_t dest = flag ? n0 + boff + rank : lb * kFlatBlock - boff + (t - rank);
            fast_record(fp, dest, g, i, S.fc);
            ecl[dest] = flag ? ecl_fx64(g.ein[i], g.eout[i]) : make_ulonglong2(0ull, 0ull);
        } else if (i == n && (n & 1)) {
            float *r = fp + 16 * (n >> 1) + 1;
            for (int q = 0; q < 16; q += 2) r[q] = 0.f;
            ecl[n] = make_ulonglong2(0ull, 0ull);
        }
    }
}

__global__ void k_phases_b(BatchDev b, const DatumRec *__restrict__ data,
                           const int64_t *__restrict__ off, int32_t n, BatchPhases ph) {
    const int np = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (np >= n || !b.models[m].live) return;
    const PhaseParams &p = b.models[m].pp;
    const DatumRec d = data[np];
    double phase, slfac;
    point_phase(p, d, phase, slfac);
    const double expose = d.expose / p.period;
    const int ndiv = d.ndiv;
    const double norm = (ndiv - 1 > 1) ? ndiv - 1 : 1;
    int64_t e = m * ph.ldp + off[np];
    for (int nd = 0; nd < ndiv; ++nd, ++e) {
        double phi, wgt;
        sub_exposure(phase, expose, ndiv, nd, phi, wgt);
        const V3 earth = set_earth(p.cosi, p.sini, phi);
        const double phin = phi - floor(phi);
        ph.w1[e] = slfac * wgt * gi_scale1(p.gi, phi) / norm;
        ph.w2[e] = slfac * wgt * gi_scale2(p.gi, phi) / norm;
        ph.ef[e] = make_float4((float)earth.x, (float)earth.y, (float)earth.z, 0.f);
        ph.pfx[e] = phase_fx64(phin);
    }
}

// Chunk partials of each slot summed in chunk order, per phase entry.
__global__ void k_reduce_b(BatchDev b, const double *__restrict__ part, int64_t ldp, int64_t nent,
                           double *osum) {
    const int s = blockIdx.y;
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nent || !b.slots[s].live) return;
    const int64_t c0 = b.chunk_pre[s], c1 = b.chunk_pre[s + 1];
    double o = 0.0;
    int64_t c = c0;
    for (; c + 8 <= c1; c += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = part[(c + u) * ldp + e];
#pragma unroll
        for (int u = 0; u < 8; u++) o += v[u];
    }
    for (; c < c1; c++) o += part[c * ldp + e];
    osum[s * ldp + e] = o;
}

// Per model and point: star 1 then star 2 sub-exposure sums, third light.
__global__ void k_scatter_b(BatchDev b, BatchPhases ph, const double *__restrict__ osum,
                            const DatumRec *__restrict__ data, const int64_t *__restrict__ off,
                            int32_t n, double *calc) {
    const int np = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (np >= n || !b.models[m].live) return;
    const int64_t row = m * ph.ldp;
    const double *o1 = osum + (2 * (int64_t)m) * ph.ldp, *o2 = o1 + ph.ldp;
    const int64_t e0 = off[np], e1 = e0 + (data[np].ndiv > 0 ? data[np].ndiv : 0);
    double c = 0.;
    for (int64_t e = e0; e < e1; e++) c += ph.w1[row + e] * o1[e];
    for (int64_t e = e0; e < e1; e++) c += ph.w2[row + e] * o2[e];
    calc[m * (int64_t)n + np] = c + b.models[m].third;
}

__global__ void __launch_bounds__(1024) k_finalize_b(BatchDev b, int32_t flags,
                                                     const DatumRec *__restrict__ data,
                                                     int32_t n, double *calc, double *sfac,
                                                     double *out) {
    __shared__ double sh[1024];
    const int m = blockIdx.x;
    if (!b.models[m].live) return;  // keeps the previous call's results
    double *sf = sfac + 5 * (int64_t)m;
    if (threadIdx.x == 0) sf[0] = b.models[m].sfac0;
    __syncthreads();
    finalize_block(flags, data, n, calc + m * (int64_t)n, sf, out + 3 * (int64_t)m, sh);
}

inline unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_pack_flat(FlatDev f, int64_t n0, int need_pos, cudaStream_t s) {
    k_pack_flat<<<nblocks(f.n > 0 ? f.n : 1, 256), 256, 0, s>>>(f, n0, need_pos);
    count_launch();
}

void launch_pack_phases(PhaseDev ph, cudaStream_t s) {
    if (ph.nent <= 0) return;
    k_pack_phases<<<nblocks(ph.nent, 256), 256, 0, s>>>(ph);
    count_launch();
}

void launch_grid(const GridParams &p, const RingRec *rings, GridDev g, DevStatus *st,
                 cudaStream_t s) {
    if (p.nhalf <= 0) return;
    k_grid<<<nblocks(p.nhalf, 128), 128, 0, s>>>(p, rings, g, st);
    count_launch();
}

// Resident blocks of 128 threads per SM for the bisection kernels: 4 (no
// register spills, 128 registers a thread) or 6 (80 registers, a few
// spills, more warps to hide FP64 latency); LCG_ECL_BISECT_BLOCKS=6 selects
// the second, for measurement.
int bisect_blocks_per_sm() {
    static const int nb = [] {
        const char *v = getenv("LCG_ECL_BISECT_BLOCKS");
        return (v && atoi(v) == 6) ? 6 : 4;
    }();
    return nb;
}

void launch_eclipse(const EclParams &p, int32_t eclipse_on, GridDev g, int32_t *queue,
                    int32_t *counters, double4 *es, int32_t *hits, DevStatus *st, int nsm,
                    int32_t warp_mode, cudaStream_t s) {
    if (g.n <= 0) return;
    cudaMemsetAsync(counters, 0, 8 * sizeof(int32_t), s);
    k_ecl_pre<<<nblocks(g.n, 256), 256, 0, s>>>(p, eclipse_on, g, queue, counters);
    count_launch();
    if (eclipse_on && p.comp_roche) {
        // 4 blocks of 4 warps per SM; no more warps than faces
        unsigned nb = (unsigned)nsm * 4u;
        const unsigned need = nblocks(g.n, 4);
        if (need < nb) nb = need;
        const int32_t warps = (int32_t)nb * 4;
        // auto: warp mode for few candidates, unless the FP32 screen serves them
        // (thread mode with the screen has the shorter latency even then)
        const int32_t warp_max =
            warp_mode < 0 ? -1 : warp_mode > 0 ? warp_mode : (p.scr.on ? -1 : 2 * warps);
        k_ecl_roche<<<nb, 128, 0, s>>>(p, g, queue, counters, st, warp_max);
        count_launch();
        k_ecl_potmin<<<nb, 128, 0, s>>>(p, g, queue, counters, es, hits, st, warp_max);
        count_launch();
        const int nbs = bisect_blocks_per_sm();
        const unsigned cap = (unsigned)nsm * (unsigned)nbs;
        const unsigned nbb = need < cap ? need : cap;
        if (nbs == 6)
            k_ecl_bisect<6><<<nbb, 128, 0, s>>>(p, g, queue, counters, es, hits, st, warp_max);
        else
            k_ecl_bisect<4><<<nbb, 128, 0, s>>>(p, g, queue, counters, es, hits, st, warp_max);
        count_launch();
    }
}

void launch_continuum(const ContParams &p, GridDev g, cudaStream_t s) {
    if (g.n <= 0) return;
    k_continuum<<<nblocks(g.n, 256), 256, 0, s>>>(p, g);
    count_launch();
}

void launch_flatten(GridDev g, FlatDev f, int32_t *blockcnt, int mixed, int need_pos,
                    const FastCoef &fc, DevStatus *st, cudaStream_t s) {
    (void)st;
    const unsigned nb = nblocks(g.n, kFlatBlock);
    if (nb == 0) {
        cudaMemsetAsync(f.n0, 0, 2 * sizeof(int64_t), s);
        return;
    }
    if (mixed && fc.on && f.npad > g.n) {
        // padding faces must add nothing: zero from the pair holding face n
        // (records interleave the two faces of a pair; the scatter below
        // rewrites face n-1's half when n is odd)
        const int64_t z0 = 16 * (g.n >> 1);
        cudaMemsetAsync(f.fp + z0, 0, (size_t)(8 * f.npad - z0) * sizeof(float), s);
    }
    k_flat_count<<<nb, kFlatBlock, 0, s>>>(g, blockcnt);
    count_launch();
    k_flat_scan<<<1, 1024, 0, s>>>(blockcnt, (int32_t)nb, g.n, f.n0);
    count_launch();
    k_flat_scatter<<<nb, kFlatBlock, 0, s>>>(g, f, blockcnt, mixed, need_pos, fc);
    count_launch();
    if (mixed && fc.on) launch_run_bounds(f.fp, f.ecl, f.npad / 2, f.runb, f.runh, s);
}

void launch_phases(const PhaseParams &p, const DatumRec *data, const int64_t *off, int32_t n,
                   PhaseDev ph, cudaStream_t s) {
    if (n <= 0) return;
    k_phases<<<nblocks(n, 128), 128, 0, s>>>(p, data, off, n, ph);
    count_launch();
}

void launch_scatter(const ScatterParams &p, const ReduceParams &r, const PhaseDev &ph,
                    const DatumRec *data, const int64_t *off, int32_t n, double *calc,
                    cudaStream_t s) {
    if (n <= 0) return;
    int64_t nmax = 0;
    for (int k = 0; k < 4; k++)
        if (r.part[k] && r.nent[k] > nmax) nmax = r.nent[k];
    if (nmax > 0) {
        k_reduce_chunks<<<dim3(nblocks(nmax, 256), 4), 256, 0, s>>>(r);
        count_launch();
    }
    k_scatter<<<nblocks(n, 128), 128, 0, s>>>(p, r.osum[0], r.osum[1], r.osum[2], r.osum[3], ph,
                                              data, off, n, calc);
    count_launch();
}

void launch_finalize(int32_t flags, const DatumRec *data, int32_t n, double *calc,
                     double *sfac_io, double *out, cudaStream_t s) {
    k_finalize<<<1, 1024, 0, s>>>(flags, data, n, calc, sfac_io, out);
    count_launch();
}

void launch_interp(const DatumRec *data, int32_t n, const int64_t *idx, int32_t m,
                   const double *mc, double *calc, int32_t rdata, double *out, cudaStream_t s) {
    if (n <= 0 || m <= 0) return;
    k_interp<<<1, 1024, 0, s>>>(data, n, idx, m, mc, calc, rdata, out);
    count_launch();
}

void launch_run_bounds(const float *fp, const ulonglong2 *ecl, int64_t npairs, float4 *runb,
                       ulonglong2 *runh, cudaStream_t s) {
    const int64_t nruns = (npairs + 31) / 32;
    if (nruns <= 0) return;
    k_run_bounds<<<nblocks(nruns * 32, 256), 256, 0, s>>>(fp, ecl, npairs, runb, runh);
    count_launch();
}

void launch_batch_run_bounds(const BatchDev &b, int nsm, cudaStream_t s) {
    k_run_bounds_b<<<nsm * 4, 256, 0, s>>>(b);
    count_launch();
}

void launch_gather_rows(const double *src, int32_t n, const int32_t *rows, int32_t count,
                        double *dst, cudaStream_t s) {
    if (n <= 0 || count <= 0) return;
    k_gather_rows<<<dim3(nblocks(n, 256), (unsigned)count), 256, 0, s>>>(src, n, rows, dst);
    count_launch();
}

void launch_diagnostics(int star, GridDev g, double *out, cudaStream_t s) {
    const int64_t nblk = (g.n + 8191) / 8192;
    if (nblk <= 0) return;
    k_diag<<<nblocks(nblk, 64), 64, 0, s>>>(star, g, out);
    count_launch();
}

// ---- batched launchers -------------------------------------------------------

void launch_batch_grid(const BatchDev &b, int nsm, cudaStream_t s) {
    // one wave of the blocks that fit (its registers allow 5 of 128 threads per
    // SM): a grid-stride loop over more blocks than fit runs a second, partial
    // wave after the first
    static const int per_sm = [] {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_grid_b, 128, 0) != cudaSuccess ||
            nb < 1)
            nb = 4;
        return nb;
    }();
    k_grid_b<<<nsm * per_sm, 128, 0, s>>>(b);
    count_launch();
}

void launch_batch_eclipse(const BatchDev &b, int nsm, int32_t warp_mode, cudaStream_t s) {
    cudaMemsetAsync(b.counters, 0, 8 * sizeof(int32_t), s);
    k_ecl_pre_b<<<nsm * 4, 256, 0, s>>>(b);
    count_launch();
    k_ecl_join_b<<<1, 32, 0, s>>>(b);
    count_launch();
    const int32_t warps = nsm * 16;
    const int32_t warp_max = warp_mode < 0 ? -1 : warp_mode > 0 ? warp_mode : 2 * warps;
    const int32_t auto_mode = warp_mode == 0;
    k_ecl_roche_b<<<nsm * 4, 128, 0, s>>>(b, warp_max, auto_mode);
    count_launch();
    k_ecl_potmin_b<<<nsm * 4, 128, 0, s>>>(b, warp_max, auto_mode);
    count_launch();
    if (bisect_blocks_per_sm() == 6)
        k_ecl_bisect_b<6><<<nsm * 6, 128, 0, s>>>(b, warp_max, auto_mode);
    else
        k_ecl_bisect_b<4><<<nsm * 4, 128, 0, s>>>(b, warp_max, auto_mode);
    count_launch();
}

void launch_batch_continuum(const BatchDev &b, int nsm, cudaStream_t s) {
    k_continuum_b<<<nsm * 4, 256, 0, s>>>(b);
    count_launch();
}

void launch_batch_flatten(const BatchDev &b, int nsm, cudaStream_t s) {
    k_flat_count_b<<<nsm * 2, kFlatBlock, 0, s>>>(b);
    count_launch();
    k_flat_scan_b<<<nsm, 1024, 0, s>>>(b);
    count_launch();
    k_flat_scatter_b<<<nsm * 2, kFlatBlock, 0, s>>>(b);
    count_launch();
    launch_batch_run_bounds(b, nsm, s);
}

void launch_batch_phases(const BatchDev &b, const DatumRec *data, const int64_t *off, int32_t n,
                         const BatchPhases &ph, cudaStream_t s) {
    if (n <= 0 || b.nmodels <= 0) return;
    k_phases_b<<<dim3(nblocks(n, 128), (unsigned)b.nmodels), 128, 0, s>>>(b, data, off, n, ph);
    count_launch();
}

void launch_batch_reduce(const BatchDev &b, const BatchPhases &ph, const double *part,
                         int64_t ldp, double *osum, const DatumRec *data, const int64_t *off,
                         int32_t n, int32_t flags, double *calc, double *sfac, double *out,
                         cudaStream_t s) {
    if (n <= 0 || b.nmodels <= 0) return;
    if (ph.nent > 0) {
        k_reduce_b<<<dim3(nblocks(ph.nent, 256), (unsigned)b.nslots), 256, 0, s>>>(
            b, part, ldp, ph.nent, osum);
        count_launch();
    }
    k_scatter_b<<<dim3(nblocks(n, 128), (unsigned)b.nmodels), 128, 0, s>>>(b, ph, osum, data,
                                                                             off, n, calc);
    count_launch();
    k_finalize_b<<<b.nmodels, 1024, 0, s>>>(b, flags, data, n, calc, sfac, out);
    count_launch();
}

}  // namespace lcg
