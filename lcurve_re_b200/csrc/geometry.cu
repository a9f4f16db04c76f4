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
#include "eclipse.cuh"
#include "engine.h"

namespace lcg {

namespace {

__device__ __forceinline__ void set_status(DevStatus *st, int code, int64_t face) {
    if (atomicCAS(&st->code, 0, code) == 0) st->face = (int32_t)face;
}

__global__ void k_grid(GridParams p, const RingRec *__restrict__ rings, GridDev g,
                       DevStatus *st) {
    const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (h >= p.nhalf) return;
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
    int64_t i = R.off + np;
    g.px[i] = posn.x; g.py[i] = posn.y; g.pz[i] = posn.z;
    g.nx[i] = dvec.x; g.ny[i] = dvec.y; g.nz[i] = dvec.z;
    g.area[i] = af;
    g.grav[i] = gf;
    const int np2 = R.nphi - 1 - np;
    if (np2 != np) {
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

// Sphere test of every face; Roche eclipsers queue their candidates.
__global__ void k_ecl_pre(EclParams p, int32_t eclipse_on, GridDev g, int32_t *queue,
                          int32_t *counters) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool in = i < g.n;
    bool cand = false;
    if (in) {
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
    const unsigned mask = __ballot_sync(0xffffffffu, cand);
    if (mask) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(mask) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&counters[0], __popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (cand) queue[base + __popc(mask & ((1u << lane) - 1u))] = (int32_t)i;
    }
}

// Each warp takes 32 consecutive candidates at a time, so neighbouring faces
// (similar iteration counts) run in lockstep.
__global__ void __launch_bounds__(128) k_ecl_roche(EclParams p, GridDev g,
                                                   const int32_t *__restrict__ queue,
                                                   int32_t *counters, DevStatus *st) {
    const int lane = threadIdx.x & 31;
    const int total = counters[0];
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&counters[1], 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const int k = base + lane;
        if (k < total) {
            const int32_t i = queue[k];
            const V3 pos = v3(g.px[i], g.py[i], g.pz[i]);
            double ing = 0., egr = 0.;
            int s = 0;
            bool ecl = ingress_egress(p.comp_star, p.q, p.comp_spin, p.cosi, p.sini, p.delta, pos,
                                      p.comp_rref, p.comp_pref, ing, egr, s);
            if (s) {
                set_status(st, s, i);
            } else if (ecl) {
                g.necl[i] = 1;
                g.ein[i] = ing;
                g.eout[i] = egr;
            }
        }
    }
}

__global__ void k_continuum(ContParams p, GridDev g) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= g.n) return;
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

constexpr int kFlatBlock = 1024;

__global__ void k_flat_count(GridDev g, int32_t *blockcnt) {
    const int64_t i = blockIdx.x * (int64_t)kFlatBlock + threadIdx.x;
    const int flag = (i < g.n) && g.necl[i] == 1;
    const int c = __syncthreads_count(flag);
    if (threadIdx.x == 0) blockcnt[blockIdx.x] = c;
}

// Single block: exclusive scan of the per-block eclipse counts; n0 = faces
// never eclipsed.
__global__ void k_flat_scan(int32_t *blockcnt, int32_t nb, int64_t n, int64_t *n0) {
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
}

__device__ __forceinline__ uint32_t phase_fx(double ph) {
    return (uint32_t)((unsigned long long)llrint(ph * 4294967296.0) & 0xffffffffull);
}

__global__ void k_flat_scatter(GridDev g, FlatDev f, const int32_t *__restrict__ blockoff,
                               int mixed, int need_pos, FastCoef fc) {
    __shared__ int32_t warp_tot[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t i = blockIdx.x * (int64_t)kFlatBlock + t;
    const bool in = i < g.n;
    const int flag = in && g.necl[i] == 1;
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) warp_tot[w] = __popc(m);
    __syncthreads();
    int before = 0;
    for (int k = 0; k < w; k++) before += warp_tot[k];
    const int rank = before + __popc(m & ((1u << lane) - 1u));
    if (!in) return;
    const int64_t n0 = *f.n0;
    const int64_t boff = blockoff[blockIdx.x];
    const int64_t dest = flag ? n0 + boff + rank
                              : blockIdx.x * (int64_t)kFlatBlock - boff + (t - rank);
    if (mixed) {
        if (fc.on) {
            const double fl = (double)g.flux[i];
            float *r = f.fp + 16 * (dest >> 1) + (dest & 1);
            r[0] = (float)g.nx[i];
            r[2] = (float)g.ny[i];
            r[4] = (float)(fc.cosi * g.nz[i]);
            r[6] = (float)(fl * fc.p[0]);
            r[8] = (float)(fl * fc.p[1]);
            r[10] = (float)(fl * fc.p[2]);
            r[12] = (float)(fl * fc.p[3]);
            r[14] = (float)(fl * fc.p[4]);
        } else {
            f.geo[dest] = make_float4((float)g.nx[i], (float)g.ny[i], (float)g.nz[i], g.flux[i]);
        }
        uint2 e = make_uint2(0u, 0u);
        if (flag) {
            const double in1 = g.ein[i], out1 = g.eout[i];
            long long w64 = llrint((out1 - in1) * 4294967296.0);
            if (w64 < 0) w64 = 0;
            if (w64 > 4294967294ll) w64 = 4294967294ll;
            e = make_uint2(phase_fx(in1), (uint32_t)(w64 + 1));
        }
        f.ecl[dest] = e;
        if (need_pos) f.pos[dest] = make_float4((float)g.px[i], (float)g.py[i], (float)g.pz[i], 0.f);
    } else {
        f.dx[dest] = g.nx[i]; f.dy[dest] = g.ny[i]; f.dz[dest] = g.nz[i];
        f.px[dest] = g.px[i]; f.py[dest] = g.py[i]; f.pz[dest] = g.pz[i];
        f.flux[dest] = (double)g.flux[i];
        f.in1[dest] = flag ? g.ein[i] : 0.;
        f.out1[dest] = flag ? g.eout[i] : 0.;
    }
}

__global__ void k_phases(PhaseParams p, const DatumRec *__restrict__ data,
                         const int64_t *__restrict__ off, int32_t n, PhaseDev ph) {
    const int np = blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= n) return;
    const DatumRec d = data[np];
    double phase = (d.time - p.t0) / p.period;
    for (int it = 0; it < 4; it++)
        phase -= (p.t0 + phase * (p.period + p.pdot * phase) - d.time) /
                 (p.period + 2. * p.pdot * phase);
    phase += p.deltat / p.period / 2. * (cos(2. * kPi * phase) - 1.);
    const double frac = (d.time - p.middle) / p.range;
    const double slfac = 1. + frac * (p.slope + frac * (p.quad + frac * p.cube));
    const double expose = d.expose / p.period;
    const int ndiv = d.ndiv;
    const double norm = (ndiv - 1 > 1) ? ndiv - 1 : 1;
    int64_t e = off[np];
    for (int nd = 0; nd < ndiv; ++nd, ++e) {
        double phi, wgt;
        if (ndiv == 1) {
            phi = phase;
            wgt = 1.0;
        } else {
            phi = phase + expose * (nd - (ndiv - 1) / 2.0) / (ndiv - 1);
            wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
        }
        const V3 earth = set_earth(p.cosi, p.sini, phi);
        const double phin = phi - floor(phi);
        ph.ex[e] = earth.x;
        ph.ey[e] = earth.y;
        ph.ez[e] = earth.z;
        ph.phin[e] = phin;
        ph.w1[e] = slfac * wgt * gi_scale1(p.gi, phi) / norm;
        ph.w2[e] = slfac * wgt * gi_scale2(p.gi, phi) / norm;
        ph.type[e] = (uint8_t)gi_type(p.gi, phi);
        ph.ef[e] = make_float4((float)earth.x, (float)earth.y, (float)earth.z,
                               __uint_as_float(phase_fx(phin)));
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
    for (int64_t e = e0; e < e1; e++)
        if (p.copy2 || ph.type[e] == 3) c += ph.w2[e] * o2f[e];
    if (!p.copy2)
        for (int64_t e = e0; e < e1; e++)
            if (ph.type[e] != 3) c += ph.w2[e] * o2c[e];
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
__global__ void __launch_bounds__(1024) k_finalize(int32_t flags, const DatumRec *__restrict__ data,
                                                   int32_t n, double *calc, double *sfac_io,
                                                   double *out) {
    __shared__ double sh[1024];
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
    uint2 e = make_uint2(0u, 0u);
    if (i >= n0) {
        long long w64 = llrint((f.out1[i] - f.in1[i]) * 4294967296.0);
        if (w64 < 0) w64 = 0;
        if (w64 > 4294967294ll) w64 = 4294967294ll;
        e = make_uint2(phase_fx(f.in1[i]), (uint32_t)(w64 + 1));
    }
    f.ecl[i] = e;
    if (need_pos) f.pos[i] = make_float4((float)f.px[i], (float)f.py[i], (float)f.pz[i], 0.f);
}

__global__ void k_pack_phases(PhaseDev ph) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ph.nent) return;
    ph.ef[e] = make_float4((float)ph.ex[e], (float)ph.ey[e], (float)ph.ez[e],
                           __uint_as_float(phase_fx(ph.phin[e])));
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

void launch_eclipse(const EclParams &p, int32_t eclipse_on, GridDev g, int32_t *queue,
                    int32_t *counters, DevStatus *st, int nsm, cudaStream_t s) {
    if (g.n <= 0) return;
    cudaMemsetAsync(counters, 0, 2 * sizeof(int32_t), s);
    k_ecl_pre<<<nblocks(g.n, 256), 256, 0, s>>>(p, eclipse_on, g, queue, counters);
    count_launch();
    if (eclipse_on && p.comp_roche) {
        unsigned nb = (unsigned)nsm * 4u;
        const unsigned need = nblocks(g.n, 128);
        if (need < nb) nb = need;
        k_ecl_roche<<<nb, 128, 0, s>>>(p, g, queue, counters, st);
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
        cudaMemsetAsync(f.n0, 0, sizeof(int64_t), s);
        return;
    }
    if (mixed && fc.on && f.npad > g.n)  // padding faces must add nothing
        cudaMemsetAsync(f.fp + 8 * g.n, 0, (size_t)(f.npad - g.n) * 8 * sizeof(float), s);
    k_flat_count<<<nb, kFlatBlock, 0, s>>>(g, blockcnt);
    count_launch();
    k_flat_scan<<<1, 1024, 0, s>>>(blockcnt, (int32_t)nb, g.n, f.n0);
    count_launch();
    k_flat_scatter<<<nb, kFlatBlock, 0, s>>>(g, f, blockcnt, mixed, need_pos, fc);
    count_launch();
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

void launch_diagnostics(int star, GridDev g, double *out, cudaStream_t s) {
    const int64_t nblk = (g.n + 8191) / 8192;
    if (nblk <= 0) return;
    k_diag<<<nblocks(nblk, 64), 64, 0, s>>>(star, g, out);
    count_launch();
}

}  // namespace lcg
