// components.cu — accretion disc, disc rim and bright spot; iscale fits.
//
// Element kernels restate set_disc_grid (set_disc_grid.cpp:27-127), the
// outer rim of set_disc_edge (:144-264), set_bright_spot_grid
// (set_bright_spot_grid.cpp:27-100), their continua (set_disc_continuum.cpp)
// and star_eclipse (star_eclipse.cpp:15-26) with one thread per element: the
// per-ring and per-model scalars come from the host, the trigonometry, the
// continuum and the eclipse solves run on the device. Element sums per phase
// entry follow comp_disc / comp_edge / comp_spot (comp_light.cpp:323-408) with
// the elements in vector order, summed in chunks of 256 whose partial sums
// are added in order (the reference's single serial sum, regrouped: equal to
// rounding). Compiled with --fmad=false.
#include "context.h"
#include "eclipse.cuh"

namespace lcg {

namespace {

constexpr int kThreadsC = 128;

__device__ __forceinline__ void report(DevStatus *st, int code, int idx) {
    if (atomicCAS(&st->code, 0, code) == 0) st->face = idx;
}

// Component elements report -(1 + element index) so that the host can tell
// them from star faces.
__device__ __forceinline__ int elem_tag(int i) { return -1 - i; }

// The eclipses of one element: the opaque disc's (disc and rim only; the
// spot gets none, set_bright_spot_grid.cpp:80-81), then star 1's, then star
// 2's (set_disc_grid.cpp:99-113). trap1: a Roche_Error from star 1 becomes
// the range (0, 1), as for the rim's upper elements (set_disc_grid.cpp:222-231).
// One thread solves all of an element's eclipses: nearly every disc element is
// a Roche candidate of the donor, and a warp per candidate (as for star grids
// with few candidates) measured slower here.
__device__ void elem_eclipses(const CompParams &p, V3 posn, bool opaque, bool trap1, ElemRec &r,
                              DevStatus *st, int idx) {
    r.nr = 0;  // an element whose eclipse failed is left with none
    for (int k = 0; k < kMaxRanges; k++) r.r[k] = make_double2(0., 0.);
    int nr = 0;
    double rin[kMaxRanges], rout[kMaxRanges];
    int s = 0;
    if (opaque) {
        disc_eclipse(p.dg, posn, nr, rin, rout, kMaxRanges, s);
        if (s) { report(st, s, idx); return; }
    }
    for (int star = 0; star < 2; star++) {
        if (!(star == 0 ? p.eclipse1 : p.eclipse2)) continue;
        double in = 0., out = 0.;
        bool ecl;
        int es = 0;
        if (star == 0 ? p.roche1 : p.roche2) {
            ecl = ingress_egress(star == 0 ? kStar1 : kStar2, p.q, star == 0 ? p.spin1 : p.spin2,
                                 p.cosi, p.sini, p.delta, posn, star == 0 ? p.rref1 : p.rref2,
                                 star == 0 ? p.pref1 : p.pref2, in, out, es);
        } else {
            double l1, l2;
            ecl = sphere_eclipse_ph(p.cosi, p.sini, posn,
                                    star == 0 ? v3(0., 0., 0.) : v3(1., 0., 0.),
                                    star == 0 ? p.r1 : p.r2, in, out, l1, l2);
        }
        if (es) {
            if (!(star == 0 && trap1 && es == kEclRoche)) { report(st, es, idx); return; }
            ecl = true;
            in = 0.;
            out = 1.;
        }
        if (ecl) {
            if (nr < kMaxRanges) { rin[nr] = in; rout[nr] = out; }
            nr++;
        }
    }
    r.nr = nr < kMaxRanges ? nr : kMaxRanges;
    for (int k = 0; k < kMaxRanges; k++)
        r.r[k] = k < r.nr ? make_double2(rin[k], rout[k]) : make_double2(0., 0.);
}

__global__ void __launch_bounds__(kThreadsC) k_components(CompParams p, ElemRec *el, double4 *pos,
                                                          DevStatus *st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = p.nd + p.ne + p.ns;
    if (i >= n) return;
    constexpr double EFAC = 1.0000001;
    V3 posn, dirn;
    double area, flux;
    bool trap1 = false;
    if (i < p.nd) {
        // disc: ring k holds elements [off, off + ntheta)
        int lo = 0, hi = p.nrad - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.rings[mid].off <= i) lo = mid;
            else hi = mid - 1;
        }
        const DiscRing R = p.rings[lo];
        const int j = i - R.off;
        const double theta = kTwoPi * j / R.ntheta;
        const double sint = sin(theta), cost = cos(theta);
        posn = v3(R.rad * cost, R.rad * sint, R.h);
        dirn = v3(-cost * R.sinp, -sint * R.sinp, R.cosp);
        area = R.area;
        const double r = sqrt(posn.x * posn.x + posn.y * posn.y + posn.z * posn.z);
        flux = p.bright_disc * pow(r / p.rdisc2, p.texp) * (double)(float)area;
    } else if (i < p.nd + p.ne) {
        // outer rim: per longitude, the upper element then NOUT - 1 below it
        const int k = i - p.nd, it = k / p.nout, jj = k % p.nout;
        const double theta = kTwoPi * it / p.ntheta_e;
        const double sint = sin(theta), cost = cos(theta);
        if (jj == 0) {
            posn = v3(EFAC * p.rad_e * cost, EFAC * p.rad_e * sint, EFAC * p.h_e);
            area = p.area_e / 2.;
            trap1 = true;
        } else {
            const int j = jj - 1;
            posn = v3(EFAC * p.rad_e * cost, EFAC * p.rad_e * sint,
                      -p.h_e + 2 * p.h_e * j / (p.nout - 1));
            area = p.area_e;
        }
        dirn = v3(cost, sint, 0);
        // irradiation by the donor as a point source, sunset included
        // (set_disc_continuum.cpp:48-88)
        const V3 vec = v3(1. - posn.x, 0. - posn.y, 0. - posn.z);
        const double r = sqrt(vec.x * vec.x + vec.y * vec.y + vec.z * vec.z);
        const double mu = (dirn.x * vec.x + dirn.y * vec.y + dirn.z * vec.z) / r;
        double temp;
        if (mu >= p.r2) {
            const double geom = sq(p.r2 / r) * mu;
            temp = pow(pow(p.tedge, 4.0) + p.absorb_edge * pow(p.t2, 4.0) * geom, 0.25);
        } else if (mu > -p.r2) {
            const double x0 = -mu / p.r2;
            const double geom = sq(p.r2 / r) * p.r2 *
                                (sqrt(1. - x0 * x0) * (2 + x0 * x0) / 3 - x0 * (kPi / 2 - asin(x0))) /
                                kPi;
            temp = pow(pow(p.tedge, 4.0) + p.absorb_edge * pow(p.t2, 4.0) * geom, 0.25);
        } else {
            temp = p.tedge;
        }
        flux = (double)(float)area * planck(p.wave, temp);
    } else {
        // bright spot: the tilted strip, then the strip parallel to the disc
        const int k = i - p.nd - p.ne, ii = k % p.nspot;
        const bool tilted = k < p.nspot;
        const double dist = p.sfac * ii / (p.nspot - 1);
        const double c = p.length * (dist - p.bmax);
        posn = v3(p.bspot[0] + c * p.bvec[0], p.bspot[1] + c * p.bvec[1], p.bspot[2] + c * p.bvec[2]);
        dirn = tilted ? v3(p.tvec[0], p.tvec[1], p.tvec[2]) : v3(0., 0., 1.);
        area = p.area_s;
        const double bright = p.bright_s * pow(dist / p.bmax, p.expon) *
                              exp(p.expon / p.epow - pow(dist, p.epow));
        flux = bright * (tilted ? (1 - p.cfrac) : p.cfrac) * (double)(float)area;
    }
    ElemRec r;
    r.dx = dirn.x;
    r.dy = dirn.y;
    r.dz = dirn.z;
    r.flux = (float)flux;
    elem_eclipses(p, posn, p.opaque && i < p.nd + p.ne, trap1, r, st, elem_tag(i));
    el[i] = r;
    pos[i] = make_double4(posn.x, posn.y, posn.z, (double)(float)area);
}

__global__ void k_disc_faces(DiscGeom dg, GridDev g, uint8_t *ndx, double2 *xr, DevStatus *st) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    int nr = 0, s = 0;
    double rin[kDiscRanges], rout[kDiscRanges];
    disc_eclipse(dg, v3(g.px[i], g.py[i], g.pz[i]), nr, rin, rout, kDiscRanges, s);
    if (s) report(st, s, (int)i);
    nr = s ? 0 : (nr < kDiscRanges ? nr : kDiscRanges);
    ndx[i] = (uint8_t)nr;
    for (int k = 0; k < kDiscRanges; k++)
        xr[kDiscRanges * i + k] = k < nr ? make_double2(rin[k], rout[k]) : make_double2(0., 0.);
}

// One CTA per (tile of phase entries, chunk of kElemChunk elements): each
// thread sums the chunk's elements in order for its entry (the chunk staged in
// shared memory, every thread reading the same element: a broadcast) and
// writes three partial sums; k_comp_reduce adds the chunks in order.
constexpr int kElemChunk = 256;

__global__ void __launch_bounds__(kThreadsC) k_comp_sums(const ElemRec *__restrict__ el,
                                                         int32_t nd, int32_t ne, int32_t n,
                                                         double lin, double quad, PhaseDev ph,
                                                         double *part, int64_t ldc) {
    __shared__ ElemRec tile[kElemChunk];
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool ok = e < ph.nent;
    const double ex = ok ? ph.ex[e] : 0., ey = ok ? ph.ey[e] : 0., ez = ok ? ph.ez[e] : 0.;
    const double phi = ok ? ph.phin[e] : 0.;
    double s[3] = {0.0, 0.0, 0.0};
    {
        const int base = blockIdx.y * kElemChunk;
        const int m = (n - base < kElemChunk) ? n - base : kElemChunk;
        for (int t = threadIdx.x; t < m; t += blockDim.x) tile[t] = el[base + t];
        __syncthreads();
        for (int t = 0; t < m; t++) {
            const int i = base + t;
            const ElemRec &r = tile[t];
            // Point::visible (lcurve.h:81-89)
            bool vis = true;
            const int nr = r.nr < kMaxRanges ? r.nr : kMaxRanges;
            for (int k = 0; k < nr; k++) {
                const double in = r.r[k].x, o = r.r[k].y;
                if ((phi >= in && phi <= o) || phi <= o - 1.0) { vis = false; break; }
            }
            double v = 0.0;
            if (vis) {
                const double mu = ex * r.dx + ey * r.dy + ez * r.dz;
                if (i >= nd + ne) {
                    v = (mu > 0.0) ? mu * (double)r.flux : 0.0;  // spot_elem
                } else if (mu > 0.0) {                          // disc_elem
                    const double om = 1.0 - mu;
                    v = mu * (double)r.flux * (1.0 - om * (lin + quad * om));
                }
            }
            const int c = i < nd ? 0 : (i < nd + ne ? 1 : 2);
            s[c] += v;
        }
    }
    if (ok) {
        double *row = part + 3 * (int64_t)blockIdx.y * ldc;
        row[e] = s[0];
        row[ldc + e] = s[1];
        row[2 * ldc + e] = s[2];
    }
}

__global__ void k_comp_reduce(const double *__restrict__ part, int nchunk, int64_t nent,
                              double *out, int64_t ldc) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nent) return;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int c = 0; c < nchunk; c++) {
        const double *row = part + 3 * (int64_t)c * ldc;
        s0 += row[e];
        s1 += row[ldc + e];
        s2 += row[2 * ldc + e];
    }
    out[e] = s0;
    out[ldc + e] = s1;
    out[2 * ldc + e] = s2;
}

// ---- iscale -------------------------------------------------------------------
// Weighted least squares for the component scale factors, with svdfit's rule
// (svdfit.cpp:22-80): rows of points with sigma z = ferr / sqrt(weight) > 0,
// scaled by 1/z; singular values below 1e-5 of the largest dropped. Here the
// weighted design matrix [A | b] is first reduced by Householder QR (rows of
// points that do not count are zero and change nothing), then R gets a
// one-sided Jacobi SVD (Hestenes 1958): A and R have the same singular values
// and right vectors, so the truncated solution is svdfit's up to rounding.
// One CTA; deterministic tree reductions.
constexpr int kThreadsF = 512;

__device__ double tree_sum(double v, double *sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int w = kThreadsF / 2; w > 0; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kThreadsF) k_iscale(int32_t flags, int32_t nc,
                                                      const DatumRec *__restrict__ data, int32_t n,
                                                      const double *__restrict__ fcomp,
                                                      double *work, double *calc, double *sfac,
                                                      double *out) {
    __shared__ double sh[kThreadsF];
    __shared__ double R[6][6], x[5];
    const bool scale = flags & 1, rdata = flags & 2;
    const int t = threadIdx.x;
    if (scale) {
        const int m = nc + 1;  // columns: the components, then b
        double *A = work;      // column-major, n rows
        for (int i = t; i < n; i += kThreadsF) {
            const DatumRec d = data[i];
            const double z = d.weight <= 0. ? -1. : d.ferr / sqrt(d.weight);
            const double invsig = z > 0 ? 1. / z : 0.;
            for (int j = 0; j < nc; j++) A[(int64_t)j * n + i] = invsig * fcomp[5 * (int64_t)i + j];
            A[(int64_t)nc * n + i] = invsig * d.flux;
        }
        __syncthreads();
        for (int j = 0; j < nc; j++) {
            double *cj = A + (int64_t)j * n;
            double p = 0.;
            for (int i = j + t; i < n; i += kThreadsF) p += cj[i] * cj[i];
            const double norm2 = tree_sum(p, sh);
            const double ajj = j < n ? cj[j] : 0.;
            if (norm2 > 0. && j < n) {
                const double alpha = ajj > 0. ? -sqrt(norm2) : sqrt(norm2);
                const double v0 = ajj - alpha;
                const double vnorm2 = norm2 - ajj * ajj + v0 * v0;
                for (int c = j + 1; c < m; c++) {
                    double *cc = A + (int64_t)c * n;
                    double q = t == 0 ? v0 * cc[j] : 0.;
                    for (int i = j + 1 + t; i < n; i += kThreadsF) q += cj[i] * cc[i];
                    const double dot = tree_sum(q, sh);
                    const double f = 2. * dot / vnorm2;
                    if (t == 0) cc[j] -= f * v0;
                    for (int i = j + 1 + t; i < n; i += kThreadsF) cc[i] -= f * cj[i];
                    __syncthreads();
                }
                if (t == 0) cj[j] = alpha;
                __syncthreads();
            }
        }
        if (t == 0) {
            // R (upper nc x nc) and c = (Q^T b)[0 .. nc)
            double c[6];
            for (int i = 0; i < nc; i++) {
                for (int j = 0; j < nc; j++) R[i][j] = (j >= i && i < n) ? A[(int64_t)j * n + i] : 0.;
                c[i] = i < n ? A[(int64_t)nc * n + i] : 0.;
            }
            double V[5][5];
            for (int i = 0; i < nc; i++)
                for (int j = 0; j < nc; j++) V[i][j] = i == j ? 1. : 0.;
            for (int sweep = 0; sweep < 60; sweep++) {
                bool rot = false;
                for (int p = 0; p < nc - 1; p++)
                    for (int q = p + 1; q < nc; q++) {
                        double al = 0., be = 0., ga = 0.;
                        for (int i = 0; i < nc; i++) {
                            al += R[i][p] * R[i][p];
                            be += R[i][q] * R[i][q];
                            ga += R[i][p] * R[i][q];
                        }
                        if (ga == 0. || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
                        rot = true;
                        const double zeta = (be - al) / (2. * ga);
                        const double tt = (zeta >= 0. ? 1. : -1.) / (fabs(zeta) + sqrt(1. + zeta * zeta));
                        const double cs = 1. / sqrt(1. + tt * tt), sn = cs * tt;
                        for (int i = 0; i < nc; i++) {
                            const double ap = R[i][p], aq = R[i][q];
                            R[i][p] = cs * ap - sn * aq;
                            R[i][q] = sn * ap + cs * aq;
                            const double vp = V[i][p], vq = V[i][q];
                            V[i][p] = cs * vp - sn * vq;
                            V[i][q] = sn * vp + cs * vq;
                        }
                    }
                if (!rot) break;
            }
            double w[5], wmax = 0.;
            for (int j = 0; j < nc; j++) {
                double s2 = 0.;
                for (int i = 0; i < nc; i++) s2 += R[i][j] * R[i][j];
                w[j] = sqrt(s2);
                wmax = fmax(wmax, w[j]);
            }
            for (int k = 0; k < 5; k++) x[k] = 0.;
            for (int j = 0; j < nc; j++) {
                if (!(w[j] >= 1e-5 * wmax) || w[j] == 0.) continue;
                double ub = 0.;
                for (int i = 0; i < nc; i++) ub += R[i][j] * c[i];
                ub /= w[j] * w[j];
                for (int k = 0; k < nc; k++) x[k] += V[k][j] * ub;
            }
            for (int k = 0; k < 5; k++) sfac[k] = k < nc ? x[k] : 0.;
        }
        __syncthreads();
    }
    // calc from the components (light_curve_comp.cpp:532-556)
    double cs = 0., ws = 0.;
    const double s0 = sfac[0], s1 = sfac[1], s2 = sfac[2], s3 = sfac[3], s4 = sfac[4];
    for (int i = t; i < n; i += kThreadsF) {
        const double *f = fcomp + 5 * (int64_t)i;
        double c = s0 * f[0] + s1 * f[1] + s2 * f[2] + s3 * f[3];
        if (nc == 5) c += s4 * f[4];
        calc[i] = c;
        const DatumRec d = data[i];
        if (d.weight > 0.) {
            ws += d.weight;
            cs += d.weight * sq((d.flux - c) / d.ferr);
        }
    }
    const double chisq = tree_sum(cs, sh), wnok = tree_sum(ws, sh);
    if (t == 0 && (scale || rdata)) {
        out[0] = chisq;
        out[1] = wnok;
        out[2] = 1.;
    } else if (t == 0) {
        out[2] = 0.;
    }
}

int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void launch_components(const CompParams &p, ElemRec *el, double4 *pos, DevStatus *st,
                       cudaStream_t s) {
    const int n = p.nd + p.ne + p.ns;
    if (n <= 0) return;
    k_components<<<nblk(n, kThreadsC), kThreadsC, 0, s>>>(p, el, pos, st);
    count_launch();
}

void launch_disc_faces(const DiscGeom &dg, const GridDev &g, uint8_t *ndx, double2 *xr,
                       DevStatus *st, cudaStream_t s) {
    if (g.n <= 0) return;
    k_disc_faces<<<nblk(g.n, 256), 256, 0, s>>>(dg, g, ndx, xr, st);
    count_launch();
}

int64_t comp_sums_scratch(int32_t n, int64_t ldc) {
    return 3 * (int64_t)((n + kElemChunk - 1) / kElemChunk) * ldc;
}

void launch_comp_sums(const ElemRec *el, int32_t nd, int32_t ne, int32_t n, double lin,
                      double quad, const PhaseDev &ph, double *part, double *out, int64_t ldc,
                      cudaStream_t s) {
    if (ph.nent <= 0) return;
    const int nchunk = (n + kElemChunk - 1) / kElemChunk;
    if (nchunk == 0) {
        cudaMemsetAsync(out, 0, 3 * ldc * sizeof(double), s);
        return;
    }
    k_comp_sums<<<dim3(nblk(ph.nent, kThreadsC), nchunk), kThreadsC, 0, s>>>(el, nd, ne, n, lin,
                                                                             quad, ph, part, ldc);
    count_launch();
    k_comp_reduce<<<nblk(ph.nent, 256), 256, 0, s>>>(part, nchunk, ph.nent, out, ldc);
    count_launch();
}

void launch_iscale(int32_t flags, int32_t nc, const DatumRec *data, int32_t n,
                   const double *fcomp, double *work, double *calc, double *sfac, double *out,
                   cudaStream_t s) {
    k_iscale<<<1, kThreadsF, 0, s>>>(flags, nc, data, n, fcomp, work, calc, sfac, out);
    count_launch();
}

// ---- host setup -------------------------------------------------------------

namespace eng {

namespace {

// Restricted three-body acceleration in the rotating frame (rocacc.cpp).
void stream_deriv(double q, const double *y, double *dy) {
    const double f1 = 1.0 / (1.0 + q), f2 = f1 * q;
    const double yzsq = sq(y[1]) + sq(y[2]);
    const double r1sq = sq(y[0]) + yzsq, r2sq = sq(y[0] - 1.0) + yzsq;
    const double fm1 = f1 / (r1sq * sqrt(r1sq)), fm2 = f2 / (r2sq * sqrt(r2sq)), fm3 = fm1 + fm2;
    dy[0] = y[3]; dy[1] = y[4]; dy[2] = y[5];
    dy[3] = -fm3 * y[0] + fm2 + 2.0 * y[4] + y[0] - f2;
    dy[4] = -fm3 * y[1] - 2.0 * y[3] + y[1];
    dy[5] = -fm3 * y[2];
}

// One Dormand-Prince 5(4) step (Dormand & Prince 1980); returns the scaled
// error estimate of the embedded pair.
double dp5_step(double q, const double *y, double h, double *yo) {
    static const double A[6][5] = {{1. / 5},
                                   {3. / 40, 9. / 40},
                                   {44. / 45, -56. / 15, 32. / 9},
                                   {19372. / 6561, -25360. / 2187, 64448. / 6561, -212. / 729},
                                   {9017. / 3168, -355. / 33, 46732. / 5247, 49. / 176,
                                    -5103. / 18656},
                                   {35. / 384, 0., 500. / 1113, 125. / 192, -2187. / 6784}};
    static const double B6 = 11. / 84;
    static const double E[7] = {71. / 57600, 0., -71. / 16695, 71. / 1920, -17253. / 339200,
                                22. / 525, -1. / 40};
    double k[7][6], t[6];
    stream_deriv(q, y, k[0]);
    for (int s = 1; s <= 5; s++) {
        for (int i = 0; i < 6; i++) {
            double a = 0.;
            for (int j = 0; j < s; j++) a += A[s - 1][j] * k[j][i];
            t[i] = y[i] + h * a;
        }
        stream_deriv(q, t, k[s]);
    }
    for (int i = 0; i < 6; i++) {
        double a = 0.;
        for (int j = 0; j < 5; j++) a += A[5][j] * k[j][i];
        yo[i] = y[i] + h * (a + B6 * k[5][i]);
    }
    stream_deriv(q, yo, k[6]);
    double err = 0.;
    for (int i = 0; i < 6; i++) {
        double ei = 0.;
        for (int j = 0; j < 7; j++) ei += E[j] * k[j][i];
        ei *= h;
        const double sc = 1e-14 + 1e-13 * std::max(fabs(y[i]), fabs(yo[i]));
        err = std::max(err, fabs(ei) / sc);
    }
    return err;
}

double radius(const double *y) { return sqrt(sq(y[0]) + sq(y[1]) + sq(y[2])); }

}  // namespace

// Where the gas stream from L1 first reaches distance rad from star 1:
// Roche::strinit's start (strining.cpp:14-33) and the motion of rocacc.cpp,
// integrated with Dormand-Prince 5(4) under a tight tolerance, the crossing
// bisected in time to 1e-10 in radius (the accuracy stradv.cpp:27-80 asks
// for). The reference integrates with a Bulirsch-Stoer stepper whose first
// step size is kept in a static between calls, so the two agree to their
// integration error (about 1e-11 in position), not bit for bit.
bool bright_spot_position(double q, double rad, double *pos, Fail &f) {
    const double SMALL = 1.e-5, ACC = 1.e-10, SMAX = 1.e-3, TMAX = 10.;
    const double rl1 = xl1(q);
    if (rl1 < 0) {
        f = {LCG_E_NOCONVERGE, "Roche::xl1(double): exceeded maximum iterations"};
        return false;
    }
    const double mu = q / (1.0 + q);
    const double a = (1.0 - mu) / pow(rl1, 3) + mu / pow((1. - rl1), 3);
    const double lambda1 = sqrt(((a - 2.0) + sqrt(a * (9.0 * a - 8.0))) / 2.0);
    const double m1 = (lambda1 * lambda1 - 2.0 * a - 1.0) / 2.0 / lambda1;
    double y[6] = {rl1 - SMALL, -m1 * SMALL, 0., -lambda1 * SMALL, -lambda1 * m1 * SMALL, 0.};
    double yo[6], ylo[6], h = 1e-4, t = 0.;
    const double rinit = radius(y);
    auto before = [&](double r) { return (rinit > rad && r > rad) || (rinit < rad && r < rad); };
    double rnow = rinit;
    for (int guard = 0; before(rnow); guard++) {
        if (guard > 1000000 || t > TMAX) {
            f = {LCG_E_ROCHE, "Roche::stradv: taken too long without crossing radius"};
            return false;
        }
        h = std::min(h, SMAX);
        const double err = dp5_step(q, y, h, yo);
        if (err > 1.) {
            h *= std::max(0.2, 0.9 * pow(err, -0.2));
            continue;
        }
        std::copy(y, y + 6, ylo);
        std::copy(yo, yo + 6, y);
        t += h;
        rnow = radius(y);
        const double hstep = h;
        h *= err > 0. ? std::min(5., 0.9 * pow(err, -0.2)) : 5.;
        if (!before(rnow)) {
            double lo = 0., hi = hstep, rlo = radius(ylo), rhi = rnow;
            for (int g2 = 0; fabs(rhi - rlo) > ACC && g2 < 200; g2++) {
                const double tt = (lo + hi) / 2.;
                dp5_step(q, ylo, tt, y);
                rnow = radius(y);
                if ((rhi > rad && rnow > rad) || (rhi < rad && rnow < rad)) {
                    rhi = rnow;
                    hi = tt;
                } else {
                    rlo = rnow;
                    lo = tt;
                }
            }
            break;
        }
    }
    pos[0] = y[0];
    pos[1] = y[1];
    pos[2] = y[2];
    return true;
}

// Lobe checks and reference spheres of set_disc_grid / set_disc_edge /
// set_bright_spot_grid (set_disc_grid.cpp:31-66), with the reference's
// message for the component that raises it.
static bool comp_radii(const lcg_model &m, const char *who, CompParams &p, double &rdisc1,
                       Fail &f) {
    double r1, r2;
    get_r1r2(m, r1, r2);
    const double rl1 = xl11(m.q, m.spin1), rl2 = 1. - xl12(m.q, m.spin2);
    char b[160];
    if (r1 < 0) r1 = rl1;
    else if (r1 > rl1) {
        snprintf(b, sizeof b, "%s: the primary star is larger than its Roche lobe!", who);
        f = {LCG_E_LOBE, b};
        return false;
    }
    if (r2 < 0) r2 = rl2;
    else if (r2 > rl2) {
        snprintf(b, sizeof b, "%s: the secondary star is larger than its Roche lobe!", who);
        f = {LCG_E_LOBE, b};
        return false;
    }
    p.r1 = r1;
    p.r2 = r2;
    p.spin1 = m.spin1;
    p.spin2 = m.spin2;
    ref_sphere(kStar1, m.q, m.spin1, r1 / rl1, p.rref1, p.pref1);
    ref_sphere(kStar2, m.q, m.spin2, r2 / rl2, p.rref2, p.pref2);
    rdisc1 = m.rdisc1 > 0. ? m.rdisc1 : r1;
    return true;
}

bool comp_setup(const lcg_model &m, CompParams &p, std::vector<DiscRing> &rings, Fail &f) {
    p = CompParams{};
    rings.clear();
    const double ri = deg2rad(m.iangle);
    p.q = m.q;
    p.cosi = cos(ri);
    p.sini = sin(ri);
    p.delta = m.delta_phase;
    p.eclipse1 = m.eclipse1;
    p.eclipse2 = m.eclipse2;
    p.roche1 = m.roche1;
    p.roche2 = m.roche2;
    p.wave = m.wavelength;
    const double rdisc2 = m.rdisc2 > 0. ? m.rdisc2 : m.radius_spot;
    double rdisc1 = 0.;
    if (m.add_disc) {
        if (!comp_radii(m, "set_disc_grid", p, rdisc1, f)) return false;
        const double EFAC = 1.0000001;
        const double drad = (rdisc2 - rdisc1) / m.nrad, drrad = rdisc2 / m.nrad;
        int off = 0;
        for (int i = 0; i < m.nrad; i++) {
            DiscRing R;
            R.rad = rdisc1 + (rdisc2 - rdisc1) * (i + 0.5) / m.nrad;
            int nt = int(ceil(kTwoPi * R.rad / drrad));
            R.ntheta = nt > 8 ? nt : 8;
            R.h = EFAC * m.height_disc * pow(R.rad, m.beta_disc);
            const double tanp = m.beta_disc * R.h / R.rad;
            R.cosp = 1. / sqrt(1 + sq(tanp));
            R.sinp = tanp * R.cosp;
            R.area = kTwoPi / R.ntheta * R.rad * drad;
            R.off = off;
            off += R.ntheta;
            rings.push_back(R);
        }
        p.nd = off;
        p.nrad = m.nrad;
        p.bright_disc = planck(m.wavelength, m.temp_disc);
        p.rdisc2 = rdisc2;
        p.texp = m.texp_disc;
        // the outer rim (set_disc_edge with outer = true)
        const double size = rdisc2 / m.nrad;
        p.rad_e = rdisc2;
        p.h_e = m.height_disc * pow(p.rad_e, m.beta_disc);
        p.nout = int(2 * p.h_e / size) + 2;
        const int nt = int(ceil(kTwoPi * p.rad_e / size));
        p.ntheta_e = nt > 8 ? nt : 8;
        p.area_e = kTwoPi / p.ntheta_e * p.rad_e * 2 * p.h_e / (p.nout - 1);
        p.ne = p.ntheta_e * p.nout;
        p.tedge = m.temp_edge;
        p.t2 = fabs(m.t2);
        p.absorb_edge = m.absorb_edge;
        p.opaque = m.opaque;
        if (m.opaque && m.beta_disc < 1 && (p.nd + p.ne) > 0) {
            f = {LCG_E_ROCHE, "Roche::disc_eclipse: beta must be >= 1"};
            return false;
        }
    }
    p.dg = DiscGeom{sin(kPi / 180. * m.iangle), cos(kPi / 180. * m.iangle), rdisc1, rdisc2,
                    m.beta_disc, m.height_disc};
    if (m.add_spot) {
        double rd1;
        if (!comp_radii(m, "set_bright_spot_grid", p, rd1, f)) return false;
        if (m.nspot < 2) {
            f = {LCG_E_INVALID, "set_bright_spot_grid: nspot must be at least 2"};
            return false;
        }
        if (!bright_spot_position(m.q, m.radius_spot, p.bspot, f)) return false;
        const double theta =
            atan2(p.bspot[1], p.bspot[0]) + kTwoPi / 4. + deg2rad(m.angle_spot);
        const double alpha = deg2rad(m.yaw_spot), tilt = deg2rad(m.tilt_spot);
        p.bvec[0] = cos(theta); p.bvec[1] = sin(theta); p.bvec[2] = 0;
        p.tvec[0] = sin(tilt) * sin(theta + alpha);
        p.tvec[1] = -sin(tilt) * cos(theta + alpha);
        p.tvec[2] = cos(tilt);
        p.bmax = pow(m.expon_spot / m.epow_spot, 1. / m.epow_spot);
        p.sfac = 20. + p.bmax;
        p.area_s = p.sfac * m.length_spot * m.height_spot / (m.nspot - 1);
        p.bright_s = planck(m.wavelength, m.temp_spot);
        p.expon = m.expon_spot;
        p.epow = m.epow_spot;
        p.cfrac = m.cfrac_spot;
        p.length = m.length_spot;
        p.nspot = m.nspot;
        p.ns = 2 * m.nspot;
    }
    return true;
}

}  // namespace eng
}  // namespace lcg
