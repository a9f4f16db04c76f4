/*
 * lcg_oracle.h — CPU restatement of lcurve_re's model-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA engine is compared
 * against; it is never linked into, loaded by, or called from the product
 * library. Only tests/, the smoke check and the CPU-baseline leg of the
 * benchmark may use it.
 *
 * Every function restates one reference routine in plain C, in the same
 * floating-point operation order (build with -ffp-contract=off), and cites
 * the reference file:line it follows. Results are pinned against the
 * reference itself, compiled from its own sources into oracle/_ref by
 * oracle/Makefile (see tests/test_oracle_pin.py).
 */
#ifndef LCG_ORACLE_H
#define LCG_ORACLE_H

#include <stdint.h>
#include "../include/lcg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of faces of one star grid (set_star_grid.cpp:49-162). */
int lco_face_count(const lcg_model *m, int star, int fine, int32_t *nface,
                   char *err, int errlen);

/* One star grid in the reference's face order with the continuum applied
 * (set_star_grid.cpp:49-523, set_star_continuum.cpp:26-297). */
int lco_star_grid(const lcg_model *m, int star, int fine, int32_t nface,
                  double *posn, double *dirn, float *area, float *gravity,
                  float *flux, int32_t *neclipse, double *ecl_in,
                  double *ecl_out, char *err, int errlen);

/* The blocked multi-phase sweep (comp_light_flat.cpp:241-372). */
int lco_sum_star_multi(int star, int64_t n, int64_t n0, const double *dx,
                       const double *dy, const double *dz, const double *px,
                       const double *py, const double *pz, const double *flux,
                       const double *in1, const double *out1, int32_t nent,
                       const double *ex, const double *ey, const double *ez,
                       const double *phin, const double *ldc, int32_t ltype,
                       double mucrit, double beam, double spin, double vfac,
                       double xcofm, int32_t glens1, double rlens1,
                       double *out);

/* Flattens a star grid into FlatGrid order (comp_light_flat.cpp:26-65).
 * Outputs have length nface; in1/out1 have length n1-n0. Returns n0 in
 * *n0_out and n1 in *n1_out. Faces with >= 2 ranges never occur for stars. */
int lco_flatten(int32_t nface, const double *posn, const double *dirn,
                const float *flux, const int32_t *neclipse,
                const double *ecl_in, const double *ecl_out, double *dx,
                double *dy, double *dz, double *px, double *py, double *pz,
                double *fflux, double *in1, double *out1, int64_t *n0_out,
                int64_t *n1_out);

/* Sub-exposure phase batch of light_curve_comp.cpp:358-455 for coarse =
 * fine grids: for each datum, ndiv entries. Returns the number of entries
 * (sum of ndiv). Arrays must hold that many. */
int64_t lco_phase_batch(const lcg_model *m, const lcg_datum *data, int32_t n,
                        double *ex, double *ey, double *ez, double *phin,
                        double *w1, double *w2, int32_t *idx);

/* One component grid as light_curve_comp builds it: which = 0 the disc
 * (set_disc_grid.cpp:27-127 + set_disc_continuum), 1 its outer edge
 * (set_disc_grid.cpp:144-264 + set_edge_continuum), 2 the bright spot
 * (set_bright_spot_grid.cpp:27-100). *nout gets the element count; the
 * arrays (3 per element for posn/dirn, maxr per element for rin/rout) are
 * filled when it is <= cap. nr holds each element's number of ranges. */
int lco_components(const lcg_model *m, int32_t which, int32_t cap, int32_t maxr,
                   int32_t *nout, double *posn, double *dirn, float *area, float *flux,
                   int32_t *nr, double *rin, double *rout, char *err, int errlen);

/* The whole path: Lcurve::light_curve_comp (light_curve_comp.cpp:119-599). */
int lco_light_curve(const lcg_model *m, const lcg_datum *data, int32_t n,
                    int32_t flags, double *sfac, double *calc,
                    double *scalars, char *err, int errlen);

/* Lcurve::light_curve_comp_fast (light_curve_comp_fast.cpp:6-84): above
 * max_pts points, evaluate on max_pts points uniform in index and
 * interpolate linearly in time; chi**2 recomputed when rdata is set. */
int lco_light_curve_fast(const lcg_model *m, const lcg_datum *data, int32_t n,
                         int32_t flags, int32_t max_pts, double *sfac, double *calc,
                         double *scalars, char *err, int errlen);

/* Scalars derived once per model (light_curve_comp.cpp:130-138,
 * set_star_grid.cpp:63-108): r1, r2, rl1, rl2, rref1, pref1, rref2, pref2,
 * ffac1, ffac2, gref1, gref2. Returns a status. */
int lco_model_scalars(const lcg_model *m, double *out12, char *err,
                      int errlen);

#ifdef __cplusplus
}
#endif

#endif
