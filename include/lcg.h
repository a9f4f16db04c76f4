/*
 * lcg.h — C ABI of the B200 light-curve engine.
 *
 * This is the drop-in boundary for lcurve_re's model-evaluation hot path.
 * Every entry point takes plain pointers and sizes; no C++ or torch types
 * cross it. The reference interface each one replaces is cited beside it
 * (paths are relative to the lcurve_re source tree).
 *
 *   lcg_light_curve        <- Lcurve::light_curve_comp
 *                             (src/lcurve_base/lcurve.h:669-674,
 *                              src/lcurve_base/light_curve_comp.cpp:119-599)
 *   lcg_light_curve_batch  <- many light_curve_comp calls at once (the
 *                             MCMC / Levenberg-Marquardt callers,
 *                             new_scripts/mcmc_solver.cpp:1062-1070,
 *                             new_scripts/levmarq_solver.cpp:789-886)
 *   lcg_star_grid          <- Lcurve::set_star_grid + set_star_continuum
 *                             (src/lcurve_base/lcurve.h:528,550)
 *   lcg_components         <- Lcurve::set_disc_grid, set_disc_edge,
 *                             set_bright_spot_grid + their continua
 *                             (src/lcurve_base/lcurve.h:539-561)
 *   lcg_sum_star_multi     <- Lcurve::flat_sum_star1_multi / _star2_multi
 *                             (src/lcurve_base/lcurve.h:299-307) and the
 *                             reference CUDA hooks cuda_sum_star{1,2}_multi
 *                             (src/lcurve_base/comp_light_cuda.h:13-20)
 *
 * Errors: every call returns an lcg_status. The reference throws C++
 * exceptions instead (Lcurve::Lcurve_Error, Roche::Roche_Error); a C++ shim
 * rethrows Lcurve_Error(lcg_last_error(ctx)) for any status != LCG_OK.
 * There is no CPU fallback: a missing device or a CUDA failure is an error.
 *
 * Threading: a context owns one CUDA stream and its device buffers. A
 * context is used by one host thread at a time (the reference keeps its
 * caches thread_local, light_curve_comp.cpp:161).
 */
#ifndef LCG_H
#define LCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LCG_ABI_VERSION 3

typedef enum lcg_status {
    LCG_OK = 0,
    LCG_E_INVALID = 1,      /* bad argument (null pointer, n < 1, q <= 0 ...) */
    LCG_E_LOBE = 2,         /* a star overfills its Roche lobe (Lcurve_Error) */
    LCG_E_ROCHE = 3,        /* radius / eclipse solve failed (Roche_Error)    */
    LCG_E_NOCONVERGE = 4,   /* an iteration cap was reached                   */
    LCG_E_UNSUPPORTED = 5,  /* a model or call this engine does not evaluate  */
    LCG_E_CUDA = 6,         /* CUDA runtime failure or no device              */
    LCG_E_NOMEM = 7,        /* device or host allocation failed               */
    LCG_E_CAPACITY = 8      /* a size exceeds a fixed capacity                */
} lcg_status;

/* Limb-darkening law, Lcurve::LDC::LDCtype (src/lcurve_base/lcurve.h:204). */
enum { LCG_LIMB_POLY = 0, LCG_LIMB_CLARET = 1 };

/* Which star, Roche::STAR (src/lroche_base/roche.h:13). */
enum { LCG_STAR1 = 0, LCG_STAR2 = 1 };

/* Arithmetic of the per-face flux sum.
 *   LCG_PREC_FP64  : every element in FP64, faces summed in 1024-face blocks
 *                    in ascending order and the blocks merged in order, the
 *                    same arithmetic sequence as comp_light_flat.cpp:241-372.
 *   LCG_PREC_MIXED : element geometry and intensity in FP32, eclipse masks
 *                    in 32-bit fixed-point phase, FP32 partial sums of at
 *                    most LCG_MIXED_FOLD faces folded into FP64.
 * The grid, eclipse and continuum stages are FP64 in both modes. */
enum { LCG_PREC_FP64 = 0, LCG_PREC_MIXED = 1 };
#define LCG_MIXED_FOLD 64

/* Flags of lcg_light_curve, the bool arguments of light_curve_comp. */
enum {
    LCG_FLAG_SCALE = 1,        /* scale: fit the single scale factor (re_scale) */
    LCG_FLAG_RDATA = 2,        /* rdata: real data, compute chi**2             */
    LCG_FLAG_INFO = 4,         /* info: print face counts to stderr            */
    LCG_FLAG_DIAGNOSTICS = 8,  /* diagnostics: wdwarf, logg1/2, rv1/2          */
    LCG_FLAG_NO_CACHE = 16     /* rebuild grids even if the geometry is equal
                                  (LCURVE_NO_GRID_CACHE, light_curve_comp.cpp:162) */
};

/* Indices into the scalars[] output of lcg_light_curve: the scalar
 * out-parameters of light_curve_comp, in signature order. */
enum {
    LCG_OUT_WDWARF = 0, LCG_OUT_CHISQ = 1, LCG_OUT_WNOK = 2,
    LCG_OUT_LOGG1 = 3, LCG_OUT_LOGG2 = 4, LCG_OUT_RV1 = 5, LCG_OUT_RV2 = 6,
    LCG_NOUT = 7
};

/* Every Model field that the hot path reads (src/lcurve_base/lcurve.h:340-396),
 * as plain values. Pparam values are given by value; "defined" flags only
 * matter for the optional star spots (set_star_continuum.cpp:58-65). */
typedef struct lcg_model {
    double q, iangle, r1, r2, cphi3, cphi4, spin1, spin2;
    double t1, t2;
    double ldc1[4], ldc2[4];
    double velocity_scale, beam_factor1, beam_factor2;
    double t0, period, pdot, deltat;
    double gravity_dark1, gravity_dark2;
    double absorb, slope, quad, cube, third;
    /* star spots 11,12,13,21,22: {long, lat, fwhm, tcen}; a spot is on when
       all four of its Pparams are defined */
    double stsp[5][4];
    int32_t stsp_defined[5];
    /* uniform equatorial spot: long1, long2, lathw, taper, temp */
    double uesp[5];
    int32_t uesp_defined;
    /* computational parameters */
    double delta_phase;
    int32_t nlat1f, nlat2f, nlat1c, nlat2c;
    int32_t npole, nlatfill, nlngfill;
    double lfudge, llo, lhi, phase1, phase2, wavelength;
    int32_t roche1, roche2, eclipse1, eclipse2, glens1, use_radii;
    double tperiod;
    int32_t gdark_bolom1, gdark_bolom2;
    double mucrit1, mucrit2;
    int32_t limb1, limb2;
    int32_t mirror, add_disc, opaque, add_spot, iscale;
    int32_t pad_;
    /* accretion disc with its outer edge (read when add_disc is set) and the
       bright spot (read when add_spot is set), model.cpp:211-230,353-357 */
    double rdisc1, rdisc2, height_disc, beta_disc, temp_disc, texp_disc;
    double lin_limb_disc, quad_limb_disc, temp_edge, absorb_edge;
    double radius_spot, length_spot, height_spot, expon_spot, epow_spot;
    double angle_spot, yaw_spot, temp_spot, tilt_spot, cfrac_spot;
    int32_t nrad, nspot;
} lcg_model;

/* One light-curve point, byte-compatible with Lcurve::Datum
 * (src/lcurve_base/lcurve.h:427-445): a Data vector's storage can be passed
 * as-is. */
typedef struct lcg_datum {
    double time, expose, flux, ferr, weight;
    int32_t ndiv;
    int32_t pad_;
} lcg_datum;

typedef struct lcg_options {
    int32_t device;        /* CUDA device ordinal                          */
    int32_t precision;     /* LCG_PREC_FP64 or LCG_PREC_MIXED              */
    int32_t verbose;       /* print per-stage timings at destroy when > 0  */
    int32_t eclipse_warp;  /* Roche eclipse candidates up to which one warp
                              bisects each face (the rest: one thread per
                              face); -1 never. 0 automatic: one thread per
                              face whenever the FP32 screen of the
                              bisections serves the faces (mixed contexts,
                              stars with r >= 0.01), else a warp per face
                              up to twice the GPU's resident warps       */
    int32_t reserved[4];
} lcg_options;

typedef struct lcg_ctx lcg_ctx;

/* ---- context ----------------------------------------------------------- */

/* Fills *opt with defaults: device 0, mixed precision. */
void lcg_default_options(lcg_options *opt);

/* Creates a context on opt->device. Fails with LCG_E_CUDA when there is no
 * usable sm_100 device. */
lcg_status lcg_create(lcg_ctx **ctx, const lcg_options *opt);

void lcg_destroy(lcg_ctx *ctx);

/* Message of the last failing call on ctx ("" if none). Valid until the next
 * call on ctx. A NULL ctx returns the message of the last failed create. */
const char *lcg_last_error(const lcg_ctx *ctx);

int32_t lcg_abi_version(void);

/* The context's cudaStream_t, so callers can order their own work and
 * events against the engine. */
void *lcg_stream(lcg_ctx *ctx);

/* ---- the hot path ------------------------------------------------------ */

/* One light curve for one model: Lcurve::light_curve_comp.
 *   data[n]      the points (time, expose, flux, ferr, weight, ndiv)
 *   flags        LCG_FLAG_*
 *   sfac[5]      in: sfac[0] is the scale when LCG_FLAG_SCALE is clear;
 *                out: all five set to the fitted scale when it is set
 *   calc[n]      out: the model light curve
 *   scalars[7]   out: wdwarf, chisq, wnok, logg1, logg2, rv1, rv2
 * Grids are rebuilt only when a geometry parameter changed since the last
 * call on this context, and the continuum only when a brightness parameter
 * changed (the exact-reuse cache of light_curve_comp.cpp:34-117). */
lcg_status lcg_light_curve(lcg_ctx *ctx, const lcg_model *model,
                           const lcg_datum *data, int32_t n, int32_t flags,
                           double *sfac, double *calc, double *scalars);

/* Resident-data form of lcg_light_curve for callers that evaluate many
 * models over the same points (samplers, Jacobians): lcg_set_data copies the
 * points to the device once; lcg_light_curve_resident then evaluates a model
 * over them. calc may be NULL, leaving the curve on the device only
 * (lcg_device_calc). lcg_light_curve is lcg_set_data followed by
 * lcg_light_curve_resident. The reference passes the Data on every call
 * (light_curve_comp.cpp:119); these two split that call. */
lcg_status lcg_set_data(lcg_ctx *ctx, const lcg_datum *data, int32_t n);
lcg_status lcg_light_curve_resident(lcg_ctx *ctx, const lcg_model *model, int32_t flags,
                                    double *sfac, double *calc, double *scalars);
/* Lcurve::light_curve_comp_fast (light_curve_comp_fast.cpp:6-84): with more
 * than max_model_points points, the curve is computed at max_model_points
 * points picked uniformly by index (both ends included), interpolated
 * linearly in time to every point, and, with LCG_FLAG_RDATA, chi**2 and wnok
 * are recomputed over all points; otherwise it is lcg_light_curve. The scale
 * fitted (LCG_FLAG_SCALE) is the subsample's. max_model_points >= 2. The
 * sampler and Levenberg-Marquardt callers use it (mcmc_solver.cpp:1066,
 * levmarq_solver.cpp:679). */
lcg_status lcg_light_curve_fast(lcg_ctx *ctx, const lcg_model *model,
                                const lcg_datum *data, int32_t n, int32_t flags,
                                int32_t max_model_points, double *sfac, double *calc,
                                double *scalars);
/* Device pointer to the last light curve computed on ctx (n doubles). */
const double *lcg_device_calc(lcg_ctx *ctx);

/* nmodels light curves over the same data points, one per model.
 *   calc[nmodels*n], chisq[nmodels], wnok[nmodels], sfac[nmodels*5] out;
 *   status[nmodels] out: the per-model status (a failed model does not fail
 *   the batch; its calc row is zero). sfac is read when SCALE is clear.
 * Returns LCG_OK unless the batch as a whole could not run.
 * On a mixed-precision context, models without beaming, lensing, mucrit > 0,
 * separate coarse grids or infill are evaluated together: every stage runs
 * once for the whole batch (one CUDA graph, replayed while the batch keeps
 * its size and grid resolutions), and a model's grids are rebuilt only when
 * its geometry parameters changed since the previous batch call on ctx (its
 * continuum only when its brightness parameters did). Other models (every
 * model on an FP64 context) take the single-model path, concurrently on up
 * to eight worker contexts of ctx's device and precision (one host thread
 * and stream each, created on first use, holding a copy of the resident
 * points): their results are those of single calls. LCG_FLAG_DIAGNOSTICS is
 * ignored. */
lcg_status lcg_light_curve_batch(lcg_ctx *ctx, const lcg_model *models,
                                 int32_t nmodels, const lcg_datum *data,
                                 int32_t n, int32_t flags, double *sfac,
                                 double *calc, double *chisq, double *wnok,
                                 int32_t *status);

/* lcg_light_curve_batch over the points of lcg_set_data. calc, chisq and
 * wnok may be NULL: a sampler that needs the curves of a few models only
 * passes calc = NULL and fetches those rows with lcg_batch_curves. */
lcg_status lcg_light_curve_batch_resident(lcg_ctx *ctx, const lcg_model *models,
                                          int32_t nmodels, int32_t flags, double *sfac,
                                          double *calc, double *chisq, double *wnok,
                                          int32_t *status);

/* Rows (model indices) of the light curves of the last batch call on ctx,
 * copied to out [count x n]; the rows of models that call skipped as
 * unchanged hold their earlier curves. */
lcg_status lcg_batch_curves(lcg_ctx *ctx, const int32_t *rows, int32_t count, double *out);

/* The same rows gathered into device memory dst [count x n] (on ctx's
 * device), for a caller that keeps them there; returns when they are
 * written. rows = NULL with count = the batch's model count copies every row. */
lcg_status lcg_batch_curves_device(lcg_ctx *ctx, const int32_t *rows, int32_t count,
                                   double *dst);

/* ---- stage-level seams, for parity tests and integrations -------------- */

/* Number of faces of one star grid (Lcurve::numface, numface.cpp:14-52, and
 * the infill band of set_star_grid.cpp:113-159). */
lcg_status lcg_star_face_count(lcg_ctx *ctx, const lcg_model *model,
                               int32_t star, int32_t fine, int32_t *nface);

/* Builds one star grid with its continuum, in the reference's face order
 * (set_star_grid.cpp:49-523 then set_star_continuum.cpp:26-297). Outputs are
 * host arrays of length nface (posn, dirn: 3*nface, x,y,z interleaved).
 * ecl_in/ecl_out hold the ingress/egress phase of faces with neclipse = 1. */
lcg_status lcg_star_grid(lcg_ctx *ctx, const lcg_model *model, int32_t star,
                         int32_t fine, int32_t nface, double *posn,
                         double *dirn, float *area, float *gravity,
                         float *flux, int32_t *neclipse, double *ecl_in,
                         double *ecl_out);

/* One component grid of a model as light_curve_comp builds it: which = 0
 * the accretion disc (set_disc_grid.cpp:27-127 with set_disc_continuum),
 * 1 its outer rim (set_disc_grid.cpp:144-264 with set_edge_continuum),
 * 2 the bright spot (set_bright_spot_grid.cpp:27-100). *n gets the element
 * count; when it is <= cap the host arrays are filled: posn, dirn (3 per
 * element), float area and flux, the number of eclipse ranges nr and the
 * ranges in rin / rout (4 per element, in the reference's push order). */
lcg_status lcg_components(lcg_ctx *ctx, const lcg_model *model, int32_t which,
                          int32_t cap, int32_t *n, double *posn, double *dirn,
                          float *area, float *flux, int32_t *nr, double *rin,
                          double *rout);

/* The blocked multi-phase flux sweep over one flattened grid: out[k] is the
 * unweighted flux sum for phase entry k (flat_sum_star{1,2}_multi).
 *   grid: n faces in FlatGrid order, [0,n0) never eclipsed, [n0,n) one
 *         eclipse range (in1/out1 indexed i-n0). Faces with two or more
 *         ranges do not occur for stars without a disc.
 *   ldc[4], ltype, mucrit: limb darkening; beam, spin, vfac, xcofm: Doppler
 *   beaming (comp_light_flat.cpp:109-168); glens1/rlens1: lensing (star 2).
 * Host arrays in and out. */
lcg_status lcg_sum_star_multi(lcg_ctx *ctx, int32_t star, int64_t n,
                              int64_t n0, const double *dx, const double *dy,
                              const double *dz, const double *px,
                              const double *py, const double *pz,
                              const double *flux, const double *in1,
                              const double *out1, int32_t nent,
                              const double *ex, const double *ey,
                              const double *ez, const double *phin,
                              const double *ldc, int32_t ltype, double mucrit,
                              double beam, double spin, double vfac,
                              double xcofm, int32_t glens1, double rlens1,
                              double *out);

/* Allocation-free form of the FP64 sweep of lcg_sum_star_multi, for callers
 * in which this library must not allocate device memory: programs whose
 * device memory is already claimed by another framework's pooling allocator
 * (a cudaMalloc from here would fail), or latency-critical loops in which an
 * allocation would synchronise the device. No counterpart in the reference.
 *   All arrays are DEVICE arrays owned by the caller (same meaning as in
 *   lcg_sum_star_multi; in1/out1 of length n-n0); ldc is a host array of 4.
 *   Runs on `stream` (a cudaStream_t; NULL = the legacy default stream) on
 *   the device that owns `out`, and leaves the caller's current device as it
 *   found it; returns without waiting for the GPU.
 *   Only faces with zero or one eclipse range ([0,n0) and [n0,n)): faces with
 *   several ranges (opaque discs) have no place in this form's arguments.
 *   No beaming or lensing in this form; FP64 arithmetic of the reference.
 *   A launch failure returns LCG_E_CUDA and consumes the runtime's record of
 *   that failure; errors left by the caller's earlier work are not cleared.
 * Scratch: a fixed 16 MiB device array inside the library (held by every GPU
 * that loads it, until exit): ceil(n/1024) * nent must not exceed 2,097,152
 * and ceil(n/1024) must not exceed 65,535, else LCG_E_CAPACITY is returned
 * and nothing runs. The first call on a device looks up that array's
 * address (set-up, no allocation); make it before any stream capture. All
 * calls share the array: calls that overlap on the GPU race and must be
 * ordered by the caller. Calls no cudaMalloc/cudaFree. */
lcg_status lcg_sum_star_multi_noalloc(void *stream, int32_t star, int64_t n, int64_t n0,
                                      const double *dx, const double *dy, const double *dz,
                                      const double *flux, const double *in1,
                                      const double *out1, int32_t nent, const double *ex,
                                      const double *ey, const double *ez, const double *phin,
                                      const double *ldc, int32_t ltype, double mucrit,
                                      double *out);

/* ---- measurement ------------------------------------------------------- */

/* Stage timings recorded with CUDA events on the context's stream when
 * profiling is on: device milliseconds summed since the last reset, and the
 * number of launches, per stage. */
enum {
    LCG_STAGE_GRID = 0, LCG_STAGE_ECLIPSE = 1, LCG_STAGE_CONTINUUM = 2,
    LCG_STAGE_FLATTEN = 3, LCG_STAGE_PHASES = 4, LCG_STAGE_FLUX = 5,
    LCG_STAGE_REDUCE = 6, LCG_NSTAGE = 7
};
void lcg_set_profiling(lcg_ctx *ctx, int32_t on);
void lcg_stage_times(lcg_ctx *ctx, double *ms, int64_t *launches,
                     int32_t reset);

/* Elements (face x sub-phase pairs) summed by the flux stage since the last
 * reset: the algorithmic unit of the flux roofline. */
int64_t lcg_flux_elements(lcg_ctx *ctx, int32_t reset);

/* Kernels launched by this library in this process (all contexts) since the
 * last reset. */
int64_t lcg_kernel_launches(int32_t reset);

/* Measures the device's FP32 FMA throughput in TFLOP/s (2 FLOP per FMA)
 * with a register-resident FFMA chain kernel; the denominator of the flux
 * roofline. */
lcg_status lcg_measure_fp32_peak(lcg_ctx *ctx, double *tflops);

/* The same with a DFMA chain: the device's FP64 FMA throughput, the
 * denominator of the FP64 sweep's roofline. */
lcg_status lcg_measure_fp64_peak(lcg_ctx *ctx, double *tflops);

/* ---- surrogate network kernels (no reference counterpart) -------------
 * The delayed-acceptance sampler screens proposals with a small MLP whose
 * training and inference run on these kernels. Device pointers, all on the
 * caller's stream; BF16 matrices are row-major.
 *
 * lcg_mlp_gemm: D[m x n] = A[m x k] * B[n x k]^T on the tensor cores (BF16
 * in, FP32 accumulate), m a multiple of 128, k of 64, n of 64; A, B 16-byte
 * aligned. epi selects the fused epilogue:
 *   LCG_EPI_GELU    z = D + bias (BF16), y = GELU(z) (BF16), yt = y^T
 *                   (BF16, row stride ldt; may be NULL)
 *   LCG_EPI_LINEAR  out = D + bias (FP32)
 *   LCG_EPI_DGELU   y = D * GELU'(z) with z read (BF16), yt = y^T
 *   LCG_EPI_F32     out = D (FP32)
 * Rows >= mvalid are not stored. *err (may be NULL) is set if a pipeline
 * wait timed out. */
enum { LCG_EPI_GELU = 0, LCG_EPI_LINEAR = 1, LCG_EPI_DGELU = 2, LCG_EPI_F32 = 3 };
lcg_status lcg_mlp_gemm(void *stream, int32_t epi, int32_t m, int32_t n, int32_t k,
                        const void *a, const void *b, const float *bias, void *z, void *y,
                        void *yt, float *out, int32_t mvalid, int32_t ldt, int32_t *err);
/* Adam step on FP32 master weights [rows x cols] (moments m1, m2), writing
 * the BF16 weights and their BF16 transpose (either may be NULL). */
lcg_status lcg_mlp_adam(void *stream, float *w, float *m1, float *m2, const float *g,
                        int32_t rows, int32_t cols, float lr, float beta1, float beta2,
                        float eps, int32_t step, void *w_bf16, void *wt_bf16);
/* One Adam step on n <= 16 tensors in one launch (tensor j: FP32 weights
 * w[j] [rows[j] x cols[j]], moments m1[j] and m2[j], gradient g[j]; BF16
 * copy w_bf16[j] and BF16 transpose wt_bf16[j], either array or entry may
 * be NULL). The host arrays hold device pointers. Learning rate and bias
 * corrections come from device memory so that one captured graph serves
 * every step: sched = {lr_max, lr_min, total_steps, beta1, beta2, eps}
 * (FP32), step = the number of steps taken before this one (int32);
 * lr = lr_min + (lr_max - lr_min) (1 + cos(pi step / total_steps)) / 2, or
 * lr_max when total_steps <= 0. The caller advances *step. */
lcg_status lcg_mlp_adam_all(void *stream, int32_t n, float *const *w, float *const *m1,
                            float *const *m2, const float *const *g, const int32_t *rows,
                            const int32_t *cols, void *const *w_bf16, void *const *wt_bf16,
                            const float *sched, const int32_t *step);
/* out[c] = sum over the first rvalid rows of the BF16 [rows x cols] g. */
lcg_status lcg_mlp_colsum(void *stream, const void *g_bf16, int32_t rows, int32_t cols,
                          int32_t rvalid, float *out);
/* Gradient of the mean squared error of out against target ([rows x cols]
 * FP32, first rvalid rows), as BF16 and its BF16 transpose (row stride ldt),
 * and the per-row squared-error sums (may be NULL). cols <= 256. */
lcg_status lcg_mlp_mse_grad(void *stream, const float *out, const float *target, int32_t rows,
                            int32_t cols, int32_t rvalid, int32_t ldt, void *g_bf16,
                            void *gt_bf16, float *loss_rows);
/* Input layer in FP32 (kin <= 16): z = x w^T + b, y = GELU(z) as BF16 [m x n]
 * (z and yt = y^T, row stride ldt, may be NULL); rows >= mvalid are zero. */
lcg_status lcg_mlp_input(void *stream, const float *x, int32_t kin, const float *w,
                         const float *b, int32_t m, int32_t n, int32_t mvalid, void *z, void *y,
                         void *yt, int32_t ldt);
/* dw[n x kin] = g^T x over the first mvalid rows (g BF16 [m x n], x FP32). */
lcg_status lcg_mlp_input_grad(void *stream, const void *g_bf16, const float *x, int32_t kin,
                              int32_t m, int32_t n, int32_t mvalid, float *dw);
/* The whole network nin -> (depth - 1) x 256 GELU -> nout (linear) for m
 * rows (a multiple of 128) in one launch, one CTA per 128 rows, activations
 * kept on chip between layers:
 *   layer 0 in FP32 on the CUDA cores from x [m x kin] (kin <= 16), w0
 *   [256 x kin], b0 [256] (rows >= mvalid are zero); layers 1..depth from
 *   the BF16 weights w_bf16[l - 1] ([256 x 256], the last [nout x 256]) and
 *   FP32 biases bias[l - 1] on the tensor cores; out [mvalid x nout] FP32.
 * Training (z non-NULL): stores the BF16 pre-activations z[l] [m x 256] and
 * transposed activations yt[l] [256 x ldt] of layers 0..depth-1 (ldt >= m,
 * a multiple of 8). With target [m x nout] (FP32) also the gradient of the
 * mean squared error over the first mvalid rows, 2 (out - target) /
 * (mvalid nout), as BF16 g [m x nout] and its transpose gt [nout x ldt],
 * and per-row squared-error sums loss_rows [m] (may be NULL). depth <= 5,
 * nout a multiple of 64 up to 256; host arrays of device pointers; vector
 * stores need 16-byte aligned out, g, z and yt. *err (may be NULL) is set
 * if a pipeline wait timed out. */
lcg_status lcg_mlp_forward(void *stream, const float *x, int32_t kin, int32_t m, int32_t mvalid,
                           const float *w0, const float *b0, int32_t depth, int32_t nout,
                           const void *const *w_bf16, const float *const *bias, float *out,
                           void *const *z, void *const *yt, int32_t ldt, const float *target,
                           void *g, void *gt, float *loss_rows, int32_t *err);
/* The backward chain of the same network in one launch: from the output
 * gradient g_out [m x nout] (BF16), for j = 0..depth-1 the gradient of
 * layer depth-1-j, g[j] = (g_prev * W) * GELU'(z[j]) with wt_bf16[j] the
 * BF16 transpose of layer depth-j's weights ([256 x nout] for j = 0, then
 * [256 x 256]) and z[j] that layer's stored pre-activation [m x 256];
 * stores g[j] [m x 256] and, where gt and gt[j] are non-NULL, its transpose
 * [256 x ldt]. */
lcg_status lcg_mlp_backward_data(void *stream, int32_t m, int32_t depth, int32_t nout,
                                 const void *g_out, const void *const *wt_bf16,
                                 const void *const *z, void *const *g, void *const *gt,
                                 int32_t ldt, int32_t *err);
/* Per row r of coef [m x ncoef]: the surrogate curve s(c) = mean + c * basis
 * (basis [ncoef x npts]) at the data points, or, with an anchor (exact curves
 * [m x npts] at the points coef_x [m x ncoef] describes), the anchored curve
 * anchor * s(coef) / s(coef_x); then chi**2 of the data after the optimal
 * scale s = sum(w f y / e^2) / sum(w f^2 / e^2), as re_scale does
 * (chisq[m]; scale[m] may be NULL; coef_x and anchor NULL for none). */
lcg_status lcg_mlp_pca_chisq(void *stream, const float *coef, int32_t m, int32_t ncoef,
                             const float *basis, const float *mean, int32_t npts,
                             const double *flux, const double *ferr, const double *weight,
                             const float *coef_x, const double *anchor, double *chisq,
                             double *scale);

/* The inner steps of the sampler's surrogate transitions (no counterpart
 * in the reference, whose mcmc_solver runs plain Metropolis): a random walk
 * through a triangular quadratic map that straightens a curved posterior,
 * screened by the surrogate's chi**2, one thread per chain, every argument
 * a device pointer. par holds the walk, 7d + 2d^2 + d^3 doubles for
 * dimension d (d <= 16): m[d] s[d] (z = (y - m) / s), c0[d] B[d*d] (B[i*d+k]
 * multiplies z_i in P_k, i < k), A[d*d*d] (A[(k*d+i)*d+j] multiplies z_i z_j
 * in P_k, i <= j < k), chol[d*d] (row-major lower-triangular step factor),
 * mid[d] half[d] (the network's input (y - mid) / half), lo[d] hi[d] (the
 * box). With u = T(z), u_k = z_k - P_k(z_<k), the proposal of chain i is
 * T^-1(T(y_i) + chol n_i), n_i standard normal: from noise [nc x d] when
 * non-NULL, else Philox4x32-10 (subsequence i, offset from *ctr + step).
 * lcg_walk_propose writes prop [nc x d], xunit [nc x d] (FP32) and ok [nc]
 * (inside the box). lcg_walk_accept moves chain i to prop_i when
 * ok_i and log(u_i) < -(chi_i - chis_i) / 2 (u_i from unif when non-NULL),
 * updating y, chis and moves (may be NULL). lcg_walk_advance adds inc to
 * *ctr (the step counter a captured graph of steps reads). */
lcg_status lcg_walk_propose(void *stream, int32_t nc, int32_t d, const double *par,
                            const double *y, uint64_t seed, const int64_t *ctr, int32_t step,
                            const double *noise, double *prop, float *xunit, uint8_t *ok);
lcg_status lcg_walk_accept(void *stream, int32_t nc, int32_t d, const double *prop,
                           const uint8_t *ok, const double *chi, double *y, double *chis,
                           int32_t *moves, uint64_t seed, const int64_t *ctr, int32_t step,
                           const double *unif);
lcg_status lcg_walk_advance(void *stream, int64_t *ctr, int64_t inc);

#ifdef __cplusplus
}
#endif

#endif /* LCG_H */
