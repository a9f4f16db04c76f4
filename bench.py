#!/usr/bin/env python
"""Benchmark: light curves per second of the B200 engine.

Workload (default wd_dm_large): the detached WD+dM binary at nlat 200/800
(50,872 + 814,520 faces), 5000 points x ndiv 5 = 25,000 sub-exposure phases
= 2.163e10 face-phase elements per light curve, synthetic seeded data. A
step is one full light curve with the grids rebuilt (the cache disabled), as
in an MCMC step whose geometry changes.

  value  light curves/s with the points resident on the device
         (lcg_set_data once, lcg_light_curve_resident per step)
  e2e    the same through lcg_light_curve with pinned host buffers: the
         points go host->device and the curve device->host every step
  roofline  the flux sweep (the dominant kernel): 16 FLOP per element
         (5 for mu, 8 for the Claret Horner form, 2 for mu*flux*I,
         1 accumulate) over its CUDA-event time, against the FMA peak
         of the sweep's arithmetic measured live (lcg_measure_fp32_peak,
         or lcg_measure_fp64_peak with --precision fp64)
  cpu_baseline  lcurve_re's own CPU path (oracle/_ref, Release flags,
         OpenMP on all host cores) on whole light curves of the workload
         (grids rebuilt each call) for about 20 s; its curve of the exact
         model also gives the benched curve's error ("parity")

--impl reference times that reference CPU path alone (rank 0).
Multi-GPU: one process per GPU; each rank evaluates its own light curves
(independent replicas, no collective on the data path); value = all ranks'
curves / the slowest rank's time.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lcurve_re_b200 import abi  # noqa: E402  (ctypes declarations only)

METRIC = "light curves/s"
FLOP_PER_ELEMENT = 16
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="wd_dm_large",
                    choices=("wd_dm_large", "wd_dm_small", "tiny_star", "mcmc_batch",
                             "surrogate_da", "cv_disc", "mlp_train"))
    ap.add_argument("--batch-models", type=int, default=256,
                    help="models per step of mcmc_batch (256 is the benchmark)")
    ap.add_argument("--batch-variant", choices=("geometry", "brightness"), default="geometry",
                    help="mcmc_batch: q alternates between steps (every grid rebuilt), or only "
                         "T1/T2 alternate (grids reused, continuum and flux recomputed)")
    ap.add_argument("--train-curves", type=int, default=200000)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--chains", type=int, default=512)
    ap.add_argument("--mcmc-steps", type=int, default=2000)
    ap.add_argument("--burn", type=int, default=400)
    ap.add_argument("--compact", type=int, default=64,
                    help="surrogate_da: delayed acceptance's exact evaluations through a "
                         "batch of this many slots on a second engine context (0: the "
                         "whole-chain batch)")
    ap.add_argument("--burn-fixed", type=int, default=0,
                    help="surrogate_da: plain Metropolis steps after the adaptive burn-in, "
                         "with its final proposal kept (no further adaptation), before the "
                         "local draws")
    ap.add_argument("--stm-inner", type=int, nargs="*", default=[20, 50],
                    help="surrogate_da: inner steps per exact decision of each surrogate-"
                         "transition run (none: skip them)")
    ap.add_argument("--stm-layouts", nargs="*", choices=("whole", "halves"),
                    default=["whole"],
                    help="surrogate_da: surrogate-transition runs over all chains at once, "
                         "or in two halves whose exact evaluations overlap the other half's "
                         "inner steps")
    ap.add_argument("--stm-anchor", nargs="*", choices=("none", "start"),
                    default=["none", "start"],
                    help="surrogate_da: the surrogate-transition runs' approximation: the "
                         "network's own chi**2, or anchored at each chain's exact curve at its "
                         "starting state (fixed for the run)")
    ap.add_argument("--stm-steps", type=int, default=0,
                    help="surrogate_da: exact decisions per chain of a surrogate-transition "
                         "run (0: a tenth of --mcmc-steps)")
    ap.add_argument("--ncoef", type=int, default=64)
    ap.add_argument("--local-curves", type=int, default=262144)
    ap.add_argument("--refine-epochs", type=int, default=600)
    ap.add_argument("--da-min-accept", type=float, default=0.02,
                    help="surrogate_da: least pilot acceptance of a delayed-acceptance scale")
    ap.add_argument("--da-scales", type=float, nargs="+", default=[1.0, 1.5, 2.0, 2.5],
                    help="surrogate_da: multiples of the plain step scale tried by the "
                         "delayed-acceptance pilot runs")
    ap.add_argument("--adapt-rounds", type=int, default=2,
                    help="surrogate_da: adaptive burn-in rounds refitting the proposal's map")
    ap.add_argument("--local-widen", type=float, default=2.0)
    ap.add_argument("--tune-steps", type=int, default=200,
                    help="surrogate_da: plain Metropolis steps per pilot run of the proposal scale")
    ap.add_argument("--burn-tuned", type=int, default=2000,
                    help="surrogate_da: plain Metropolis steps per adaptive burn-in round")
    ap.add_argument("--is-rounds", type=int, default=8,
                    help="surrogate_da: rounds of adaptive importance sampling of the posterior")
    ap.add_argument("--is-pool", type=int, default=65536,
                    help="surrogate_da: exact curves per importance-sampling round")
    ap.add_argument("--is-target", type=float, default=20000.0,
                    help="surrogate_da: effective size at which the importance sampling stops")
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--ref-cuda-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="report the named workload alone (no batch and surrogate sub-objects)")
    ap.add_argument("--eclipse-warp", type=int, default=0,
                    help="Roche eclipse candidates up to which one warp bisects each face "
                         "(0 automatic, -1 never)")
    return ap.parse_args()


def workload(name):
    from lcurve_re_b200 import workloads as W
    if name == "wd_dm_large":
        m, d = W.wd_dm_large()
        desc = "wd_dm_large: WD+dM q=0.25 i=86 r1=0.015 r2=0.20, nlat 200/800, 5000 pts x ndiv 5"
    elif name == "wd_dm_small":
        m, d = W.wd_dm_small()
        desc = "wd_dm_small: WD+dM q=0.25 i=86 r1=0.015 r2=0.20, nlat 40/80, 500 pts"
    elif name == "cv_disc":
        m = W.cv_disc(nlat1f=100, nlat2f=200, nrad=60, nspot=100)
        d = W.data(2000)
        desc = ("cv_disc: WD + Roche-filling donor q=0.15 i=84, opaque flared disc 0.03-0.3 "
                "(nrad 60) with its rim, bright spot (nspot 100), nlat 100/200, 2000 pts")
    else:
        m, d = W.tiny_star()
        desc = "tiny_star: r1=0.005 q=0.2 i=87, nlat 400/200, 10000 pts in +-0.03"
    return m, d, desc


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


# ---- clocks ---------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---- CPU baseline: the reference's own CPU path ------------------------------------
class RefTimer:
    """Times lcurve_re's CPU light_curve_comp (oracle/_ref Release build, OpenMP
    over all host cores; the C port in oracle/ if that build is absent) on
    whole light curves: every timed call evaluates all points of the
    workload with the geometry perturbed (q x (1 + 1e-13 k)), so that the
    reference's grid cache (light_curve_comp.cpp:156-170) misses and the
    grids, eclipses, continuum and FlatGrids are rebuilt, as the GPU arm's
    FLAG_NO_CACHE does. Nothing is extrapolated."""

    def __init__(self, model, data, path=None):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as OL
        self.kind = "reference"
        if path is not None:
            self.lib = OL.Reference(path)
        elif os.path.exists(OL.REF_RELEASE_SO):
            self.lib = OL.Reference(OL.REF_RELEASE_SO)
        else:
            self.kind = "port"
            self.lib = OL.Oracle()
        self.model = model
        self.data = data
        self.n = data.shape[0]
        self.k = 0

    def exact_curve(self):
        """The unperturbed model's curve, chi**2 and scale factors (untimed)."""
        st, err, calc, sfac, sc = self.lib.light_curve(self.model, self.data)
        if st:
            raise RuntimeError(err)
        return calc, sc[abi.OUT_CHISQ], sfac

    def curve(self):
        """One timed whole light curve with the grids rebuilt: seconds."""
        self.k += 1
        m = self.model.copy()
        m["q"] = m["q"] * (1 + 1e-13 * self.k)
        t = time.perf_counter()
        st, err, *_ = self.lib.light_curve(m, self.data)
        dt = time.perf_counter() - t
        if st:
            raise RuntimeError(err)
        return dt

    def describe(self, reps, t_curve):
        return ("whole light curves (%d points each, grids rebuilt every call), %d timed calls; "
                "one light curve = %.3f s" % (self.n, reps, t_curve))


def cpu_reference_rate(model, data, budget_s=20.0, gpu_calc=None, gpu_chisq=None):
    """The reference CPU path on whole light curves of the workload: one
    untimed call on the exact model (its curve checks the GPU's benched curve
    when gpu_calc is given), then timed calls until budget_s is spent (at
    least two)."""
    r = RefTimer(model, data)
    calc, chisq, _ = r.exact_curve()
    ts = []
    while len(ts) < 2 or (sum(ts) < budget_s and len(ts) < 50):
        ts.append(r.curve())
    t_curve = float(np.mean(ts))
    out = {"value": 1.0 / t_curve, "unit": METRIC, "cores": os.cpu_count(), "kind": r.kind,
           "sample": r.describe(len(ts), t_curve)}
    if gpu_calc is not None:
        out["parity"] = {
            "checker": "this reference build's curve of the same model and points",
            "max_rel_flux_error": float(np.max(np.abs(gpu_calc - calc) / np.abs(calc))),
            "chi2_rel_error": (abs(gpu_chisq - chisq) / abs(chisq)) if gpu_chisq else None}
    return out


def run_reference(args):
    rank, _, world = rank_info()
    if rank != 0:
        return None
    model, data, desc = workload(args.workload)
    r = RefTimer(model, data)
    cpu_calc = r.exact_curve()[0]
    for _ in range(args.warmup):
        r.curve()
    ts = [r.curve() for _ in range(args.steps)]
    mean_t = float(np.mean(ts))
    v = 1.0 / mean_t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc, "precision": "fp64 (reference CPU)"},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": os.cpu_count(), "kind": r.kind,
                             "sample": r.describe(args.steps, mean_t)},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "wd_dm_large" and r.kind == "reference":
        rc = reference_cuda_rate(args, cpu_calc)
        if rc is not None:
            line["reference_cuda"] = rc
    return line


REF_CUDA_SO = os.path.join(ROOT, "oracle", "_ref", "liblcurve_ref_cuda.so")


def reference_cuda_child(args):
    """Runs in a child process (the reference's GPU build and its CPU build
    define the same symbols): times whole light curves of the workload
    through the reference's own CUDA path (oracle/_ref/liblcurve_ref_cuda.so:
    its CPU sources with HAVE_CUDA plus comp_light_cuda.cu and
    set_star_grid_cuda.cu for sm_100a, switched on by LCURVE_CUDA=1 and
    LCURVE_CUDA_GRID=1 as its users do), and writes the unperturbed curve
    for the parent's check."""
    model, data, _ = workload(args.workload)
    r = RefTimer(model, data, path=REF_CUDA_SO)
    calc, chisq, _ = r.exact_curve()
    np.save(args.ref_cuda_child, calc)
    for _ in range(2):
        r.curve()
    ts = []
    while len(ts) < 3 or (sum(ts) < 15.0 and len(ts) < 50):
        ts.append(r.curve())
    print(json.dumps({"t_curve": float(np.mean(ts)), "calls": len(ts), "chisq": chisq}),
          flush=True)


def reference_cuda_rate(args, cpu_calc):
    """The reference's own GPU path on the same workload, timed in a child
    process on whole light curves (an informative secondary baseline: the
    reference arm's value stays its CPU path); None when that build is
    absent."""
    if not os.path.exists(REF_CUDA_SO):
        return None
    import subprocess
    import tempfile
    env = dict(os.environ, LCURVE_CUDA="1", LCURVE_CUDA_GRID="1")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "calc.npy")
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--workload", args.workload,
                            "--ref-cuda-child", out], env=env, capture_output=True, text=True,
                           timeout=600)
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not lines:
            return {"unavailable": "reference CUDA build failed: %s" % r.stderr.strip()[-300:]}
        res = json.loads(lines[-1])
        calc = np.load(out)
    v = 1.0 / res["t_curve"]
    return {"value": v, "unit": METRIC, "kind": "reference GPU path (comp_light_cuda.cu, "
                                                "set_star_grid_cuda.cu, sm_100a)",
            "precision": "the reference's CUDA default (FP32 sweep and grid)",
            "sample": "whole light curves, grids rebuilt every call, %d timed calls; one light "
                      "curve = %.3f s" % (res["calls"], res["t_curve"]),
            "max_rel_flux_error_vs_its_cpu_path": float(np.max(np.abs(calc - cpu_calc) /
                                                                np.abs(cpu_calc)))}


# ---- our arm -------------------------------------------------------------------------
def run_ours(args, dist=None):
    import ctypes as C
    import torch
    from lcurve_re_b200.replicas import max_over_ranks
    rank, local, world = rank_info()
    from lcurve_re_b200 import abi
    from lcurve_re_b200 import workloads as W
    from lcurve_re_b200.engine import Engine

    model, data, desc = workload(args.workload)
    eng = Engine(device=local, precision=args.precision, eclipse_warp=args.eclipse_warp)
    lib, ctx = eng.lib, eng.ctx
    # synthetic noisy data from the model itself (seeded per rank)
    calc0 = eng.light_curve_comp(model, data, scale=False, rdata=False, diagnostics=False)[0]
    data = W.add_noise(data, calc0, seed=1234 + rank)
    n = data.shape[0]
    mc = model.to_c()
    flags = abi.FLAG_SCALE | abi.FLAG_RDATA | abi.FLAG_NO_CACHE
    sfac = np.ones(5)
    scal = np.zeros(abi.NOUT)
    dptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    fp64 = args.precision == "fp64"
    peak = eng.fp64_peak_tflops() if fp64 else eng.fp32_peak_tflops()

    ext = torch.cuda.ExternalStream(eng.stream_ptr)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def check(st):
        if st != abi.OK:
            raise RuntimeError(lib.lcg_last_error(ctx).decode())

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # ---- device-resident value
    check(lib.lcg_set_data(ctx, data.ctypes.data, n))
    for _ in range(args.warmup):
        check(lib.lcg_light_curve_resident(ctx, C.byref(mc), flags, dptr(sfac), None, dptr(scal)))
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    eng.set_profiling(True)
    eng.stage_times(reset=True)
    eng.flux_elements(reset=True)
    barrier()
    lib.lcg_kernel_launches(1)
    clocks = Clocks(local)
    clocks.start()
    with torch.cuda.stream(ext):
        for k in range(args.steps):
            flush.fill_(float(k))  # L2 flush, outside the timed span
            e0[k].record(ext)
            check(lib.lcg_light_curve_resident(ctx, C.byref(mc), flags, dptr(sfac), None,
                                               dptr(scal)))
            e1[k].record(ext)
    barrier()
    launches = int(lib.lcg_kernel_launches(1))
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in zip(e0, e1))
    st = eng.stage_times(reset=True)
    elements = eng.flux_elements(reset=True)
    eng.set_profiling(False)
    total_ms = max_over_ranks(total_ms, dist, device="cuda")
    value = world * args.steps / (total_ms / 1e3)
    flux_ms, flux_n = st["flux"]
    achieved = elements * FLOP_PER_ELEMENT / (flux_ms / 1e3) / 1e12 if flux_ms > 0 else None

    # ---- end to end through lcg_light_curve with pinned host buffers
    hdata = torch.empty(n * data.itemsize, dtype=torch.uint8, pin_memory=True).numpy()
    hdata[:] = data.view(np.uint8).reshape(-1)
    hcalc = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    ke = min(args.e2e_steps, args.steps)
    for _ in range(2):
        check(lib.lcg_light_curve(ctx, C.byref(mc), hdata.ctypes.data, n, flags, dptr(sfac),
                                  dptr(hcalc), dptr(scal)))
    f0 = [torch.cuda.Event(enable_timing=True) for _ in range(ke)]
    f1 = [torch.cuda.Event(enable_timing=True) for _ in range(ke)]
    barrier()
    with torch.cuda.stream(ext):
        for k in range(ke):
            flush.fill_(float(k))
            f0[k].record(ext)
            check(lib.lcg_light_curve(ctx, C.byref(mc), hdata.ctypes.data, n, flags, dptr(sfac),
                                      dptr(hcalc), dptr(scal)))
            f1[k].record(ext)
    barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in zip(f0, f1))
    e2e_value = world * ke / (max_over_ranks(e2e_ms, dist, device="cuda") / 1e3)
    h2d = n * data.itemsize + (n + 1) * 8 + 5 * 8
    d2h = n * 8 + 5 * 8 + 3 * 8 + 8

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_rate(model, data, gpu_calc=hcalc.copy(),
                                     gpu_chisq=float(scal[abi.OUT_CHISQ]))
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": str(ex)}

    traffic = None
    prof = os.path.join(ROOT, "profiles", "flux_fast_wd_dm_large.txt")
    if os.path.exists(prof) and args.workload == "wd_dm_large" and args.precision == "mixed":
        for line in open(prof):
            if line.startswith("dram_bytes_per_light_curve:"):
                traffic = float(line.split(":")[1]) / 2  # two sweeps per curve

    nf1 = eng.face_count(model, 0)
    nf2 = eng.face_count(model, 1)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 elements + f64 accumulation" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded model + Gaussian noise sigma=1.5e-3)",
        "config": {"workload": desc, "faces": [nf1, nf2], "sub_phases": int(data["ndiv"].sum()),
                   "precision": args.precision, "grids": "rebuilt every step",
                   "l2": "flushed by a 256 MiB write between timed steps (untimed)",
                   "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "fp64" if fp64 else "fp32",
                     "kernel": "k_flux64" if fp64 else "k_flux_fast",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": ("measured live: DFMA-chain kernel (lcg_measure_fp64_peak)"
                                     if fp64 else
                                     "measured live: FFMA-chain kernel (lcg_measure_fp32_peak)"),
                     "flop_per_element": FLOP_PER_ELEMENT,
                     "flux_ms_per_step": flux_ms / args.steps,
                     "flux_launches_per_step": flux_n / args.steps},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": ke},
        "gpu_launches": launches,
        "stage_ms_per_step": {k: v[0] / args.steps for k, v in st.items()},
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    eng.close()
    return line if rank == 0 else None


# ---- batched workload: 256 models per step -------------------------------------------
BATCH_DESC = ("mcmc_batch: 256 models around wd_dm_small (q~N(0.25,0.02), i~N(86,0.5), r1,r2 "
              "x N(1,0.05), T1,T2 x N(1,0.03); nlat2f ~ U{60..400}, nlat1f = nlat2f/2), "
              "2000 points")


BATCH_GRIDS = {
    "geometry": "every model's grids rebuilt every step (q alternates by 1e-4)",
    "brightness": "grids reused, continuum and flux recomputed every step (T1, T2 alternate by "
                  "1e-4; geometry unchanged)",
}


def batch_workload(nmodels=256, variant="geometry"):
    """The models, a second set with every q (variant "geometry": alternating
    steps rebuild every grid, as an MCMC step does) or every T1 and T2
    (variant "brightness": the grids stay, the continuum changes) scaled by
    1 + 1e-4, and noisy data from the first model's curve."""
    from lcurve_re_b200 import workloads as W
    ms, d = W.mcmc_batch(nmodels)
    alt = []
    fq, ft = (1 + 1e-4, 1.0) if variant == "geometry" else (1.0, 1 + 1e-4)
    for m in ms:
        c = m.to_c()
        alt.append(W.model(q=c.q * fq, iangle=c.iangle, r1=c.r1, r2=c.r2, t1=c.t1 * ft,
                           t2=c.t2 * ft, nlat1f=c.nlat1f, nlat2f=c.nlat2f))
    return ms, alt, d


class RefBatch:
    """The reference CPU path (oracle/_ref Release build, OpenMP on all host
    cores; the C port if that build is absent) over every model of a batch,
    one whole light curve per model. Consecutive models differ in geometry,
    so each call rebuilds its grids. With warm (the same models with only T1
    and T2 changed), each timed call follows an untimed call on its warm
    partner, so the reference's own per-thread grid cache
    (light_curve_comp.cpp:156-170) skips the grids, as the engine does."""

    def __init__(self, models, data, warm=None):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as OL
        from lcurve_re_b200 import workloads as W
        self.kind = "reference"
        if os.path.exists(OL.REF_RELEASE_SO):
            self.lib = OL.Reference(OL.REF_RELEASE_SO)
        else:
            self.kind = "port"
            self.lib = OL.Oracle()
        # models whose nlat makes the reference's grid build write past its
        # own vector cannot run in this process: the rate is over the others
        keep = [i for i, m in enumerate(models) if W.reference_safe(m)]
        self.left_out = len(models) - len(keep)
        self.models = [models[i] for i in keep]
        self.warm = [warm[i] for i in keep] if warm is not None else None
        self.data = data

    def batch(self):
        """Seconds for one pass over the whole batch (timed calls only)."""
        t_used = 0.0
        for i, m in enumerate(self.models):
            if self.warm is not None:
                self.lib.light_curve(self.warm[i], self.data)
            t = time.perf_counter()
            st, err, *_ = self.lib.light_curve(m, self.data)
            t_used += time.perf_counter() - t
            if st:
                raise RuntimeError(err)
        return t_used

    def describe(self, passes, t_batch):
        return ("%d models of the batch (%d left out: their nlat makes the reference's ring "
                "tiling write past its Point vector), one whole %d-point light curve each, %s; "
                "%d pass(es); %.2f s per pass" % (
                    len(self.models), self.left_out, self.data.shape[0],
                    "cold grids" if self.warm is None else
                    "grids from the reference's cache (only T1/T2 changed)" if
                    self.kind == "reference" else "grids rebuilt (the port has no cache)",
                    passes, t_batch))


def cpu_batch_rate(models, data, warm=None, passes=1):
    r = RefBatch(models, data, warm)
    ts = [r.batch() for _ in range(passes)]
    t = float(np.mean(ts))
    return {"value": len(r.models) / t, "unit": METRIC, "cores": os.cpu_count(), "kind": r.kind,
            "sample": r.describe(passes, t)}


def run_batch(args, dist=None):
    import ctypes as C
    import torch
    from lcurve_re_b200.replicas import max_over_ranks
    rank, local, world = rank_info()
    from lcurve_re_b200 import abi
    from lcurve_re_b200 import workloads as W
    from lcurve_re_b200.engine import Engine

    ms, alt, data = batch_workload(args.batch_models, args.batch_variant)
    eng = Engine(device=local, precision="mixed")
    lib, ctx = eng.lib, eng.ctx
    calc0 = eng.light_curve_comp(ms[0], data, scale=False, rdata=False, diagnostics=False)[0]
    data = W.add_noise(data, calc0, seed=1234 + rank)
    n, nm = data.shape[0], len(ms)
    A = (abi.LcgModel * nm)(*[m.to_c() for m in ms])
    B = (abi.LcgModel * nm)(*[m.to_c() for m in alt])
    flags = abi.FLAG_SCALE | abi.FLAG_RDATA
    sfac = np.ones(5 * nm)
    chisq = np.zeros(nm)
    wnok = np.zeros(nm)
    status = np.zeros(nm, dtype=np.int32)
    dptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    i32 = status.ctypes.data_as(C.POINTER(C.c_int32))
    peak = eng.fp32_peak_tflops()
    ext = torch.cuda.ExternalStream(eng.stream_ptr)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def check(st):
        if st != abi.OK:
            raise RuntimeError(lib.lcg_last_error(ctx).decode())
        if np.any(status != 0):
            raise RuntimeError("model status %s" % np.unique(status))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # one running counter over every call, so each call's models differ from
    # the previous call's (the engine skips models identical to the last call's)
    calls = [0]

    def models_now():
        calls[0] += 1
        return A if calls[0] % 2 else B

    def step(k, calc_out=None):
        check(lib.lcg_light_curve_batch_resident(ctx, models_now(), nm, flags, dptr(sfac),
                                                 calc_out, dptr(chisq), dptr(wnok), i32))

    # ---- device-resident value (CUDA graph path)
    check(lib.lcg_set_data(ctx, data.ctypes.data, n))
    for k in range(args.warmup):
        step(k)
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    lib.lcg_kernel_launches(1)
    clocks = Clocks(local)
    clocks.start()
    with torch.cuda.stream(ext):
        for k in range(args.steps):
            flush.fill_(float(k))
            e0[k].record(ext)
            step(k)
            e1[k].record(ext)
    barrier()
    launches = int(lib.lcg_kernel_launches(1))
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in zip(e0, e1))
    total_ms = max_over_ranks(total_ms, dist, device="cuda")
    value = world * nm * args.steps / (total_ms / 1e3)

    # ---- stage breakdown and the flux roofline (profiled, untimed)
    eng.set_profiling(True)
    eng.stage_times(reset=True)
    eng.flux_elements(reset=True)
    kp = 4
    with torch.cuda.stream(ext):
        for k in range(kp):
            flush.fill_(float(k))
            step(k)
    barrier()
    st = eng.stage_times(reset=True)
    elements = eng.flux_elements(reset=True)
    eng.set_profiling(False)
    flux_ms, flux_n = st["flux"]
    achieved = elements * FLOP_PER_ELEMENT / (flux_ms / 1e3) / 1e12 if flux_ms > 0 else None

    # ---- end to end: lcg_light_curve_batch with pinned host data and curves
    hdata = torch.empty(n * data.itemsize, dtype=torch.uint8, pin_memory=True).numpy()
    hdata[:] = data.view(np.uint8).reshape(-1)
    hcalc = torch.empty(nm * n, dtype=torch.float64, pin_memory=True).numpy()
    ke = min(args.e2e_steps, args.steps)

    def step_e2e(k):
        check(lib.lcg_light_curve_batch(ctx, models_now(), nm, hdata.ctypes.data, n,
                                        flags, dptr(sfac), dptr(hcalc), dptr(chisq), dptr(wnok),
                                        i32))
    for k in range(2):
        step_e2e(k)
    f0 = [torch.cuda.Event(enable_timing=True) for _ in range(ke)]
    f1 = [torch.cuda.Event(enable_timing=True) for _ in range(ke)]
    barrier()
    with torch.cuda.stream(ext):
        for k in range(ke):
            flush.fill_(float(k))
            f0[k].record(ext)
            step_e2e(k)
            f1[k].record(ext)
    barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in zip(f0, f1))
    e2e_value = world * nm * ke / (max_over_ranks(e2e_ms, dist, device="cuda") / 1e3)
    h2d = n * data.itemsize + (n + 1) * 8 + nm * C.sizeof(abi.LcgModel)
    d2h = nm * (n * 8 + 5 * 8 + 3 * 8 + 8)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_batch_rate(ms, data, warm=alt if args.batch_variant == "brightness"
                                 else None)
        except Exception as ex:
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": str(ex)}
    faces = [eng.face_count(m, 0) + eng.face_count(m, 1) for m in ms]
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 elements + f64 accumulation",
        "data": "synthetic (seeded models + Gaussian noise sigma=1.5e-3)",
        "config": {"workload": BATCH_DESC, "models_per_step": nm, "faces_per_step": int(sum(faces)),
                   "points": n, "precision": "mixed",
                   "grids": BATCH_GRIDS[args.batch_variant],
                   "l2": "flushed by a 256 MiB write between timed steps (untimed)",
                   "graph": "one CUDA graph per step", "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "fp32", "kernel": "k_flux_batch", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "peak_source": "measured live: FFMA-chain kernel (lcg_measure_fp32_peak)",
                     "flop_per_element": FLOP_PER_ELEMENT,
                     "flux_ms_per_step": flux_ms / kp},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": ke},
        "gpu_launches": launches,
        "stage_ms_per_step": {k: v[0] / kp for k, v in st.items()},
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    eng.close()
    return line if rank == 0 else None


def run_reference_batch(args):
    rank, _, world = rank_info()
    if rank != 0:
        return None
    from lcurve_re_b200 import workloads as W
    ms, alt, data = batch_workload(variant=args.batch_variant)
    warm = alt if args.batch_variant == "brightness" else None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as OL
    calc0 = OL.Oracle().light_curve(ms[0], data, scale=False, rdata=False)[2]
    data = W.add_noise(data, calc0, seed=1234)
    r = RefBatch(ms, data, warm)
    for _ in range(args.warmup):
        r.batch()
    ts = [r.batch() for _ in range(args.steps)]
    t = float(np.mean(ts))
    v = len(r.models) / t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": BATCH_DESC, "precision": "fp64 (reference CPU)",
                                            "grids": BATCH_GRIDS[args.batch_variant]},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": os.cpu_count(), "kind": r.kind,
                             "sample": r.describe(args.steps, t)},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


# ---- learned surrogate + delayed acceptance ---------------------------------------------
def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def _bf16_peak():
    p = _peaks()
    for k in ("bf16_tflops", "bf16_dense_tflops"):
        if isinstance(p.get(k), (int, float)):
            return float(p[k]), "measured (MEASURED_PEAKS.json %s)" % k
    return 1590.0, "fallback 1.59 PFLOP/s"


def run_surrogate(args):
    """cfg4: the surrogate trained on engine curves over the prior box, then
    plain vs delayed-acceptance Metropolis (same start states, same draws) on
    wd_dm_small data; effective samples per second of sampling.

    Start states: a first adaptive burn-in locates the posterior; adaptive
    importance sampling of exact engine curves (the box-uniform training set,
    then Gaussian pools around the running weighted estimate; each row
    weighted by its exact likelihood over the density of the mixture of the
    pools) gives the posterior's sample, and the chains start from a resample
    of it, then adaptive burn-in rounds with the final proposal, so both
    samplers begin at (close to) the stationary distribution and their means
    can be compared against their Monte Carlo errors. Proposal: a random walk
    in coordinates that straighten the posterior's curved ridge
    (sampler.TriangularWalk), refitted over adaptive burn-in rounds; plain
    Metropolis' step scale by acceptance nearest 0.234, delayed acceptance's
    boldness by pilot runs (largest squared jump per second). The network is
    refined on engine curves drawn along the ridge through the same map.

    value: bulk ESS (rank-normalised multi-chain ESS over split chains,
    minimum over parameters) per second of delayed-acceptance sampling; the
    reference's Geyer estimator and a between-chain estimate are reported
    beside it."""
    import torch
    rank, local, world = rank_info()
    from lcurve_re_b200 import surrogate as S
    from lcurve_re_b200 import workloads as W
    from lcurve_re_b200.engine import Engine
    from lcurve_re_b200.sampler import (CompactExact, DeviceTransitions, ExactChi2,
                                        TriangularWalk, delayed_acceptance, mean_shift,
                                        metropolis, shift_verdict, summary,
                                        surrogate_transitions)

    eng = Engine(device=local, precision="mixed")
    clocks = Clocks(local)
    clocks.start()
    # training curves from the batched engine
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    theta, curves = S.training_set(eng, args.train_curves, seed=100 + rank, batch=2048)
    t_gen = time.perf_counter() - t0
    sur = S.Surrogate(ncoef=args.ncoef, batch=4096, seed=rank)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    losses = sur.fit(theta, curves, epochs=args.epochs)
    ev1.record()
    torch.cuda.synchronize()
    t_fit = ev0.elapsed_time(ev1) / 1e3
    nsteps_fit = args.epochs * (args.train_curves // sur.net.B)
    train_flop = nsteps_fit * sur.net.B * sur.net.flops_per_sample(train=True)
    # held-out accuracy
    th_h, cu_h = S.training_set(eng, 2048, seed=999, batch=2048)
    pred = sur.curves(th_h)
    rel_err = float(np.sqrt(np.mean((pred - cu_h) ** 2)))
    # data: wd_dm_small physics at the even points of the grid
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    calc = eng.light_curve_comp(S.ModelFactory()(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                                scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)[0]
    data = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 1234 + rank)
    exact = ExactChi2(eng, data)
    sur_chi = S.SurrogateChi2(sur, data, idx)
    rng = np.random.default_rng(7 + rank)
    scale0 = (S.BOX[:, 1] - S.BOX[:, 0]) * 1e-3
    theta0 = truth + rng.standard_normal((args.chains, 9)) * scale0
    # adaptive burn-in with plain Metropolis in two rounds, each adapting the
    # proposal to 2.38^2 / d times the covariance of its second half (pooled
    # over the chains): it locates the posterior for the local draws
    cov = np.diag(scale0 ** 2)
    for k in range(2):
        ch, theta0, _, acc_b, _ = metropolis(exact, theta0, cov, args.burn // 2, seed=11 + k)
        samp = ch[ch.shape[0] // 2:].reshape(-1, 9)
        cov = np.cov(samp.T) * 2.38 ** 2 / 9 + np.diag((scale0 * 1e-3) ** 2)
    del ch
    if args.burn_fixed > 0:
        chf, theta0, _, _, _ = metropolis(exact, theta0, cov, args.burn_fixed, seed=13)
        samp = chf[chf.shape[0] // 2:].reshape(-1, 9)
        del chf
    # the posterior by adaptive importance sampling of exact engine curves
    # (surrogate.adaptive_posterior; the box-uniform training set is the first
    # pool, the burn-in's spread places the first Gaussian one)
    t0 = time.perf_counter()
    chi_box = S.curves_chi2(curves, data, idx)
    del curves

    def exact_chi2(th):
        _, cu = S.training_set(eng, 0, theta=th, batch=2048)
        return S.curves_chi2(cu, data, idx)
    pools, chi_pool, mu_k, cov_k, ess_rounds = S.adaptive_posterior(
        exact_chi2, [(theta, S.log_uniform_box())], chi_box, samp.mean(0), np.cov(samp.T),
        rounds=args.is_rounds, pool=args.is_pool, target=args.is_target,
        widen0=args.local_widen, seed=19 + rank)
    theta0, mu_is, cov_is, ess_is = S.posterior_resample(pools, chi_pool, args.chains,
                                                         seed=17 + rank)
    t_sir = time.perf_counter() - t0
    # proposal: the posterior is a curved ridge (iangle, r1, r2 and q follow
    # one another along a curve: quadratic terms predict them 5-7x better than
    # linear ones), so a random walk with one covariance moves at the ridge's
    # local width. sampler.TriangularWalk walks in coordinates that straighten
    # it (a volume-preserving quadratic map, so the proposal stays symmetric):
    # fitted to the importance sample first, then refitted on the second half
    # of each adaptive burn-in round of plain Metropolis; before every round
    # and the comparison, pilot runs pick the step scale whose acceptance is
    # nearest 0.234
    exact = ExactChi2(eng, data)
    tw = TriangularWalk(S.posterior_resample(pools, chi_pool, 65536, seed=31 + rank)[0])
    tuning = []

    def tune(walk, start):
        accs = [(f, metropolis(exact, start, None, args.tune_steps, seed=23, record=False,
                               propose=walk.with_scale(f))[3])
                for f in (1.0, 0.7, 0.5, 0.35, 0.25)]
        tuning.append(accs)
        return walk.with_scale(min(accs, key=lambda t: abs(t[1] - 0.234))[0])
    tw = tune(tw, theta0)
    for r in range(args.adapt_rounds):
        ch_b, theta0, _, _, _ = metropolis(exact, theta0, None, args.burn_tuned, seed=29 + r,
                                           propose=tw)
        tw = tune(TriangularWalk(ch_b[ch_b.shape[0] // 2:].reshape(-1, 9)), theta0)
        del ch_b
    f_best = tw.scale
    # refinement: the same network trained again on engine curves drawn along
    # the posterior's ridge (Gaussian in the walk's straightened coordinates,
    # local_widen x its spread there, mapped back, inside the box); its error
    # is measured on held-out draws of the same kind
    t0 = time.perf_counter()
    th_loc = tw.draws(args.local_curves, widen=args.local_widen, seed=5 + rank,
                      box_check=S.in_box)
    _, cu_loc = S.training_set(eng, 0, theta=th_loc, batch=2048)
    sur_loc = S.Surrogate(ncoef=args.ncoef, batch=4096, seed=rank + 1)
    losses_loc = sur_loc.fit(th_loc, cu_loc, epochs=args.refine_epochs)
    t_ref = time.perf_counter() - t0
    del cu_loc
    th_lh = tw.draws(2048, widen=args.local_widen, seed=77 + rank, box_check=S.in_box)
    _, cu_lh = S.training_set(eng, 0, theta=th_lh, batch=2048)
    loc_err = float(np.sqrt(np.mean((sur_loc.curves(th_lh) - cu_lh) ** 2)))
    glob_err_loc = float(np.sqrt(np.mean((sur.curves(th_lh) - cu_lh) ** 2)))
    # the training curves above went through the same engine on their own
    # phase grid: the samplers' evaluator binds the data again
    exact = ExactChi2(eng, data)
    sur_loc_chi = S.SurrogateChi2(sur_loc, data, idx)
    # inference throughput of the network alone (the DA screening pass)
    xin = torch.rand(args.chains, 9, device="cuda") * 2 - 1
    for _ in range(3):
        sur.net.forward(xin)
    ev0.record()
    for _ in range(50):
        sur.net.forward(xin)
    ev1.record()
    torch.cuda.synchronize()
    t_inf = ev0.elapsed_time(ev1) / 1e3 / 50
    lib = eng.lib
    lib.lcg_kernel_launches(1)
    e_plain0 = exact.evals
    chp, _, _, accp, wall_p = metropolis(exact, theta0, None, args.mcmc_steps, seed=21,
                                         propose=tw)
    launches_plain = int(lib.lcg_kernel_launches(1))
    n_plain = exact.evals - e_plain0
    eng_c = Engine(device=local, precision="mixed") if args.compact > 0 else None
    exact_g = ExactChi2(eng, data, curves=True)
    comp_g = CompactExact(eng_c, data, k=args.compact) if eng_c else None
    # delayed acceptance can afford bolder steps, since the surrogate screens
    # them: short pilot runs pick the multiple of the plain step scale with
    # the largest expected squared jump (in the walk's whitened coordinates)
    # per second of sampling, among those whose acceptance stays at or above
    # da_min_accept (rarer, larger jumps score well on the squared jump while
    # the chains stick between them)
    da_pilots = []
    for k in args.da_scales:
        walk = tw.with_scale(tw.scale * k)
        ex_p = ExactChi2(eng, data, curves=True)
        comp_p = CompactExact(eng_c, data, k=args.compact) if eng_c else None
        cpl, _, _, acc_k, wall_k, _ = delayed_acceptance(ex_p, sur_loc_chi, theta0, None,
                                                         args.tune_steps, seed=27,
                                                         compact=comp_p, propose=walk)
        u = tw.forward(cpl.reshape(-1, 9)).reshape(cpl.shape) @ np.linalg.inv(tw.chol.T)
        esjd = float(np.mean(np.sum(np.diff(u, axis=0) ** 2, axis=2)))
        # the slowest parameter's squared jump over its variance (1 - its lag-1
        # autocorrelation, x2): reported beside the choice
        per = np.mean(np.diff(cpl, axis=0) ** 2, axis=(0, 1)) / cpl.reshape(-1, 9).var(0)
        da_pilots.append((k, acc_k, esjd / wall_k, float(per.min()) / wall_k))
    ok = [t for t in da_pilots if t[1] >= args.da_min_accept] or da_pilots[:1]
    da_scale = max(ok, key=lambda t: t[2])[0]
    walk_da = tw.with_scale(tw.scale * da_scale)
    chg, _, _, accg, wall_g, stg = delayed_acceptance(exact_g, sur_chi, theta0, None,
                                                       args.mcmc_steps, seed=21, compact=comp_g,
                                                       propose=walk_da)
    exact2 = ExactChi2(eng, data, curves=True)
    comp2 = CompactExact(eng_c, data, k=args.compact) if eng_c else None
    lib.lcg_kernel_launches(1)
    chd, _, _, accd, wall_d, st = delayed_acceptance(exact2, sur_loc_chi, theta0, None,
                                                      args.mcmc_steps, seed=21, compact=comp2,
                                                      propose=walk_da)
    launches_da = int(lib.lcg_kernel_launches(1)) + getattr(sur_loc_chi, "graph_launches", 0)
    # surrogate transitions: per exact decision, a run of inner Metropolis
    # steps on the refined network's own posterior, on the device (one CUDA
    # graph per run), with the plain step scale; all chains at once, or in
    # two halves, one half's exact evaluations overlapping the other's inner
    # steps
    stm_runs, stm_error = [], None
    stm_steps = args.stm_steps or max(1, args.mcmc_steps // 10)
    half = args.chains // 2
    try:
        fixed = None
        if "start" in args.stm_anchor:
            # every chain's exact curve at its starting state, the anchor of
            # its approximation for the whole run
            ex_a = ExactChi2(eng, data, curves=True)
            ex_a(theta0)
            f0 = torch.empty((args.chains, eng._n), dtype=torch.float64, device="cuda")
            ex_a.curves_all_device(f0)
            fixed = sur_loc_chi.fixed_anchor(theta0, f0)
        for mode in args.stm_anchor:
            sur_t = fixed if mode == "start" else sur_loc_chi
            for layout in args.stm_layouts:
                parts = ([slice(0, args.chains)] if layout == "whole" else
                         [slice(0, half), slice(half, args.chains)])
                for L in args.stm_inner:
                    runners = [DeviceTransitions(
                        sur_loc_chi, tw, S.BOX, part.stop - part.start, L,
                        seed=41 + 2 * rank + k,
                        anchor=fixed.rows(part) if mode == "start" else None)
                        for k, part in enumerate(parts)]
                    ex_t = ExactChi2(eng, data)
                    lib.lcg_kernel_launches(1)
                    cht, _, _, acct, wall_t, stt = surrogate_transitions(
                        ex_t, sur_t, theta0, None, stm_steps, L, seed=21,
                        device=runners[0] if layout == "whole" else runners)
                    stt["layout"], stt["anchor"] = layout, mode
                    stm_runs.append((L, cht, acct, wall_t, stt, ex_t.evals,
                                     int(lib.lcg_kernel_launches(1)) +
                                     sum(d.launches for d in runners)))
                    del runners
    except Exception as exc:  # a comparison beside the metric: the line keeps the rest
        stm_error = "%s: %s" % (type(exc).__name__, exc)
    clk = clocks.stop()
    sum_p, sum_d, sum_g = summary(chp, wall_p), summary(chd, wall_d), summary(chg, wall_g)
    shift, mcse = mean_shift(chd, chp)
    shift_g, mcse_g = mean_shift(chg, chp)
    sd_p = chp.reshape(-1, 9).std(0)
    mcse_is = np.sqrt(np.diag(cov_is) / ess_is) / sd_p
    shift_is = {k: (np.abs(c.reshape(-1, 9).mean(0) - mu_is) / sd_p).max()
                for k, c in (("plain", chp), ("delayed_acceptance", chd))}
    del chg
    stm = []
    for L, cht, acct, wall_t, stt, evals_t, launches_t in stm_runs:
        sum_t = summary(cht, wall_t)
        shift_t, mcse_t = mean_shift(cht, chp)
        stm.append(dict(sum_t, steps=cht.shape[0],
                        ms_per_step=wall_t / cht.shape[0] * 1e3, acceptance=acct,
                        exact_evals=evals_t, gpu_launches=launches_t,
                        ess_per_s_ratio=sum_t["ess_bulk_per_s"] / sum_p["ess_bulk_per_s"],
                        ess_per_s_ratio_geyer=sum_t["ess_geyer_per_s"] /
                        sum_p["ess_geyer_per_s"],
                        posterior_mean_shift_sigma_max=float(shift_t.max()),
                        mcse_max=float(mcse_t.max()),
                        verdict_0_1_sigma=shift_verdict(shift_t, mcse_t), **stt))
    del stm_runs
    peak, peak_src = _bf16_peak()
    train_tflops = train_flop / sur.train_s / 1e12
    value = sum_d["ess_bulk_per_s"]
    nbytes_model = C_sizeof_model()
    line = {
        "metric": "MCMC effective samples/s", "value": value,
        "unit": "effective samples/s", "n_gpus": world, "steps": args.mcmc_steps,
        "warmup": args.burn + args.burn_fixed + args.adapt_rounds * args.burn_tuned,
        "ms_per_step": wall_d / args.mcmc_steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 tensor-core MLP (fp32 accumulate) + f32/f64 engine",
        "data": "synthetic (wd_dm_small physics at 500 points + noise sigma=1.5e-3)",
        "config": {"workload": "surrogate_da: %d chains x %d steps, 9 parameters; surrogate "
                               "9 -> 4x256 GELU -> 64 PCA coefficients of a %d-point curve, "
                               "%d training curves" % (args.chains, args.mcmc_steps, S.NGRID,
                                                       args.train_curves),
                   "ess": "bulk ESS: rank-normalised multi-chain ESS of the split chains "
                          "(Vehtari, Gelman, Simpson, Carpenter & Buerkner 2021), minimum "
                          "over parameters; ess_geyer: the reference's estimator "
                          "(new_scripts/mcmc_solver.cpp:80-115) summed over chains, frozen "
                          "chains counted as zero",
                   "start": "both samplers from the same %d states, resampled from an "
                            "importance sample of the posterior (%d exact curves in %d pools, "
                            "effective size %.0f; after each adaptive round: %s)"
                            % (args.chains, len(chi_pool), len(pools), ess_is,
                               [round(x) for x in ess_rounds])},
        "plain": dict(sum_p, acceptance=accp, exact_evals=n_plain),
        "delayed_acceptance": dict(sum_d, surrogate="refined along the posterior's ridge",
                                   acceptance=accd,
                                   exact_evals=exact2.evals + (comp2.evals if comp2 else 0),
                                   exact_batch="%d slots" % args.compact if comp2 else "chains",
                                   **st),
        "delayed_acceptance_global": dict(sum_g, surrogate="prior box only", acceptance=accg,
                                          exact_evals=exact_g.evals +
                                          (comp_g.evals if comp_g else 0),
                                          posterior_mean_shift_sigma_max=float(shift_g.max()),
                                          **stg),
        "ess_per_s_ratio": value / sum_p["ess_bulk_per_s"],
        "ess_per_s_ratio_geyer": sum_d["ess_geyer_per_s"] / sum_p["ess_geyer_per_s"],
        "ess_per_s_ratio_between_chains": (sum_d["ess_between_chains"] / wall_d) /
                                          (sum_p["ess_between_chains"] / wall_p),
        "posterior_mean_shift": {
            "sigma_max": float(shift.max()), "per_parameter": shift.tolist(),
            "mcse_per_parameter": mcse.tolist(),
            "verdict_0.1_sigma": shift_verdict(shift, mcse),
            "rule": "within: every |mean_DA - mean_plain| / sd_plain + 2 mcse < 0.1; outside: "
                    "some shift - 2 mcse > 0.1",
            "vs_importance_sample": {k: float(v) for k, v in shift_is.items()},
            "importance_sample_mcse_max": float(mcse_is.max())},
        "surrogate": {"train_curves": args.train_curves, "curve_generation_s": t_gen,
                      "curves_per_s": args.train_curves / t_gen, "fit_s": t_fit,
                      "pca_s": sur.pca_s,
                      "epochs": args.epochs, "final_loss": losses[-1],
                      "heldout_rms_curve_error": rel_err, "pca_max_error": sur.pca_max_err,
                      "inference_ms_per_batch": t_inf * 1e3,
                      "refined": {"curves": args.local_curves, "seconds": t_ref,
                                  "final_loss": losses_loc[-1],
                                  "local_rms_curve_error": loc_err,
                                  "global_net_local_rms_curve_error": glob_err_loc,
                                  "pca_max_error": sur_loc.pca_max_err},
                      "importance_resampling_s": t_sir},
        "roofline": {"bound": "tensor",
                     "kernel": "training steps (one graph each: k_mlp_chain forward and "
                               "backward, k_gemm weight gradients), PCA excluded",
                     "achieved": train_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": train_tflops / peak, "traffic": None, "peak_source": peak_src,
                     "flop_per_sample_train": sur.net.flops_per_sample(train=True),
                     "ms_per_training_step": sur.train_s / sur.train_steps * 1e3},
        # the samplers' wall clock already covers every per-step transfer: the
        # proposals (models) to the device, chi**2 back to the host
        "e2e": {"value": value, "unit": "effective samples/s",
                "h2d_bytes_per_step": int(args.chains * 9 * 4 +
                                          st["stage1_rate"] * args.chains * nbytes_model),
                "d2h_bytes_per_step": int(2 * args.chains * 8),
                "note": "wall-clock sampling: every step sends the proposals and reads chi**2"},
        "gpu_launches": launches_da,
        "gpu_launches_plain": launches_plain,
        "proposal": "random walk in coordinates straightening the posterior's curved ridge "
                    "(sampler.TriangularWalk: volume-preserving quadratic triangular map, "
                    "refitted on %d adaptive burn-in rounds of %d steps)"
                    % (args.adapt_rounds, args.burn_tuned),
        "proposal_tuning": {"scale_acceptance": tuning, "chosen": f_best,
                            "burn_in_steps": args.adapt_rounds * args.burn_tuned},
        "da_scale_pilots": [{"scale": k, "acceptance": a, "sq_jump_per_s": e,
                             "min_param_jump_per_s": mp}
                            for k, a, e, mp in da_pilots],
        "da_proposal_scale": da_scale,
        "surrogate_transitions": stm if stm_error is None else {"runs": stm,
                                                                 "error": stm_error},
        "clocks": clk,
    }
    if eng_c is not None:
        eng_c.close()
    eng.close()
    return line if rank == 0 else None


def run_mlp_train(args):
    """The surrogate network's training step alone: cfg4's network (9 -> 4 x
    256 GELU -> 64) at its training batch of 4096, each step one CUDA graph
    (fused forward with the loss gradient, fused backward chain, the four
    weight-gradient GEMMs, bias gradients, the input layer's gradient, one
    Adam launch), as Surrogate.fit runs it. value: training samples/s with
    the batch resident; e2e: the batch copied from pinned host memory and the
    loss read back every step; roofline: the network's FLOPs (3 x forward)
    per step over its CUDA-event time against the BF16 tensor peak. Also
    times the one-launch inference of 512 rows (the delayed-acceptance
    screening batch)."""
    import torch
    from lcurve_re_b200.mlp import MLP
    rank, local, world = rank_info()
    net = MLP(nin=9, nout=64, batch=4096, seed=rank)
    g = torch.Generator(device="cuda").manual_seed(rank)
    x = torch.rand(net.B, 9, device="cuda", generator=g) * 2 - 1
    t = torch.sin(2 * x @ torch.randn(9, 64, device="cuda", generator=g)).contiguous()
    net.x.copy_(x)
    net.tgt.copy_(t)
    net.set_schedule(1e-3)
    lib = net.lib
    lib.lcg_kernel_launches(1)
    net.graph_step()  # eager, then captured
    launches = int(lib.lcg_kernel_launches(1))
    for _ in range(max(args.warmup, 3)):
        net.graph_step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        net.graph_step()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    # end to end: the batch from pinned host memory, the loss back, every step
    hx, ht = x.cpu().pin_memory(), t.cpu().pin_memory()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.x.copy_(hx, non_blocking=True)
        net.tgt.copy_(ht, non_blocking=True)
        net.graph_step()
        loss = net.take_loss()
    e2e_s = (time.perf_counter() - t0) / args.steps
    # inference, 512 rows
    xin = x[:512].contiguous()
    for _ in range(3):
        net.forward(xin)
    ev0.record()
    for _ in range(50):
        net.forward(xin)
    ev1.record()
    torch.cuda.synchronize()
    inf_ms = ev0.elapsed_time(ev1) / 50
    clk = clocks.stop()
    net.check()
    flop = net.B * net.flops_per_sample(train=True)
    peak, peak_src = _bf16_peak()
    tflops = flop / (ms * 1e-3) / 1e12
    if rank != 0:
        return None
    return {
        "metric": "surrogate training samples/s", "value": net.B / (ms * 1e-3),
        "unit": "samples/s", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 tensor-core GEMMs (fp32 accumulate), fp32 input layer and optimiser",
        "data": "synthetic (uniform inputs, sinusoidal targets)",
        "config": {"workload": "mlp_train: 9 -> 4x256 GELU -> 64, batch 4096, one CUDA graph "
                               "per step", "l2": "not flushed (the weights, 0.9 MB, and the "
                                                 "batch stay in L2 as they do in training)",
                   "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "tensor", "kernel": "training step (k_mlp_chain x 2 + k_gemm x 4 "
                                                  "+ small kernels)",
                     "achieved": tflops, "peak": peak, "unit": "TFLOP/s", "frac": tflops / peak,
                     "traffic": None, "peak_source": peak_src,
                     "flop_per_step": flop},
        "e2e": {"value": net.B / e2e_s, "unit": "samples/s",
                "h2d_bytes_per_step": int(hx.numel() * 4 + ht.numel() * 4),
                "d2h_bytes_per_step": 8, "last_loss": loss},
        "inference_ms_512_rows": inf_ms,
        "gpu_launches": launches * args.steps,
        "gpu_launches_per_step": launches,
        "clocks": clk,
    }


def C_sizeof_model():
    import ctypes as C
    return C.sizeof(abi.LcgModel)


def run_reference_da(args):
    """The reference's own CPU path driving plain Metropolis on the same data
    (wd_dm_small physics at 500 points): a few chains for a bounded number of
    steps, so the run takes seconds; ESS/s by the same estimator."""
    rank, _, world = rank_info()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as OL
    from lcurve_re_b200 import surrogate as S
    from lcurve_re_b200 import workloads as W
    from lcurve_re_b200.sampler import metropolis, summary
    kind = "reference" if os.path.exists(OL.REF_RELEASE_SO) else "port"
    lib = OL.Reference(OL.REF_RELEASE_SO) if kind == "reference" else OL.Oracle()
    fac = S.ModelFactory()
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    st, err, calc, _, _ = lib.light_curve(fac(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                                          scale=False, rdata=False)
    data = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 1234)

    class RefChi2:
        evals = 0

        def __call__(self, theta):
            out = np.empty(theta.shape[0])
            for i, t in enumerate(theta):
                st, err, _, _, sc = lib.light_curve(fac(t[None])[0], data)
                out[i] = sc[1] if st == 0 else np.inf
            RefChi2.evals += theta.shape[0]
            return out

    exact = RefChi2()
    chains = 8
    rng = np.random.default_rng(7)
    scale0 = (S.BOX[:, 1] - S.BOX[:, 0]) * 1e-3
    theta0 = truth + rng.standard_normal((chains, 9)) * scale0
    cov = np.diag(scale0 ** 2)
    burn = max(20, args.warmup * 10)
    ch, theta0, _, _, _ = metropolis(exact, theta0, cov, burn, seed=11)
    samp = ch[burn // 2:].reshape(-1, 9)
    cov = np.cov(samp.T) * 2.38 ** 2 / 9 + np.diag((scale0 * 1e-3) ** 2)
    steps = min(400, max(40, args.steps * 20))  # about half a minute of CPU
    chp, _, _, acc, wall = metropolis(exact, theta0, cov, steps, seed=21)
    sm = summary(chp, wall)
    v = sm["ess_bulk_per_s"]
    line = {"impl": "reference", "metric": "MCMC effective samples/s", "value": v,
            "unit": "effective samples/s", "n_gpus": world, "steps": steps, "warmup": burn,
            "ms_per_step": wall / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (wd_dm_small physics at 500 points + noise sigma=1.5e-3)",
            "config": {"workload": "surrogate_da reference arm: plain Metropolis, %d chains x "
                                   "%d steps on the reference CPU path" % (chains, steps),
                       "ess": "bulk ESS (rank-normalised multi-chain ESS of the split chains), "
                              "minimum over parameters"},
            "plain": sm,
            "cpu_baseline": {"value": v, "unit": "effective samples/s", "cores": os.cpu_count(),
                             "kind": kind,
                             "sample": "%d chains x %d steps after %d burn-in steps, one light "
                                       "curve per chain and step, acceptance %.2f"
                                       % (chains, steps, burn, acc)},
            "e2e": {"value": v, "unit": "effective samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    return line


def launch_ranks(n):
    """bench.py --gpus N started without a launcher: one process per GPU on
    this node, with RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* set as
    torch.distributed.run sets them, and the same arguments. Only rank 0
    prints. Returns the first non-zero exit status of the ranks."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n),
                   LOCAL_WORLD_SIZE=str(n), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:],
                                      env=env))
    rcs = [p.wait() for p in procs]
    return next((rc for rc in rcs if rc), 0)


def init_dist(world):
    """The process group for max-over-ranks timing (NCCL on GPUs, gloo where
    CUDA is absent); None for one rank."""
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return dist


def sub_args(args, **over):
    a = argparse.Namespace(**vars(args))
    for k, v in over.items():
        setattr(a, k, v)
    return a


def extra_workloads(args, world):
    """The default run at one GPU also reports the batched engine (cfg2) and
    the surrogate's delayed acceptance (cfg4, the named 512 chains x 20,000
    steps), each as a sub-object with its own value, e2e, cpu_baseline and
    clocks."""
    return (world == 1 and args.workload == "wd_dm_large" and args.precision == "mixed"
            and not args.headline_only)


MCMC_NAMED = dict(mcmc_steps=20000)


def main():
    args = parse()
    if args.ref_cuda_child:
        return reference_cuda_child(args) or 0
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus)
    rank, local, world = rank_info()
    more = extra_workloads(args, world)
    if args.impl == "reference":
        if args.workload == "surrogate_da":
            line = run_reference_da(args)
        elif args.workload == "mcmc_batch":
            line = run_reference_batch(args)
        else:
            line = run_reference(args)
        if line is not None and more:
            line["workloads"] = {
                "mcmc_batch": run_reference_batch(sub_args(args, steps=1, warmup=0)),
                "surrogate_da": run_reference_da(sub_args(args, **MCMC_NAMED))}
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    import torch
    torch.cuda.set_device(local)
    dist = init_dist(world)
    try:
        if args.workload == "surrogate_da":
            line = run_surrogate(args)
        elif args.workload == "mlp_train":
            line = run_mlp_train(args)
        elif args.workload == "mcmc_batch":
            line = run_batch(args, dist)
        else:
            line = run_ours(args, dist)
            if line is not None and more:
                line["workloads"] = {
                    "mcmc_batch": run_batch(sub_args(args, steps=min(args.steps, 20)), dist),
                    "surrogate_da": run_surrogate(sub_args(args, **MCMC_NAMED))}
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
