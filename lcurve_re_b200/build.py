"""Builds the engine library lcurve_re_b200/liblcg.so for sm_100a.

Per-file flags: the FP64 stages (geometry.cu, flux64.cu, engine.cu) are
compiled with --fmad=false so each product and sum rounds separately, as in
the reference CPU code; the mixed-precision sweep (flux.cu) keeps FMA
contraction. The CUDA runtime is linked statically, so the library has no
dependency beyond the driver.

    python -m lcurve_re_b200.build [--force] [--jobs N]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liblcg.so")
OBJDIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
SOURCES = {
    "geometry.cu": ["--fmad=false"],
    "flux64.cu": ["--fmad=false"],
    "engine.cu": ["--fmad=false"],
    "flux.cu": ["--fmad=true"],
    "noalloc.cu": ["--fmad=false"],
    "batch_host.cu": ["--fmad=false"],
    "mlp.cu": ["--fmad=true"],
    "mlp_chain.cu": ["--fmad=true"],
    "components.cu": ["--fmad=false"],
    "walk.cu": ["--fmad=false"],
}
HEADERS = ["roche.cuh", "eclipse.cuh", "disc.cuh", "ecl_screen.cuh", "engine.h", "tma.cuh",
           "context.h", "fixed_phase.cuh", "mlp_tc.cuh"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, jobs=4, verbose=False, extra=()):
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "lcg.h")]
    cmds = []
    objs = []
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmds.append([nvcc()] + ARCH + COMMON + flags + list(extra) + ["-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for err in ex.map(run, cmds):
            if verbose and err.strip():
                print(err)
    if force or cmds or _stale(LIB, objs):
        run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills (-Xptxas -v)")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    print(build(force=a.force or a.ptxas_info, jobs=a.jobs, verbose=a.verbose or a.ptxas_info,
                extra=extra))


if __name__ == "__main__":
    sys.exit(main())
