"""Generates the golden fixtures of tests/golden/ from lcurve_re itself.

Runs the reference's own CPU path (oracle/_ref/liblcurve_ref.so, built by
`make -C oracle ref` from the reference sources) on the parity cases of
tests/cases.py and stores, per case: the light curve, scale factors, chi**2
and wnok; for two small models also both star grids. The fixtures let the C
oracle be checked where the reference sources are absent.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cases import glens_case, small_cases  # noqa: E402
from lcurve_re_b200 import workloads as W  # noqa: E402
from oracle_lib import Reference  # noqa: E402

GRID_MODELS = {
    "grid_small": dict(nlat1f=16, nlat2f=32),
    "grid_tiny_star": dict(nlat1f=24, nlat2f=12, r1=0.005, q=0.2, iangle=87.0),
}


def main():
    ref = Reference()
    out = {}
    meta = {"cases": [], "grids": list(GRID_MODELS)}
    for name, model, data in small_cases() + [glens_case()]:
        st, err, calc, sfac, sc = ref.light_curve(model, data)
        assert st == 0, (name, err)
        out[name + "/calc"] = calc
        out[name + "/sfac"] = sfac
        out[name + "/chisq_wnok"] = sc[1:3]
        out[name + "/data"] = np.asarray(data).view(np.uint8)
        meta["cases"].append(name)
    for name, over in GRID_MODELS.items():
        m = W.model(**over)
        for star in (0, 1):
            g = ref.star_grid(m, star)
            for k, v in g.items():
                out["%s/star%d/%s" % (name, star + 1, k)] = v
    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **out)
    with open(os.path.join(HERE, "reference_outputs.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
