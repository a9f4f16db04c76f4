"""Per-face eclipse-flag agreement between two star grids, phase by phase.

A face's eclipse flag at phase p (p = phin, the sub-exposure phase reduced to
[0, 1)) is the reference's test (comp_light_flat.cpp:150-167, ecl_range):

    eclipsed(p) = (p >= ingress && p <= egress) || p <= egress - 1

for a face with one eclipse range, and false for a face with none. Two grids
agree "away from the boundary band" when every (face, phase) pair on which
their flags differ lies within `band` of a boundary (ingress, egress or
egress - 1) of either grid. `compare` checks that on the phases a workload
actually evaluates and also reports face-level figures: how many faces carry
different ranges, the largest ingress/egress difference where both grids see
an eclipse, and the widest window of a face that only one grid eclipses.
"""
import numpy as np


def _window_mask(phin, ein, eout):
    return ((phin >= ein) & (phin <= eout)) | (phin <= eout - 1.0)


def compare(g_test, g_ref, phin, band=1e-9):
    """Returns a dict of figures; `outside_band` must be 0 for agreement."""
    ne_t, ne_r = g_test["neclipse"], g_ref["neclipse"]
    assert ne_t.shape == ne_r.shape
    assert np.all(ne_t <= 1) and np.all(ne_r <= 1), "faces with several ranges"
    in_t, out_t = g_test["ecl_in"], g_test["ecl_out"]
    in_r, out_r = g_ref["ecl_in"], g_ref["ecl_out"]
    both = (ne_t == 1) & (ne_r == 1)
    same = (ne_t == ne_r) & (~both | ((in_t == in_r) & (out_t == out_r)))
    flag_diff = ne_t != ne_r
    d_in = np.abs(in_t[both] - in_r[both])
    d_out = np.abs(out_t[both] - out_r[both])
    width_only = np.where(ne_t == 1, out_t - in_t, out_r - in_r)[flag_diff]
    phin = np.asarray(phin, dtype=np.float64)
    pairs, outside = 0, 0
    worst = 0.0
    for f in np.nonzero(~same)[0]:
        wt = _window_mask(phin, in_t[f], out_t[f]) if ne_t[f] else np.zeros(phin.shape, bool)
        wr = _window_mask(phin, in_r[f], out_r[f]) if ne_r[f] else np.zeros(phin.shape, bool)
        dis = wt != wr
        k = int(dis.sum())
        if not k:
            continue
        pairs += k
        bounds = []
        if ne_t[f]:
            bounds += [in_t[f], out_t[f], out_t[f] - 1.0]
        if ne_r[f]:
            bounds += [in_r[f], out_r[f], out_r[f] - 1.0]
        dist = np.min(np.abs(phin[dis][:, None] - np.asarray(bounds)[None, :]), axis=1)
        worst = max(worst, float(dist.max()))
        outside += int((dist > band).sum())
    return {
        "faces": int(ne_t.shape[0]),
        "eclipsed_faces_ref": int(ne_r.sum()),
        "faces_with_different_ranges": int((~same).sum()),
        "faces_with_different_flags": int(flag_diff.sum()),
        "max_abs_ingress_diff": float(d_in.max()) if d_in.size else 0.0,
        "max_abs_egress_diff": float(d_out.max()) if d_out.size else 0.0,
        "max_window_of_one_sided_faces": float(width_only.max()) if width_only.size else 0.0,
        "phases": int(phin.shape[0]),
        "disagreeing_face_phase_pairs": pairs,
        "outside_band": outside,
        "max_distance_to_a_boundary": worst,
    }
