"""The per-phase flag comparison the GPU parity tests use (tests/eclipse_flags.py),
on crafted grids: it passes identical grids and boundaries moved within the band,
and it counts a disagreement outside the band, for a moved boundary, for a face
only one grid eclipses, and across the wrap of a range past phase 1."""
import numpy as np

from eclipse_flags import compare


def _grid(ne, ein, eout):
    return {"neclipse": np.asarray(ne, np.int32), "ecl_in": np.asarray(ein, float),
            "ecl_out": np.asarray(eout, float)}


PHASES = np.linspace(0.0, 0.999, 1000)


def test_identical_grids_agree():
    g = _grid([1, 0, 1], [0.1, 0.0, 0.95], [0.2, 0.0, 1.05])
    f = compare(g, g, PHASES)
    assert f["faces_with_different_ranges"] == 0 and f["outside_band"] == 0


def test_boundary_moved_within_the_band_agrees():
    a = _grid([1], [0.1005], [0.2])
    b = _grid([1], [0.1005 + 5e-10], [0.2 - 5e-10])
    ph = np.r_[PHASES, 0.1005 + 2e-10]  # a phase between the two ingresses
    f = compare(a, b, ph)
    # that phase and the grid phase 0.2 (on a's egress) disagree, both in the band
    assert f["disagreeing_face_phase_pairs"] == 2 and f["outside_band"] == 0
    assert f["max_abs_ingress_diff"] <= 1e-9


def test_boundary_moved_beyond_the_band_is_counted():
    a = _grid([1], [0.1], [0.2])
    b = _grid([1], [0.1 + 3e-3], [0.2])
    f = compare(a, b, PHASES)
    # 0.100, 0.101, 0.102 disagree; 0.100 sits on a's ingress (in the band)
    assert f["disagreeing_face_phase_pairs"] == 3 and f["outside_band"] == 2
    assert f["max_abs_ingress_diff"] > 1e-9


def test_one_sided_face():
    a = _grid([1, 1], [0.1, 0.3], [0.2, 0.3 + 1e-12])
    b = _grid([0, 0], [0.0, 0.0], [0.0, 0.0])
    ph = np.r_[PHASES, 0.3 + 5e-13]
    f = compare(a, b, ph)
    # the wide window disagrees at its 101 grid phases (0.1 and 0.2 on its
    # boundaries), the 1e-12 one at 0.3 and 0.3 + 5e-13, within the band
    assert f["faces_with_different_flags"] == 2
    assert f["outside_band"] == 99 and f["disagreeing_face_phase_pairs"] == 103


def test_wrapped_range():
    a = _grid([1], [0.95], [1.05])
    b = _grid([1], [0.95], [1.06])
    f = compare(a, b, PHASES)
    # phases 0.051 ... 0.060 are eclipsed in b only (p <= egress - 1); 0.060
    # sits on b's wrapped egress
    assert f["disagreeing_face_phase_pairs"] == 10 and f["outside_band"] == 9
