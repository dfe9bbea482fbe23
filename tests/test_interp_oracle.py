"""Oracle restatement of the post-processing (Nedelec-2 field interpolation
and the port overlap integral of the S-parameters) against the golden
fixture made by the reference's own code (tests/golden/make_golden_interp.py).
Tolerance 1e-12 relative (max entry / absolute value)."""
import numpy as np

from emerge_b200 import workloads as W
from oracle import oracle as O
from tests.golden_util import load_npz

TOL = 1e-12


def test_interpolation_matches_reference():
    g = load_npz("interp.npz")
    wl = W.wr90_air()
    E = O.ned2_interp(wl.field, g["x"], g["pts"], g["tet_of"])
    assert np.abs(E - g["E"]).max() <= TOL * np.abs(g["E"]).max()
    # outside points are NaN, as in the reference
    E2 = O.ned2_interp(wl.field, g["x"], g["pts"][:, :3], np.array([-1, 0, -1]))
    assert np.isnan(E2[:, 0]).all() and np.isnan(E2[:, 2]).all() and np.isfinite(E2[:, 1]).all()


def test_port_overlap_matches_reference():
    g = load_npz("interp.npz")
    wl = W.wr90_air()
    for q, key in ((1.0, "overlap_active"), (0.0, "overlap_passive")):
        tot, per = O.port_overlap(wl.field, g["x"], g["port_ids"], g["port_tets"], g["rule5"], g["U5"], q)
        ref = complex(g[key])
        assert abs(tot - ref) <= TOL * abs(ref), (key, tot, ref)
        assert abs(per.sum() - tot) <= 1e-14 * abs(tot)
