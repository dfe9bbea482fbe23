"""Characterisation of the reference's own FP64 rounding (CPU only).

The reference forms its barycentric coefficients from absolute-coordinate
cofactors and evaluates L = a + b x + c y + d z at absolute quadrature
points (curlcurl.py:142-212, 319-321; ccbf.py); both cancel heavily when the
mesh sits far from the origin relative to its cell size. Against an 80-bit
evaluation of the exact integrals its element matrices err by ~1e-12 on the
12x6x30 WR-90 box and by up to ~1e-10 on the 100x50x67 grid; the exact closed
form in FP64 errs by ~1e-15. This is why the plain GPU form reproduces the
reference's arithmetic (parity) and the closed form is offered as the
separate "exact" form.
"""
import numpy as np

from emerge_b200 import workloads as W
from oracle import oracle as O
from tests.accuracy_util import element_ld, matinv, per_tet_errors


def _sampled(wl, n, seed):
    f = wl.field
    m = f.mesh
    ids = np.sort(np.random.default_rng(seed).choice(f.ntets, n, replace=False)).astype(np.int64)
    dE, dB, _, _ = O.matrix_builder(m.nodes, m.tets, m.tris, m.edges, f.get_tet_to_field(), m.tet_to_edge,
                                    m.tet_to_tri, wl.ur, wl.er, ids)
    ref = [element_ld(m.nodes[:, m.tets[:, it]], m.tets[:, it], matinv(wl.ur[:, :, it]), wl.er[:, :, it]) for it in ids]
    return dE.reshape(-1, 20, 20), dB.reshape(-1, 20, 20), ref


def test_reference_rounding_grows_with_distance_over_cell_size():
    dE, dB, ref = _sampled(W.wr90_dielectric(n=(50, 25, 34)), 60, 1)
    eK = per_tet_errors(dE, [r[0] for r in ref])
    eM = per_tet_errors(dB, [r[1] for r in ref])
    # the reference is far less accurate than FP64 round-off on this mesh
    assert np.median(np.maximum(eK, eM)) > 1e-13
    assert np.max(np.maximum(eK, eM)) < 1e-8
