"""Port S-parameters at the size of the survey's config 0 (the 12x6x30
WR-90 air box, 12,960 tets, 10 GHz): the system assembled on the GPU (plain
FP64 and mixed forms, TE10 port terms, port excitation) and the same system
assembled by the oracle are each solved with scipy's SuperLU under the
reference's SolverSuperLU settings; S11 and S21 (GPU port overlaps vs the
oracle's) must agree to 1e-9 for FP64 and to 1e-5 for the mixed form, whose
A is within 1e-6 of FP64. The K, M and A errors of both forms against the
oracle are checked too (1e-12 / 1e-6 relative, Frobenius and max entry).
Run with -s to see the deviations."""
import numpy as np
import pytest
import torch
from scipy.sparse import csc_matrix

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.mesh import plane_tris
from emerge_b200.postprocess import TRI_RULE_6, FieldOnDevice, PortOverlap
from emerge_b200.robin import RobinTerm
from emerge_b200.solve_dofs import SolveSubmatrix, superlu_like_reference
from oracle import oracle as O
from tests.golden_util import rel_err

pytestmark = pytest.mark.gpu


def test_config0_s_parameters_against_the_oracle_chain():
    wl = W.wr90_air(n=(12, 6, 30))
    f = wl.field
    m = f.mesh
    a, b, length = W.WR90
    k0, gamma = wl.k0, W.rect_port_gamma(wl.freq)
    beta = abs(gamma)
    p1, p2 = plane_tris(m, 2, 0.0), plane_tris(m, 2, float(m.nodes[2].max()))
    walls = np.concatenate([plane_tris(m, ax, v) for ax, vals in ((0, (0.0, a)), (1, (0.0, b))) for v in vals])
    solve = np.setdiff1d(np.arange(f.n_field), np.unique(f.tri_to_field[:, walls]))

    def mode(P):
        e = np.zeros(P.shape, np.complex128)
        e[1] = np.sin(np.pi * P[0] / a)
        return e

    # oracle chain
    dE, dB, oc = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    shape = (f.n_field, f.n_field)
    Kref = oc.values_lincomb(dE, dB, 1.0, 0.0)
    Mref = oc.values_lincomb(dE, dB, 0.0, 1.0)
    Aref_v = oc.values_lincomb(dE, dB, 1.0, -k0 ** 2)
    Aref = (csc_matrix((Aref_v, oc.indices, oc.indptr), shape=shape)
            + O.generate_csc(f, O.robin_entries(f, np.concatenate([p1, p2]), gamma))).tocsc()
    bref = O.force_entries(f, p1, -2j * beta * mode(O.tri_points(f, p1)))
    xr = np.zeros(f.n_field, np.complex128)
    xr[solve] = superlu_like_reference(Aref[:, solve][solve, :], bref[solve])
    fod = FieldOnDevice(f)
    po1, po2 = PortOverlap(fod, p1), PortOverlap(fod, p2)
    U1, U2 = mode(po1.quadrature_points()), mode(po2.quadrature_points())
    z0 = np.zeros_like(xr)
    S11r = (O.port_overlap(f, xr, p1, po1.tri_tets, TRI_RULE_6, U1, 1.0)[0]
            / O.port_overlap(f, z0, p1, po1.tri_tets, TRI_RULE_6, U1, -1.0)[0])
    S21r = (O.port_overlap(f, xr, p2, po2.tri_tets, TRI_RULE_6, U2, 0.0)[0]
            / O.port_overlap(f, z0, p2, po2.tri_tets, TRI_RULE_6, U2, -1.0)[0])
    assert abs(abs(S21r) - 1) < 1e-2 and abs(S11r) < 1e-2, (S11r, S21r)  # the physics holds on this mesh
    print(f"\noracle: S11 {S11r:.6e} S21 {S21r:.9f} (exact S21 {np.exp(-1j * beta * length):.9f})")
    for precision, tol_v, tol_s in (("fp64", 1e-12, 1e-9), ("mixed", 1e-6, 1e-5)):
        E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64), precision=precision)
        errs = {}
        for key, data, ref in (("K", E * 1.0, Kref), ("M", B * 1.0, Mref), ("A", E - B * k0 ** 2, Aref_v)):
            errs[key] = rel_err(cmap.to_device(data).cpu().numpy(), ref)
            assert errs[key][0] <= tol_v and errs[key][1] <= tol_v, (precision, key, errs[key])
        R1, R2 = RobinTerm(f, p1, cmap), RobinTerm(f, p2, cmap)
        sub = SolveSubmatrix(cmap, solve)
        Asel = sub.to_csc(E - B * k0 ** 2 + (R1 + R2) * gamma)
        bsel = sub.rhs(R1.force(-2j * beta * mode(R1.quadrature_points()))).cpu().numpy()
        x = sub.expand(torch.from_numpy(superlu_like_reference(Asel, bsel)).to(cmap.device))
        zero = torch.zeros_like(x)
        S11 = po1(x, U1, 1.0)[0] / po1(zero, U1, -1.0)[0]
        S21 = po2(x, U2, 0.0)[0] / po2(zero, U2, -1.0)[0]
        d11, d21 = abs(S11 - S11r), abs(S21 - S21r)
        print(f"{precision}: |dS11| {d11:.3e} |dS21| {d21:.3e}; K/M/A fro, max "
              + ", ".join(f"{k} {v[0]:.2e} {v[1]:.2e}" for k, v in errs.items()))
        assert d11 <= tol_s and d21 <= tol_s, (precision, d11, d21)
