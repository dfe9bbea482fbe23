"""Post-processing on the GPU against the reference's own output
(tests/golden/interp.npz): the solution at points (ned2_tet_interp) and the
port overlap integral of the S-parameters. Tolerance 1e-12 relative."""
import numpy as np
import pytest

from emerge_b200 import workloads as W
from emerge_b200.postprocess import TRI_RULE_6, FieldOnDevice, PortOverlap
from oracle import oracle as O
from tests.golden_util import load_npz

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_interpolation_matches_reference():
    g = load_npz("interp.npz")
    wl = W.wr90_air()
    fod = FieldOnDevice(wl.field)
    E = fod.interpolate(g["x"], g["pts"], g["tet_of"]).cpu().numpy()
    assert np.abs(E - g["E"]).max() <= TOL * np.abs(g["E"]).max()
    E2 = fod.interpolate(g["x"], g["pts"][:, :3], np.array([-1, 0, wl.n_tets])).cpu().numpy()
    assert np.isnan(E2[:, 0]).all() and np.isnan(E2[:, 2]).all() and np.isfinite(E2[:, 1]).all()


def test_port_overlap_matches_reference():
    g = load_npz("interp.npz")
    wl = W.wr90_air()
    fod = FieldOnDevice(wl.field)
    assert np.array_equal(g["rule5"], TRI_RULE_6)
    po = PortOverlap(fod, g["port_ids"])
    assert np.array_equal(po.tri_tets, g["port_tets"])
    P = po.quadrature_points()
    U = np.zeros(P.shape, np.complex128)
    U[1] = (1 + 0.5j) * np.sin(np.pi * P[0] / W.WR90[0])
    assert np.abs(U - g["U5"]).max() <= 1e-15
    for q, key in ((1.0, "overlap_active"), (0.0, "overlap_passive")):
        tot, per = po(g["x"], U, q)
        ref = complex(g[key])
        assert abs(tot - ref) <= TOL * abs(ref), (key, tot, ref)
        _, oper = O.port_overlap(wl.field, g["x"], g["port_ids"], g["port_tets"], TRI_RULE_6, U, q)
        assert np.abs(per.cpu().numpy() - oper).max() <= TOL * np.abs(oper).max()


def test_te10_guide_s_parameters_known_answer():
    """The analytic known answer: an air-filled WR-90 section with PEC walls
    and matched TE10 ports transmits the mode with S21 = exp(-j beta L) and
    reflects nothing. The whole chain runs on the GPU (assembly, port terms,
    port excitation, the solve-DoF submatrix, interpolation and the port
    overlaps); only the sparse solve runs on the host (scipy's SuperLU).
    Checked against physics and against the same chain on the oracle (1e-9)."""
    import torch
    from scipy.sparse import csc_matrix
    from scipy.sparse.linalg import splu

    from emerge_b200.assembly import tet_mass_stiffness_matrices
    from emerge_b200.mesh import plane_tris
    from emerge_b200.robin import RobinTerm
    from emerge_b200.solve_dofs import SolveSubmatrix

    wl = W.wr90_air(n=(6, 3, 15))
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

    # GPU chain
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R1, R2 = RobinTerm(f, p1, cmap), RobinTerm(f, p2, cmap)
    sub = SolveSubmatrix(cmap, solve)
    Asel = sub.to_csc(E - B * k0 ** 2 + (R1 + R2) * gamma)
    bsel = sub.rhs(R1.force(-2j * beta * mode(R1.quadrature_points()))).cpu().numpy()
    x = torch.zeros(f.n_field, dtype=torch.complex128, device=cmap.device)
    x[sub.d_ids] = torch.from_numpy(splu(Asel).solve(bsel)).to(cmap.device)
    fod = FieldOnDevice(f)
    po1, po2 = PortOverlap(fod, p1), PortOverlap(fod, p2)
    U1, U2 = mode(po1.quadrature_points()), mode(po2.quadrature_points())
    zero = torch.zeros_like(x)
    S11 = po1(x, U1, 1.0)[0] / po1(zero, U1, -1.0)[0]
    S21 = po2(x, U2, 0.0)[0] / po2(zero, U2, -1.0)[0]
    assert abs(S11) < 1e-3, S11
    assert abs(abs(S21) - 1) < 1e-3, S21
    assert abs(np.angle(S21 / np.exp(-1j * beta * length))) < 5e-3, S21
    # oracle chain
    dE, dB, oc = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    A = (csc_matrix((oc.values_lincomb(dE, dB, 1.0, -k0 ** 2), oc.indices, oc.indptr), shape=(f.n_field,) * 2)
         + O.generate_csc(f, O.robin_entries(f, np.concatenate([p1, p2]), gamma))).tocsc()
    bref = O.force_entries(f, p1, -2j * beta * mode(O.tri_points(f, p1)))
    xr = np.zeros(f.n_field, np.complex128)
    xr[solve] = splu(A[:, solve][solve, :]).solve(bref[solve])
    z0 = np.zeros_like(xr)
    S11r = (O.port_overlap(f, xr, p1, po1.tri_tets, TRI_RULE_6, U1, 1.0)[0]
            / O.port_overlap(f, z0, p1, po1.tri_tets, TRI_RULE_6, U1, -1.0)[0])
    S21r = (O.port_overlap(f, xr, p2, po2.tri_tets, TRI_RULE_6, U2, 0.0)[0]
            / O.port_overlap(f, z0, p2, po2.tri_tets, TRI_RULE_6, U2, -1.0)[0])
    assert abs(S21 - S21r) <= 1e-9 and abs(S11 - S11r) <= 1e-9, (S21, S21r, S11, S11r)


def test_te10_known_answer_with_the_solve_on_the_gpu():
    """The same guide with nothing on the host between the mesh and the
    S-parameters: the reduced system is solved on the device
    (SolveSubmatrix.solve), the solution expanded on the device. S21 =
    exp(-j beta L), S11 = 0 as in the host-solve chain."""
    import torch

    from emerge_b200.assembly import tet_mass_stiffness_matrices
    from emerge_b200.mesh import plane_tris
    from emerge_b200.robin import RobinTerm
    from emerge_b200.solve_dofs import SolveSubmatrix

    wl = W.wr90_air(n=(6, 3, 15))
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

    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R1, R2 = RobinTerm(f, p1, cmap), RobinTerm(f, p2, cmap)
    sub = SolveSubmatrix(cmap, solve)
    Asel = sub.values(cmap.to_device(E - B * k0 ** 2 + (R1 + R2) * gamma))
    bsel = sub.rhs(R1.force(-2j * beta * mode(R1.quadrature_points())))
    x = sub.expand(sub.solve(Asel, bsel))
    fod = FieldOnDevice(f)
    po1, po2 = PortOverlap(fod, p1), PortOverlap(fod, p2)
    U1, U2 = mode(po1.quadrature_points()), mode(po2.quadrature_points())
    zero = torch.zeros_like(x)
    S11 = po1(x, U1, 1.0)[0] / po1(zero, U1, -1.0)[0]
    S21 = po2(x, U2, 0.0)[0] / po2(zero, U2, -1.0)[0]
    assert abs(S11) < 1e-3, S11
    assert abs(abs(S21) - 1) < 1e-3, S21
    assert abs(np.angle(S21 / np.exp(-1j * beta * length))) < 5e-3, S21
