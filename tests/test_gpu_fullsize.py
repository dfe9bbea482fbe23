"""Size-independent properties at the full size of the headline workload
(100x50x67 hexes, 2,010,000 tets, 557.8M nonzeros), where no oracle run fits
a test: the exact nonzero count 4E + 52F + 168T, the sum of A's values equal
to the sum of all element-slot values (every slot lands in exactly one
nonzero; FP64, 1e-12 of the absolute sum), bitwise determinism, linearity in
the combination's coefficients (1e-13), and the mixed form within 1e-6 of
FP64 (relative Frobenius and max entry) for A."""
import numpy as np
import pytest
import torch

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices

pytestmark = pytest.mark.gpu


def test_full_size_properties():
    wl = W.wr90_dielectric()
    f = wl.field
    m = f.mesh
    none = np.zeros(0, np.int64)
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, none)
    assert f.ntets == 2_010_000
    assert cmap.nnz == 4 * m.n_edges + 52 * m.n_tris + 168 * f.ntets
    assert np.array_equal(np.diff(cmap.indptr) > 0, np.ones(cmap.N, bool))
    k2 = wl.k0 ** 2
    A = cmap.to_device(E - B * k2).clone()
    # every element slot lands in exactly one nonzero
    slots = E.to_device() - k2 * B.to_device()
    s_slots = complex(slots.sum().item())
    scale = float(slots.abs().sum().item())
    del slots
    assert abs(complex(A.sum().item()) - s_slots) <= 1e-12 * scale
    # bitwise determinism
    assert torch.equal(cmap.to_device(E - B * k2), A)
    # linearity: 2K - 3M from the combination equals 2 K - 3 M formed apart
    K = cmap.to_device(E * 1.0).clone()
    M = cmap.to_device(B * 1.0).clone()
    L2 = cmap.to_device(E * 2.0 - B * 3.0)
    d = L2 - (2.0 * K - 3.0 * M)
    assert float(d.abs().max()) <= 1e-13 * float(L2.abs().max())
    del K, M, L2, d
    torch.cuda.empty_cache()
    # the mixed form within its stated tolerance
    E2, B2, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, none, cmap, precision="mixed")
    A32 = cmap.to_device(E2 - B2 * k2)
    diff = A32 - A
    fro = float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(A))
    mx = float(diff.abs().max() / A.abs().max())
    assert fro <= 1e-6 and mx <= 1e-6, (fro, mx)


def test_full_size_pml_mixed_tolerance():
    """The 84x50x40 PML + slivers workload (1,008,000 tets, diagonal complex
    er = ur in the shell, 2% slivers): exact nonzero count; mixed vs FP64
    within 1e-6 for K, M and A with all tensor components, and with only the
    xx, yy or zz component kept (the others 1). Against the exact closed form
    (FP64, edge-vector geometry) the mixed form stays within 2e-7: most of its
    difference from the FP64 form is the reference arithmetic's own error on
    the thinnest slivers, which the FP64 form reproduces."""
    wl = W.wr90_pml_slivers()
    f = wl.field
    m = f.mesh
    assert f.ntets == 1_008_000
    _, _, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets)
    assert cmap.nnz == 4 * m.n_edges + 52 * m.n_tris + 168 * (f.ntets - len(wl.conductor_tets))

    def comp(t, c):
        o = np.zeros_like(t)
        for d in range(3):
            o[d, d] = t[d, d] if d == c else 1.0
        return o

    k2 = wl.k0 ** 2
    for c in (None, 0, 1, 2):
        er = wl.er if c is None else comp(wl.er, c)
        ur = wl.ur if c is None else comp(wl.ur, c)
        E, B, _ = tet_mass_stiffness_matrices(f, er, ur, wl.conductor_tets, cmap)
        E2, B2, _ = tet_mass_stiffness_matrices(f, er, ur, wl.conductor_tets, cmap, precision="mixed")
        for name, a, b in (("K", E * 1.0, E2 * 1.0), ("M", B * 1.0, B2 * 1.0), ("A", E - B * k2, E2 - B2 * k2)):
            v64 = cmap.to_device(a).clone()
            v32 = cmap.to_device(b)
            d = v32 - v64
            fro = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(v64))
            mx = float(d.abs().max() / v64.abs().max())
            assert fro <= 1e-6 and mx <= 1e-6, (c, name, fro, mx)
            del v64, v32, d
    E, B, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets, cmap, precision="exact")
    E2, B2, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets, cmap, precision="mixed")
    for name, a, b in (("K", E * 1.0, E2 * 1.0), ("M", B * 1.0, B2 * 1.0), ("A", E - B * k2, E2 - B2 * k2)):
        vex = cmap.to_device(a).clone()
        v32 = cmap.to_device(b)
        d = v32 - vex
        fro = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(vex))
        mx = float(d.abs().max() / vex.abs().max())
        assert fro <= 2e-7 and mx <= 2e-7, ("vs exact", name, fro, mx)
        del vex, v32, d


def test_full_size_sweep_with_ports():
    """The resident sweep with two TE10 port terms on the full 2.01M-tet mesh
    against assembling each frequency from scratch (1e-13 relative)."""
    from emerge_b200.mesh import plane_tris
    from emerge_b200.robin import RobinTerm
    from emerge_b200.sweep import FrequencySweep

    wl = W.wr90_dielectric()
    f = wl.field
    z = f.mesh.nodes[2]
    none = np.zeros(0, np.int64)
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, none)
    R1 = RobinTerm(f, plane_tris(f.mesh, 2, float(z.min())), cmap)
    R2 = RobinTerm(f, plane_tris(f.mesh, 2, float(z.max())), cmap)
    sw = FrequencySweep(E, B, cmap, robin=[R1, R2])
    freqs = np.array([8e9, 10e9, 12e9])
    gam = np.array([W.rect_port_gamma(x) for x in freqs])
    A = sw.form(FrequencySweep.coefficients(freqs), robin_gamma=np.stack([gam, gam], axis=1))
    for i, fr in enumerate(freqs):
        k0 = 2 * np.pi * fr / W.C0
        direct = cmap.to_device(E - B * k0 ** 2 + R1 * gam[i] + R2 * gam[i])
        d = A[i] - direct
        assert float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(direct)) <= 1e-13
        assert float(d.abs().max() / direct.abs().max()) <= 1e-13


def test_full_size_heat_properties():
    """The 2.01M-tet Lagrange-2 heat box: K 1 = 0 (the basis sums to one), the
    entries of M sum to sum_q w_q * sum_t rho_cp V_t (the reference's 8-digit
    weights), the two element forms agree to 1e-9 (they differ by the
    reference's own rounding, which grows with the mesh's offset/size ratio)."""
    from emerge_b200.heat import tet_mass_matrix, tet_stiffness_matrix

    wl = W.heat_box()
    f = wl.field
    m = f.mesh
    K, cmap = tet_stiffness_matrix(f, wl.cond)
    Kx, _ = tet_stiffness_matrix(f, wl.cond, precision="exact")
    kv, kxv = cmap.to_device(K), cmap.to_device(Kx)
    assert float((kxv - kv).abs().max() / kv.abs().max()) <= 1e-9
    ptr = torch.from_numpy(cmap.indptr.astype(np.int64)).to(kv.device)
    col = torch.repeat_interleave(torch.arange(cmap.N, device=kv.device), ptr[1:] - ptr[:-1])
    row_sums = torch.zeros(cmap.N, dtype=torch.float64, device=kv.device).index_add_(0, col, kv)  # K^T 1 = K 1
    assert float(row_sums.abs().max()) <= 1e-9 * float(kv.abs().max())
    M, _ = tet_mass_matrix(f, wl.rho_cp)
    X = m.nodes[:, m.tets]
    V = np.abs(np.einsum("it,it->t", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0], axis=0))) / 6
    expect = (-0.078933 + 4 * 0.04573333 + 6 * 0.14933333) * float((wl.rho_cp * V).sum())
    assert abs(float(cmap.to_device(M).sum()) - expect) <= 1e-10 * expect
