"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (no public dataset is involved).

* ``wr90_air``        12x6x30-hex WR-90 box (22.86 x 10.16 x 50 mm), +-5%
                      jitter, air, 10 GHz: 12,960 tets.
* ``wr90_dielectric`` the same box on a 100x50x67-hex grid (2,010,000 tets),
                      +-15% jitter, eps_r ~ U[1,10] and tan(delta) ~
                      U[1e-3,1e-2] per 8x8x8-cell block, mu_r = 1, 10 GHz.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import Nedelec2Field, TetMesh, structured_box

C0 = 299792458.0
WR90 = (22.86e-3, 10.16e-3, 50e-3)


@dataclass
class Workload:
    name: str
    field: Nedelec2Field
    er: np.ndarray  # c16[3,3,nT] (the reference's layout)
    ur: np.ndarray
    conductor_tets: np.ndarray
    freq: float
    hex_grid: tuple

    @property
    def k0(self) -> float:
        return 2 * np.pi * self.freq / C0

    @property
    def n_tets(self) -> int:
        return self.field.ntets


def _iso(nT, eps):
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = eps
        ur[d, d] = 1.0
    return er, ur


def block_ids(nx, ny, nz, block=8):
    """Block index of every tet (6 per hex, hex index x fastest)."""
    h = np.arange(nx * ny * nz)
    hi, hj, hk = h % nx, (h // nx) % ny, h // (nx * ny)
    bx, by = -(-nx // block), -(-ny // block)
    blk = (hi // block) + bx * ((hj // block) + by * (hk // block))
    return np.repeat(blk, 6)


def wr90_air(n=(12, 6, 30), jitter=0.05, seed=0, freq=10e9) -> Workload:
    nodes, tets = structured_box(*n, size=WR90, jitter=jitter, seed=seed)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er, ur = _iso(f.ntets, 1.0)
    return Workload("wr90_air", f, er, ur, np.zeros(0, np.int64), freq, tuple(n))


def wr90_dielectric(n=(100, 50, 67), jitter=0.15, seed=1, freq=10e9, block=8) -> Workload:
    nodes, tets = structured_box(*n, size=WR90, jitter=jitter, seed=seed)
    f = Nedelec2Field(TetMesh(nodes, tets))
    rng = np.random.default_rng(seed + 1000)
    blk = block_ids(*n, block=block)
    nb = int(blk.max()) + 1
    eps = rng.uniform(1.0, 10.0, nb)
    tand = rng.uniform(1e-3, 1e-2, nb)
    er, ur = _iso(f.ntets, (eps * (1 - 1j * tand))[blk])
    return Workload("wr90_dielectric", f, er, ur, np.zeros(0, np.int64), freq, tuple(n))


def rect_port_gamma(freq: float, width: float = WR90[0], height: float = WR90[1], er: float = 1.0,
                    mode=(1, 0)) -> complex:
    """Robin coefficient of a rectangular waveguide port, gamma = j beta with
    beta = sqrt(er k0^2 - (pi m / width)^2 - (pi n / height)^2)
    (bcs/port_bcs.py:963-983)."""
    k0 = 2 * np.pi * freq / C0
    beta = np.sqrt(er * k0 ** 2 - (np.pi * mode[0] / width) ** 2 - (np.pi * mode[1] / height) ** 2)
    return 1j * beta


def port_tris(wl: Workload) -> np.ndarray:
    """Triangles of the two waveguide ports of a WR-90 box: the z = 0 and
    z = length faces."""
    from .mesh import plane_tris

    m = wl.field.mesh
    z = m.nodes[2]
    return np.concatenate([plane_tris(m, 2, float(z.min())), plane_tris(m, 2, float(z.max()))])


def alg_bytes(n_nodes: int, n_tets: int, nnz: int, material_bytes_per_tet: int = 16) -> int:
    """Algorithmic bytes of one assembly: nodes + tets + material + int32
    slot->nnz map + segment offsets + complex128 A written."""
    S = 400 * n_tets
    return 24 * n_nodes + 16 * n_tets + material_bytes_per_tet * n_tets + 4 * S + 4 * (nnz + 1) + 16 * nnz


def floor_bytes(n_nodes: int, n_tets: int, nnz: int, material_bytes_per_tet: int = 16) -> int:
    """Compulsory traffic without the mandated map: inputs + A written."""
    return 24 * n_nodes + 16 * n_tets + material_bytes_per_tet * n_tets + 16 * nnz


def element_alg_bytes(n_nodes: int, n_tets: int, value_bytes: int, material_bytes_per_tet: int = 16,
                      values_per_tet: int = 220) -> int:
    """Algorithmic bytes of one element-kernel launch: nodes + tets + material
    read, the element values written (values_per_tet = 220 in the entity-pair
    block layout, 210 in the packed triangle; value_bytes = 16 for
    complex128, 8 for complex64)."""
    return (24 * n_nodes + 16 * n_tets + material_bytes_per_tet * n_tets
            + values_per_tet * value_bytes * n_tets)


def gather_alg_bytes(n_tets: int, nnz: int, value_bytes: int, values_per_tet: int = 220) -> int:
    """Algorithmic bytes of one gather launch: the element values read once,
    the int32 slot->nnz map (4 B per COO slot) and segment offsets, complex128
    A written. element_alg_bytes + gather_alg_bytes = alg_bytes + the
    2 x values_per_tet x value_bytes per tet of the intermediate round trip."""
    return values_per_tet * value_bytes * n_tets + 4 * 400 * n_tets + 4 * (nnz + 1) + 16 * nnz


def wr90_pml_slivers(n=(84, 50, 40), jitter=0.05, seed=4, freq=10e9, shell=0.10, sliver_frac=0.02,
                     sliver_aspect=50.0) -> Workload:
    """1,008,000-tet box (84x50x40 hexes over the WR-90 footprint) whose outer
    10% shell carries a diagonal complex uniaxial PML tensor, with 2% of the
    tets turned into slivers.

    PML: per axis s_a = 1 - j * sigma_a / k0 with sigma_a = sigma_max * (d_a /
    delta)^2, d_a the depth into the shell along axis a, delta the shell
    thickness along that axis and sigma_max = 2 / delta (so sigma / k0 is
    dimensionless); er = ur = diag(s_y s_z / s_x, s_z s_x / s_y, s_x s_y / s_z)
    (the stretched-coordinate form of geo/pmlbox.py:80-92).

    Slivers: for a seeded 2% of tets one vertex is moved toward the plane of
    its opposite face until its height is 1/50 of the face's circumradius-scale
    edge length; tets that any move inverts are re-oriented (det > 0 kept in
    FP64 for every tet)."""
    from .mesh import orient_positive, tet_signed_volumes

    size = WR90
    nodes, tets = structured_box(*n, size=size, jitter=jitter, seed=seed)
    rng = np.random.default_rng(seed + 77)
    nT = tets.shape[1]
    pick = np.sort(rng.choice(nT, int(round(sliver_frac * nT)), replace=False))
    nodes = nodes.copy()
    used = np.zeros(nodes.shape[1], bool)
    for t in pick:
        q = int(rng.integers(0, 4))
        v = tets[q, t]
        if used[v]:
            continue
        others = [tets[k, t] for k in range(4) if k != q]
        a, b, c = (nodes[:, o] for o in others)
        nrm = np.cross(b - a, c - a)
        nn = np.linalg.norm(nrm)
        if nn == 0:
            continue
        nrm /= nn
        h = float(np.dot(nodes[:, v] - a, nrm))
        edge = max(np.linalg.norm(b - a), np.linalg.norm(c - a), np.linalg.norm(c - b))
        target = np.sign(h) * edge / sliver_aspect
        nodes[:, v] = nodes[:, v] - (h - target) * nrm
        used[v] = True
    tets = orient_positive(nodes, tets)
    vol = tet_signed_volumes(nodes, tets)
    if not (vol > 0).all():
        raise RuntimeError("sliver construction produced a zero-volume tet")
    f = Nedelec2Field(TetMesh(nodes, tets))
    # PML tensors from tet centroids
    cen = nodes[:, tets].mean(axis=1)  # (3, nT)
    k0 = 2 * np.pi * freq / C0
    s = np.ones((3, nT), np.complex128)
    for ax in range(3):
        L = size[ax]
        delta = shell * L
        smax = 2.0 / delta
        d = np.maximum(np.maximum(delta - cen[ax], cen[ax] - (L - delta)), 0.0)
        s[ax] = 1.0 - 1j * smax * (d / delta) ** 2 / k0
    diag = np.stack([s[1] * s[2] / s[0], s[2] * s[0] / s[1], s[0] * s[1] / s[2]])
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for a in range(3):
        er[a, a] = diag[a]
        ur[a, a] = diag[a]
    wl = Workload("wr90_pml_slivers", f, er, ur, np.zeros(0, np.int64), freq, tuple(n))
    wl.slivers = pick
    return wl


class HeatWorkload:
    """A Lagrange-2 heat-conduction case: a jittered box, a random symmetric
    positive-definite conductivity tensor and a rho_cp per tet."""

    def __init__(self, name, field, cond, rho_cp, hex_grid):
        self.name, self.field, self.cond, self.rho_cp, self.hex_grid = name, field, cond, rho_cp, hex_grid

    @property
    def n_tets(self) -> int:
        return int(self.field.mesh.n_tets)


def heat_box(n=(100, 50, 67), jitter=0.15, seed=6, size=(0.1, 0.05, 0.067)) -> HeatWorkload:
    from .heat import Legrange2

    nodes, tets = structured_box(*n, size=size, jitter=jitter, seed=seed)
    m = TetMesh(nodes, tets)
    rng = np.random.default_rng(seed)
    nT = m.n_tets
    cond = np.empty((3, 3, nT))
    for lo in range(0, nT, 1 << 20):  # Q Q^T + 0.5 I, blockwise to bound host memory
        hi = min(nT, lo + (1 << 20))
        Q = rng.normal(size=(hi - lo, 3, 3))
        cond[:, :, lo:hi] = np.einsum("nij,nkj->ikn", Q, Q) + 0.5 * np.eye(3)[:, :, None]
    rho_cp = rng.uniform(1e6, 4e6, nT)
    return HeatWorkload(f"heat_box_{nT // 1000}k", Legrange2(m), cond, rho_cp, tuple(n))


def heat_element_alg_bytes(n_nodes: int, n_tets: int, kind: str) -> int:
    """One Lagrange-2 element launch: node coordinates once, 4 node indices
    and the material per tet (9 or 1 f8), 100 f8 values written."""
    return 24 * n_nodes + n_tets * (16 + (72 if kind == "stiff" else 8) + 800)


def heat_gather_alg_bytes(n_tets: int, nnz: int) -> int:
    """One COO -> CSC gather: per slot its index (4 B) and value (8 B), per
    entry its run start (4 B) read and its value (8 B) written."""
    return n_tets * 100 * 12 + nnz * 12
