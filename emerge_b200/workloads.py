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


def alg_bytes(n_nodes: int, n_tets: int, nnz: int, material_bytes_per_tet: int = 16) -> int:
    """Algorithmic bytes of one assembly: nodes + tets + material + int32
    slot->nnz map + segment offsets + complex128 A written."""
    S = 400 * n_tets
    return 24 * n_nodes + 16 * n_tets + material_bytes_per_tet * n_tets + 4 * S + 4 * (nnz + 1) + 16 * nnz


def floor_bytes(n_nodes: int, n_tets: int, nnz: int, material_bytes_per_tet: int = 16) -> int:
    """Compulsory traffic without the mandated map: inputs + A written."""
    return 24 * n_nodes + 16 * n_tets + material_bytes_per_tet * n_tets + 16 * nnz
