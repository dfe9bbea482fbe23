"""Helpers to load the golden fixtures (made by tests/golden/make_golden.py
from the reference's own numba code) and rebuild their inputs."""
import json
import os

import numpy as np

from emerge_b200.mesh import Nedelec2Field, TetMesh, structured_box

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
C0 = 299792458.0


def load_npz(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def field_from(nodes, tets):
    return Nedelec2Field(TetMesh(nodes, tets))


def config0_inputs():
    nodes, tets = structured_box(12, 6, 30, size=(22.86e-3, 10.16e-3, 50e-3), jitter=0.05, seed=0)
    nT = tets.shape[1]
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = 1.0
        ur[d, d] = 1.0
    return nodes, tets, er, ur


def dielectric_inputs(g):
    nodes, tets = structured_box(6, 4, 8, size=(22.86e-3, 10.16e-3, 50e-3), jitter=0.15, seed=7)
    nT = tets.shape[1]
    hexid = np.arange(nT) // 6
    hi, hj, hk = hexid % 6, (hexid // 6) % 4, hexid // 24
    blk = (hi // 2) + 3 * ((hj // 2) + 2 * (hk // 2))
    eps_b = np.array(g["eps_blocks"])
    tand_b = np.array(g["tand_blocks"])
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = eps_b[blk] * (1 - 1j * tand_b[blk])
        ur[d, d] = 1.0
    return nodes, tets, er, ur, blk


def rel_err(x, ref):
    x = np.asarray(x)
    ref = np.asarray(ref)
    fro = np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300)
    mx = np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300) if ref.size else 0.0
    return fro, mx
