"""Generate the golden fixtures by running the REFERENCE's own numba code.

Run in a container that holds the EMerge source tree (default
``/root/reference``)::

    python tests/golden/make_golden.py [--ref /root/reference]

Reference functions executed (unmodified, imported from the source tree):
``curlcurl._matrix_builder`` (curlcurl.py:387-456), ``CSCMapping.from_rowcol``
and ``CSCMapping.to_csc`` (csc_cast.py:51-63). Mesh topology comes from the
loop restatement of mesh3d.py:706-776 in ``oracle.oracle.topology_loops``
(the reference's ``Mesh3D`` needs gmsh); synthetic meshes come from
``emerge_b200.mesh.structured_box`` and their bytes are hashed into the
fixtures so that generator drift is detected.

Fixtures written next to this script:
* ``tiny.npz``       12 tets, some negatively oriented, non-symmetric complex
                     full er/ur tensors, one conductor tet excluded; every
                     output array in full.
* ``small_diag.npz`` 24 tets, diagonal complex tensors; full outputs.
* ``config0.json``   12x6x30 WR-90 box (12,960 tets, air, 10 GHz): pattern
                     hashes, norms of K, M, A and 4096 sampled entries.
* ``dielectric.json`` 6x4x8 box with blocky lossy dielectric: same summary.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from emerge_b200.mesh import structured_box  # noqa: E402
from oracle.oracle import topology_loops  # noqa: E402
from oracle.ref_loader import load_reference  # noqa: E402

C0 = 299792458.0
DOFCODES = np.array([64] * 6 + [66] * 6 + [128] * 4 + [129] * 4, dtype=np.int64)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_reference(R, nodes, tets, er, ur, conductor_tets, k0):
    edges, tris, t2e, t2t, t2f = topology_loops(tets)
    nT = tets.shape[1]
    tet_assy = np.arange(nT)
    if len(conductor_tets):
        tet_assy = np.delete(tet_assy, conductor_tets)
    dataE, dataB, rows, cols = R.curlcurl._matrix_builder(nodes, tets, tris, edges, t2f, t2e, t2t, ur, er,
                                                          tet_assy.astype(np.int64), DOFCODES)
    NF = 2 * edges.shape[1] + 2 * tris.shape[1]
    cmap = R.csc_cast.CSCMapping.from_rowcol(rows, cols, NF)
    K = cmap.to_csc(dataE)
    M = cmap.to_csc(dataB)
    A = cmap.to_csc(dataE - dataB * (k0 ** 2))
    return dict(dataE=dataE, dataB=dataB, rows=rows, cols=cols, indptr=np.asarray(A.indptr),
                indices=np.asarray(A.indices), K=np.asarray(K.data), M=np.asarray(M.data), A=np.asarray(A.data),
                NF=NF, edges=edges, tris=tris)


def rand_tensor(rng, nT, kind):
    if kind == "full":
        t = rng.uniform(0.5, 2.0, (3, 3, nT)) + 1j * rng.uniform(-0.3, 0.3, (3, 3, nT))
        t[0, 0] += 2.0
        t[1, 1] += 2.0
        t[2, 2] += 2.0
        return t.astype(np.complex128)
    t = np.zeros((3, 3, nT), dtype=np.complex128)
    for d in range(3):
        t[d, d] = rng.uniform(1.0, 4.0, nT) - 1j * rng.uniform(0.0, 0.5, nT)
    return t


def summary(out, k0, rng, nsample=4096):
    nnz = out["A"].shape[0]
    S = out["dataE"].shape[0]
    ids = np.sort(rng.choice(nnz, size=min(nsample, nnz), replace=False))
    sl = np.sort(rng.choice(S, size=min(nsample, S), replace=False))
    d = {"NF": int(out["NF"]), "nnz": int(nnz), "S": int(S), "k0": k0,
         "indptr_sha256_i64": sha(out["indptr"].astype(np.int64)),
         "indices_sha256_i64": sha(out["indices"].astype(np.int64)),
         "indptr_dtype": str(out["indptr"].dtype), "indices_dtype": str(out["indices"].dtype),
         "sample_nnz": ids.tolist(), "sample_slot": sl.tolist()}
    for key in ("K", "M", "A"):
        v = out[key]
        d[f"{key}_fro"] = float(np.linalg.norm(v))
        d[f"{key}_max"] = float(np.abs(v).max())
        d[f"{key}_sample_re"] = v[ids].real.tolist()
        d[f"{key}_sample_im"] = v[ids].imag.tolist()
    for key in ("dataE", "dataB"):
        d[f"{key}_sample_re"] = out[key][sl].real.tolist()
        d[f"{key}_sample_im"] = out[key][sl].imag.tolist()
    d["rows_sample"] = out["rows"][sl].tolist()
    d["cols_sample"] = out["cols"][sl].tolist()
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    R = load_reference(args.ref)
    k0 = 2 * np.pi * 10e9 / C0

    # tiny: negative orientations + non-symmetric full tensors + a conductor tet
    rng = np.random.default_rng(11)
    nodes, tets = structured_box(2, 1, 1, size=(2e-3, 1e-3, 1e-3), jitter=0.1, seed=11)
    tets = tets.copy()
    for t in (1, 4, 7):  # flip orientation of a few tets (swap two vertices)
        tets[[0, 1], t] = tets[[1, 0], t]
    nT = tets.shape[1]
    er, ur = rand_tensor(rng, nT, "full"), rand_tensor(rng, nT, "full")
    cond = np.array([3], dtype=np.int64)
    out = run_reference(R, nodes, tets, er, ur, cond, k0)
    np.savez_compressed(os.path.join(HERE, "tiny.npz"), nodes=nodes, tets=tets, er=er, ur=ur, conductor_tets=cond,
                        k0=k0, **{k: out[k] for k in ("dataE", "dataB", "rows", "cols", "indptr", "indices", "K", "M",
                                                     "A", "edges", "tris")})

    # small_diag: diagonal complex tensors, all positive
    rng = np.random.default_rng(5)
    nodes, tets = structured_box(1, 2, 2, size=(1e-3, 2e-3, 2e-3), jitter=0.1, seed=5)
    nT = tets.shape[1]
    er, ur = rand_tensor(rng, nT, "diag"), rand_tensor(rng, nT, "diag")
    out = run_reference(R, nodes, tets, er, ur, np.zeros(0, np.int64), k0)
    np.savez_compressed(os.path.join(HERE, "small_diag.npz"), nodes=nodes, tets=tets, er=er, ur=ur,
                        conductor_tets=np.zeros(0, np.int64), k0=k0,
                        **{k: out[k] for k in ("dataE", "dataB", "rows", "cols", "indptr", "indices", "K", "M", "A",
                                               "edges", "tris")})

    # config 0: WR-90 box, air, 10 GHz
    nodes, tets = structured_box(12, 6, 30, size=(22.86e-3, 10.16e-3, 50e-3), jitter=0.05, seed=0)
    nT = tets.shape[1]
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = 1.0
        ur[d, d] = 1.0
    out = run_reference(R, nodes, tets, er, ur, np.zeros(0, np.int64), k0)
    s = summary(out, k0, np.random.default_rng(123))
    s.update({"mesh": {"n": [12, 6, 30], "size": [22.86e-3, 10.16e-3, 50e-3], "jitter": 0.05, "seed": 0},
              "nodes_sha256": sha(nodes), "tets_sha256": sha(tets), "material": "air"})
    with open(os.path.join(HERE, "config0.json"), "w") as f:
        json.dump(s, f)

    # blocky lossy dielectric (config-1 style materials on a small box)
    rng = np.random.default_rng(7)
    nodes, tets = structured_box(6, 4, 8, size=(22.86e-3, 10.16e-3, 50e-3), jitter=0.15, seed=7)
    nT = tets.shape[1]
    hexid = np.arange(nT) // 6
    hi, hj, hk = hexid % 6, (hexid // 6) % 4, hexid // 24
    blk = (hi // 2) + 3 * ((hj // 2) + 2 * (hk // 2))
    nb = int(blk.max()) + 1
    eps_b = rng.uniform(1, 10, nb)
    tand_b = rng.uniform(1e-3, 1e-2, nb)
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = eps_b[blk] * (1 - 1j * tand_b[blk])
        ur[d, d] = 1.0
    out = run_reference(R, nodes, tets, er, ur, np.zeros(0, np.int64), k0)
    s = summary(out, k0, np.random.default_rng(321))
    s.update({"mesh": {"n": [6, 4, 8], "size": [22.86e-3, 10.16e-3, 50e-3], "jitter": 0.15, "seed": 7},
              "nodes_sha256": sha(nodes), "tets_sha256": sha(tets), "material": "blocky lossy dielectric",
              "eps_blocks": eps_b.tolist(), "tand_blocks": tand_b.tolist(), "block_of_tet_sha256": sha(blk)})
    with open(os.path.join(HERE, "dielectric.json"), "w") as f:
        json.dump(s, f)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
