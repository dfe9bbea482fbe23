"""Serving engine on the GPU: each job's A(f) is bitwise the same whether the
job runs alone or mixed with other jobs in shared batches, and equals the
drop-in's to_csc(Evec - Bvec*k0**2) within the plain-FP64 tolerance."""
import numpy as np
import pytest

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.serving import C0, AssemblyJob, AssemblyServer, latency_summary
from tests.golden_util import rel_err

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12


def _specs():
    a = W.wr90_air(n=(6, 4, 10))
    b = W.wr90_dielectric(n=(8, 5, 9), seed=3)
    c = W.wr90_pml_slivers(n=(10, 6, 6))
    d = W.wr90_air(n=(12, 6, 30), seed=5)
    cond = np.arange(0, d.n_tets, 97, dtype=np.int64)  # a scattered conductor set
    return [
        (a, np.linspace(8e9, 12e9, 5), np.zeros(0, np.int64)),
        (b, np.array([9.5e9, 10e9, 10.5e9]), np.zeros(0, np.int64)),
        (c, np.linspace(9e9, 11e9, 7), np.zeros(0, np.int64)),
        (d, np.array([7e9, 13e9]), cond),
    ]


def _jobs(specs):
    return [AssemblyJob(wl.field, wl.er, wl.ur, f, cond, keep_results=True, job_id=i)
            for i, (wl, f, cond) in enumerate(specs)]


@pytest.fixture(scope="module")
def alone():
    specs = _specs()
    out = []
    with AssemblyServer(precision="fp64", budget_bytes=8e9) as srv:
        for j in _jobs(specs):
            srv.submit(j)
            srv.wait([j], timeout=120)
            out.append(j)
    return specs, out


def _assert_same(jobs, ref):
    for j, r in zip(jobs, ref):
        assert sorted(j.results) == list(range(len(j.freqs)))
        assert np.array_equal(j.indptr, r.indptr) and np.array_equal(j.indices, r.indices)
        for fi in range(len(j.freqs)):
            assert np.array_equal(j.results[fi], r.results[fi]), (j.job_id, fi)


def test_alone_matches_dropin(alone):
    specs, jobs = alone
    for (wl, freqs, cond), j in zip(specs, jobs):
        E, B, cmap = tet_mass_stiffness_matrices(wl.field, wl.er, wl.ur, cond)
        assert np.array_equal(j.indptr, cmap.indptr) and np.array_equal(j.indices, cmap.indices)
        for fi, f in enumerate(freqs):
            k0 = 2 * np.pi * f / C0
            ref = cmap.to_csc(E - B * k0 ** 2).data
            fro, mx = rel_err(j.results[fi], ref)
            assert fro <= TOL_FP64 and mx <= TOL_FP64, (j.job_id, fi, fro, mx)


@pytest.mark.parametrize("max_items,slots,graph", [(5, 2, True), (512, 4, True), (3, 1, False)])
def test_mix_bitwise_equal_to_alone(alone, max_items, slots, graph):
    specs, ref = alone
    with AssemblyServer(precision="fp64", budget_bytes=8e9, max_items=max_items, slots_per_job=slots,
                        use_graph=graph) as srv:
        jobs = [srv.submit(j) for j in _jobs(specs)]
        srv.wait(jobs, timeout=120)
        assert srv.n_items == sum(len(j.freqs) for j in jobs)
        if max_items < 10:
            assert srv.n_batches >= sum(len(j.freqs) for j in jobs) // max_items
        srv.drop_mesh_cache()
        assert srv.in_use == 0
    _assert_same(jobs, ref)
    s = latency_summary(jobs)
    assert s["jobs"] == len(jobs) and s["p99_ms"] >= s["p50_ms"] > 0


def test_budget_admission_fifo(alone):
    specs, ref = alone
    jobs = _jobs(specs)
    need = max(j.footprint(0, 2) for j in jobs)
    budget = int(need * 1.05)  # room for one job at a time
    with AssemblyServer(precision="fp64", budget_bytes=budget, slots_per_job=2) as srv:
        for j in jobs:
            srv.submit(j)
        srv.wait(jobs, timeout=120)
        assert srv.peak_in_use <= budget
    # FIFO: admission order is submission order
    adm = [j.t_admitted for j in jobs]
    assert adm == sorted(adm)
    _assert_same(jobs, ref)


def test_job_over_budget_is_rejected():
    wl = W.wr90_air(n=(6, 4, 10))
    with AssemblyServer(precision="fp64", budget_bytes=1 << 20) as srv:
        j = srv.submit(AssemblyJob(wl.field, wl.er, wl.ur, np.array([10e9])))
        with pytest.raises(MemoryError):
            srv.wait([j], timeout=60)


def test_mixed_precision_jobs_alone_vs_mix():
    specs = _specs()[:3]
    with AssemblyServer(precision="mixed", budget_bytes=8e9) as srv:
        ref = []
        for j in _jobs(specs):
            srv.submit(j)
            srv.wait([j], timeout=120)
            ref.append(j)
    with AssemblyServer(precision="mixed", budget_bytes=8e9, max_items=4, slots_per_job=2) as srv:
        jobs = [srv.submit(j) for j in _jobs(specs)]
        srv.wait(jobs, timeout=120)
    _assert_same(jobs, ref)
    for (wl, freqs, cond), j in zip(specs, jobs):
        E, B, cmap = tet_mass_stiffness_matrices(wl.field, wl.er, wl.ur, cond)
        k0 = 2 * np.pi * freqs[0] / C0
        fro, mx = rel_err(j.results[0], cmap.to_csc(E - B * k0 ** 2).data)
        assert fro <= 1e-6 and mx <= 1e-6


def test_shared_meshes_and_batched_setup(alone):
    """Jobs on one mesh share its resident entry (built once); results stay
    bitwise those of the jobs run alone, and scalar materials give what the
    reference's [3, 3, nT] tensors give."""
    specs, ref = alone
    with AssemblyServer(precision="fp64", budget_bytes=8e9) as srv:
        jobs = [srv.submit(j) for j in _jobs(specs) + _jobs(specs)]
        srv.wait(jobs, timeout=120)
        assert srv.n_mesh_builds == len(specs)
        assert 1 <= srv.n_km_batches <= len(jobs)
    _assert_same(jobs[:len(specs)], ref)
    _assert_same(jobs[len(specs):], ref)
    wl, freqs, cond = specs[1]  # isotropic dielectric
    scalar = AssemblyJob(wl.field, wl.er[0, 0].copy(), None, freqs, cond, keep_results=True)
    with AssemblyServer(precision="fp64", budget_bytes=8e9) as srv:
        srv.submit(scalar)
        srv.wait([scalar], timeout=120)
    _assert_same([scalar], [ref[1]])
