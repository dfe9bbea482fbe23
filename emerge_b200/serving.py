"""Serving engine: continuous batching of Nedelec-2 assembly jobs on one GPU.

A job is what EMerge's frequency sweep asks for (microwave_3d.py:1280 ->
assembler.py:391-494 per frequency): a mesh, per-tet materials and a list of
frequencies; its result is A(f) = K - k0(f)^2 M for every frequency, on the
device (latency = arrival -> last A(f) ready).

* Admission: jobs wait in FIFO order until their HBM footprint fits in the
  budget; finished jobs return their share.
* Setup (one worker thread and CUDA stream per in-flight setup): upload,
  pattern + gather plan, K and M assembled once and kept resident.
* Batching: one batcher thread packs ready (job, frequency) items of every
  active job - jobs that arrived while others were running included - into a
  single persistent-grid launch (``emg_form_batch``). The launch and the copy
  of its descriptor are captured once in a CUDA graph and replayed per batch.
  Each job has a few output slots; an item writes one slot and frees it when
  the result has been handed over.

Results are deterministic: every kernel sums in a fixed order and a batch's
items are independent, so a job's A(f) is bitwise the same alone and in a mix.
"""
from __future__ import annotations

import ctypes
import queue
import threading
import time
from collections import deque
from dataclasses import dataclass, field as dfield

import numpy as np
import torch

from . import _lib as L
from .assembly import DeviceMaterial, DeviceMesh, GpuCSCMapping, _Job, _prec

C0 = 299792458.0


@dataclass
class AssemblyJob:
    """One request: mesh (a Nedelec2 field), per-tet er/ur c16[3,3,nT], the
    frequencies in Hz, optionally conductor tets."""

    field: object
    er: np.ndarray
    ur: np.ndarray
    freqs: np.ndarray
    conductor_tets: np.ndarray = dfield(default_factory=lambda: np.zeros(0, np.int64))
    keep_results: bool = False
    job_id: int = -1
    # filled by the server
    arrival: float = 0.0
    t_admitted: float = 0.0
    t_setup: float = 0.0
    t_done: float = 0.0
    results: dict = dfield(default_factory=dict)
    error: BaseException | None = None
    done: threading.Event = dfield(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival

    @property
    def n_tets(self) -> int:
        return int(self.field.ntets)

    def footprint(self, precision: int, slots: int) -> int:
        """HBM bytes this job holds while active (plan, pattern, K, M, element
        workspace, output slots, mesh and materials), an upper estimate."""
        m = self.field.mesh
        nT, E, F = m.n_tets, m.n_edges, m.n_tris
        nnz = nnz_of(nT, E, F)
        items = 10 * nT
        plan = 4 * (E + F) * 2 + items * (16 + 40 + 40 + 160)
        pattern = 4 * (2 * E + 2 * F + 1) + 4 * nnz
        values = 210 * nT * (8 if precision == L.EMG_MIXED else 16)
        return int(plan + pattern + values + (2 + slots) * 16 * nnz + 24 * m.n_nodes + 64 * nT + (64 << 20))


def nnz_of(n_tets: int, n_edges: int, n_tris: int) -> int:
    """Nonzeros of the Nedelec-2 pattern of a conforming mesh with every tet
    assembled. Entity pairs that share a tet: edge-edge E + 2(3F + 3T) (pairs
    sharing a vertex lie in one face, opposite pairs in one tet), edge-face
    2(3F + 12T), face-face F + 2*6T; each entity pair carries 2x2 DoFs."""
    return 4 * (n_edges + 13 * n_tris + 42 * n_tets)


class _Active:
    """Device state of an admitted job."""

    def __init__(self, job: AssemblyJob, slots: int):
        self.job = job
        self.cmap = None
        self.K = self.M = None
        self.out = []
        self.free_slots = deque(range(slots))
        self.next_f = 0
        self.n_done = 0


class AssemblyServer:
    """Continuous-batching assembly server (see module docstring)."""

    def __init__(self, device=0, budget_bytes: float = 120e9, setup_workers: int = 3, precision: str = "mixed",
                 slots_per_job: int = 4, max_items: int = 512, use_graph: bool = True):
        self.dev = torch.device("cuda", device)
        self.budget = int(budget_bytes)
        self.precision = _prec(precision)
        self.slots = slots_per_job
        self.max_items = max_items
        self.use_graph = use_graph
        self._lock = threading.Lock()
        self._pending: deque[AssemblyJob] = deque()
        self._in_use = 0
        self.peak_in_use = 0
        self._setup_q: queue.Queue = queue.Queue()
        self._active: list[_Active] = []
        self._stop = threading.Event()
        self._wake = threading.Event()
        self.completed: list[AssemblyJob] = []
        self.n_batches = 0
        self.n_items = 0
        # batch descriptors: pinned host copy and device copy at fixed addresses
        isz = ctypes.sizeof(L.FormItem)
        self._h_items = torch.zeros(max_items * isz, dtype=torch.uint8, pin_memory=True)
        self._h_tiles = torch.zeros(max_items + 1, dtype=torch.int64, pin_memory=True)
        self._h_n = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self._d_items = torch.zeros(max_items * isz, dtype=torch.uint8, device=self.dev)
        self._d_tiles = torch.zeros(max_items + 1, dtype=torch.int64, device=self.dev)
        self._d_n = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._items_view = (L.FormItem * max_items).from_address(self._h_items.data_ptr())
        self._batch_stream = torch.cuda.Stream(self.dev)
        self._graph = None
        if use_graph:
            # an empty batch (n = 0) initialises the launch path, then the
            # descriptor copies + the persistent launch are captured once
            with torch.cuda.stream(self._batch_stream):
                self._issue()
            self._batch_stream.synchronize()
            self._graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self._graph, stream=self._batch_stream):
                self._issue()
        self._threads = [threading.Thread(target=self._setup_loop, daemon=True) for _ in range(setup_workers)]
        self._threads.append(threading.Thread(target=self._batch_loop, daemon=True))
        for t in self._threads:
            t.start()

    # ------------------------------------------------------------ public
    def submit(self, job: AssemblyJob) -> AssemblyJob:
        job.arrival = time.perf_counter()
        with self._lock:
            self._pending.append(job)
        self._admit()
        return job

    def wait(self, jobs, timeout: float | None = None) -> None:
        for j in jobs:
            if not j.done.wait(timeout):
                raise TimeoutError(f"job {j.job_id} did not finish")
            if j.error is not None:
                raise j.error

    def close(self) -> None:
        self._stop.set()
        self._wake.set()
        for _ in range(len(self._threads)):
            self._setup_q.put(None)
        for t in self._threads:
            t.join(timeout=30)
        self._graph = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def in_use(self) -> int:
        return self._in_use

    # ------------------------------------------------------------ admission
    def _admit(self) -> None:
        admitted = []
        with self._lock:
            while self._pending:
                j = self._pending[0]
                need = j.footprint(self.precision, self.slots)
                if need > self.budget:
                    self._pending.popleft()
                    j.error = MemoryError(f"job {j.job_id} needs {need} B, over the {self.budget} B budget")
                    j.done.set()
                    continue
                if self._in_use + need > self.budget:
                    break  # FIFO: wait for memory
                self._pending.popleft()
                self._in_use += need
                self.peak_in_use = max(self.peak_in_use, self._in_use)
                j._need = need
                j.t_admitted = time.perf_counter()
                admitted.append(j)
        for j in admitted:
            self._setup_q.put(j)

    def _release(self, act: _Active) -> None:
        j = act.job
        act.K = act.M = act.cmap = None
        act.out = []
        with self._lock:
            self._in_use -= j._need
            self._active.remove(act)
        j.t_done = time.perf_counter()
        self.completed.append(j)
        j.done.set()
        self._admit()

    # ------------------------------------------------------------ setup workers
    def _setup_loop(self) -> None:
        torch.cuda.set_device(self.dev)
        stream = torch.cuda.Stream(self.dev)
        while not self._stop.is_set():
            j = self._setup_q.get()
            if j is None:
                return
            act = _Active(j, self.slots)
            try:
                with torch.cuda.stream(stream):
                    dmesh = DeviceMesh(j.field, j.conductor_tets, self.dev)
                    cmap = GpuCSCMapping(dmesh)
                    dmat = DeviceMaterial(j.er, j.ur, dmesh.n_tets, self.dev)
                    job = _Job(dmesh, dmat, self.precision)
                    act.K = cmap.assemble_device(job, 1.0 + 0j, 0j)
                    act.M = cmap.assemble_device(job, 0j, 1.0 + 0j)
                    cmap._ws = None  # element workspace no longer needed
                    act.out = [torch.empty(max(cmap.nnz, 1), dtype=torch.complex128, device=self.dev)
                               for _ in range(self.slots)]
                    act.cmap = cmap
                    stream.synchronize()
                    dmesh.check_status()
                j.t_setup = time.perf_counter()
            except BaseException as e:  # reported on the job, the server keeps serving
                j.error = e
                with self._lock:
                    self._in_use -= j._need
                j.done.set()
                self._admit()
                continue
            with self._lock:
                self._active.append(act)
            self._wake.set()

    # ------------------------------------------------------------ batcher
    def _collect(self):
        batch = []
        with self._lock:
            for act in self._active:
                j = act.job
                while act.free_slots and act.next_f < len(j.freqs) and len(batch) < self.max_items:
                    batch.append((act, act.next_f, act.free_slots.popleft()))
                    act.next_f += 1
        return batch

    def _launch(self, batch) -> None:
        tiles = 0
        self._h_tiles[0] = 0
        for i, (act, fi, slot) in enumerate(batch):
            k0 = 2 * np.pi * float(act.job.freqs[fi]) / C0
            it = self._items_view[i]
            it.K, it.M, it.P = act.K.data_ptr(), act.M.data_ptr(), None
            it.out = act.out[slot].data_ptr()
            it.nnz = act.cmap.nnz
            it.coef[:] = (1.0, 0.0, -k0 * k0, 0.0, 0.0, 0.0)
            tiles += (act.cmap.nnz + L.FORM_TILE - 1) // L.FORM_TILE
            self._h_tiles[i + 1] = tiles
        self._h_n[0] = len(batch)
        with torch.cuda.stream(self._batch_stream):
            if self._graph is not None:
                self._graph.replay()
            else:
                self._issue()
        self._batch_stream.synchronize()

    def _issue(self) -> None:
        self._d_items.copy_(self._h_items, non_blocking=True)
        self._d_tiles.copy_(self._h_tiles, non_blocking=True)
        self._d_n.copy_(self._h_n, non_blocking=True)
        L.check(L.lib().emg_form_batch(L.ptr(self._d_items), L.ptr(self._d_tiles), L.ptr(self._d_n), self.max_items,
                                       L.stream_handle(self.dev)))

    def _batch_loop(self) -> None:
        torch.cuda.set_device(self.dev)
        while not self._stop.is_set():
            batch = self._collect()
            if not batch:
                self._wake.wait(0.005)
                self._wake.clear()
                continue
            try:
                self._launch(batch)
            except BaseException as e:
                for act, _, _ in batch:
                    act.job.error = e
                    self._release(act)
                continue
            self.n_batches += 1
            self.n_items += len(batch)
            finished = []
            for act, fi, slot in batch:
                j = act.job
                if j.keep_results:
                    j.results[fi] = act.out[slot][: act.cmap.nnz].cpu().numpy()
                act.n_done += 1
                with self._lock:
                    act.free_slots.append(slot)
                if act.n_done == len(j.freqs):
                    finished.append(act)
            for act in finished:
                if act.job.keep_results:
                    act.job.indptr, act.job.indices = act.cmap.indptr, act.cmap.indices
                self._release(act)


def latency_summary(jobs) -> dict:
    lat = np.array([j.latency for j in jobs]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "jobs": int(lat.size)}


# ---------------------------------------------------------------- synthetic stream
def box_grid(n_tets: int, size=(22.86e-3, 10.16e-3, 50e-3)) -> tuple:
    """Hex grid (nx, ny, nz) of a WR-90-proportioned box with about n_tets
    Kuhn tets (6 per hex)."""
    h = max(n_tets / 6.0, 1.0)
    ax, az = size[0] / size[1], size[2] / size[1]
    ny = max(1, int(round((h / (ax * az)) ** (1.0 / 3.0))))
    nx = max(1, int(round(ax * ny)))
    nz = max(1, int(round(h / (nx * ny))))
    return nx, ny, nz


def synthetic_stream(n_jobs: int = 50, rate: float = 50.0, tets=(5_000, 500_000), n_freq=(1, 64),
                     freq_hz=(1e9, 40e9), n_sizes: int = 16, seed: int = 0):
    """Seeded job list of a serving stream: Poisson arrivals (mean ``rate``
    jobs/s), tet counts log-uniform in ``tets`` (snapped to ``n_sizes``
    log-spaced box meshes, each built once and shared), eps_r ~ U[1,12] and
    tan(delta) ~ U[0,1e-2] per 8x8x8-cell block, mu_r = 1, a U{n_freq}
    number of frequencies ~ U[freq_hz]. Returns (jobs, arrival offsets in s)."""
    from .mesh import Nedelec2Field, TetMesh, structured_box
    from .workloads import block_ids

    rng = np.random.default_rng(seed)
    sizes = np.geomspace(tets[0], tets[1], n_sizes)
    meshes = {}
    jobs, t, arrivals = [], 0.0, []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        target = float(np.exp(rng.uniform(np.log(tets[0]), np.log(tets[1]))))
        k = int(np.argmin(np.abs(np.log(sizes) - np.log(target))))
        if k not in meshes:
            grid = box_grid(int(sizes[k]))
            nodes, tt = structured_box(*grid, jitter=0.1, seed=100 + k)
            meshes[k] = (Nedelec2Field(TetMesh(nodes, tt)), grid)
        field, grid = meshes[k]
        nT = field.ntets
        blk = block_ids(*grid)
        nb = int(blk.max()) + 1
        eps = rng.uniform(1.0, 12.0, nb) * (1 - 1j * rng.uniform(0.0, 1e-2, nb))
        er = np.zeros((3, 3, nT), np.complex128)
        ur = np.zeros((3, 3, nT), np.complex128)
        for d in range(3):
            er[d, d] = eps[blk]
            ur[d, d] = 1.0
        nf = int(rng.integers(n_freq[0], n_freq[1] + 1))
        freqs = np.sort(rng.uniform(freq_hz[0], freq_hz[1], nf))
        jobs.append(AssemblyJob(field, er, ur, freqs, job_id=i))
        arrivals.append(t)
    return jobs, np.array(arrivals)


def run_stream(server: AssemblyServer, jobs, arrivals, timeout: float = 600.0) -> dict:
    """Submit ``jobs`` at their arrival offsets (wall clock), wait for all and
    summarise: makespan, tets/s, tet-frequencies/s, latency percentiles."""
    t0 = time.perf_counter()
    for j, a in zip(jobs, arrivals):
        d = t0 + a - time.perf_counter()
        if d > 0:
            time.sleep(d)
        server.submit(j)
    server.wait(jobs, timeout)
    t1 = max(j.t_done for j in jobs)
    span = t1 - t0
    n_t = sum(j.n_tets for j in jobs)
    n_tf = sum(j.n_tets * len(j.freqs) for j in jobs)
    out = {"makespan_s": span, "tets_per_s": n_t / span, "tet_freqs_per_s": n_tf / span,
           "jobs": len(jobs), "tets": n_t, "tet_freqs": n_tf, "freqs": int(sum(len(j.freqs) for j in jobs)),
           "batches": server.n_batches, "items": server.n_items, "peak_budget_bytes": server.peak_in_use,
           "arrival_span_s": float(arrivals[-1]) if len(arrivals) else 0.0}
    out.update(latency_summary(jobs))
    return out
