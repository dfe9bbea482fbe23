"""Serving engine: continuous batching of Nedelec-2 assembly jobs on one GPU.

A job is what EMerge's frequency sweep asks for (microwave_3d.py:1280 ->
assembler.py:391-494 per frequency): a mesh, per-tet materials and a list of
frequencies; its result is A(f) = K - k0(f)^2 M for every frequency, on the
device (latency = arrival -> last A(f) ready).

* Admission: jobs wait in FIFO order until their HBM footprint fits in the
  budget; finished jobs return their share. A job's footprint is its own
  arrays (materials, K, M, element-value workspaces, output slots) plus, when
  its mesh is not resident yet, the mesh's (coordinates, tets, pattern and
  gather plan).
* Mesh cache: a mesh's device arrays and plan are built once and shared by
  every job on that mesh (the reference caches its CSCMapping the same way
  across a sweep); an entry no job uses is evicted, least recently used
  first, when an admission needs its memory.
* Setup (worker threads, one CUDA stream each): the mesh entry (built or
  reused) and the job's materials are uploaded; the job then waits for the
  batcher.
* Batching: one batcher thread (a) assembles K and M of every job whose
  setup finished since its last pass -- all of them in one element-kernel
  launch and one gather launch over a job table (``emg_assemble_batch``) --
  and (b) packs ready (job, frequency) items of every active job into one
  forming launch (``emg_form_batch``); jobs with the least remaining work go
  first and a batch is capped in size. The forming launch and the copy of
  its descriptor are captured once in a CUDA graph and replayed per batch.
  Each job has a few output slots; an item writes one slot and frees it when
  the result has been handed over. A job's items in one batch form a group:
  every tile reads that job's K and M once and writes all the group's
  outputs.

Results are deterministic: every kernel sums in a fixed order and a batch's
jobs and items are independent, so a job's A(f) is bitwise the same alone and
in a mix.
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
    """One request: mesh (a Nedelec2 field), per-tet er/ur -- c16[3,3,nT]
    tensors, or c16[nT] scalar er with ur None for isotropic materials --
    the frequencies in Hz, optionally conductor tets."""

    field: object
    er: np.ndarray
    ur: np.ndarray | None
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
    setup_parts: dict = dfield(default_factory=dict)
    error: BaseException | None = None
    done: threading.Event = dfield(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival

    def materials(self):
        """(er, ur) as DeviceMaterial takes them: c16[3, 3, nT] tensors, or
        c16[nT] scalar er with ur None (mu_r = 1) or c16[nT]."""
        return self.er, self.ur

    def tensors(self):
        """(er, ur) in the reference's c16[3, 3, nT] layout."""
        er = np.asarray(self.er)
        if er.ndim == 3:
            return er, np.asarray(self.ur)
        nT = er.shape[0]
        out = np.zeros((3, 3, nT), np.complex128), np.zeros((3, 3, nT), np.complex128)
        ur = np.ones(nT, np.complex128) if self.ur is None else np.asarray(self.ur)
        for d in range(3):
            out[0][d, d] = er
            out[1][d, d] = ur
        return out

    @property
    def n_tets(self) -> int:
        return int(self.field.ntets)

    @property
    def mesh_key(self):
        """Jobs with the same key share one resident mesh entry: the same
        mesh object and the same conductor (excluded) tets."""
        c = np.unique(np.asarray(self.conductor_tets, dtype=np.int64))
        return (id(self.field), hash(c.tobytes()))

    def _n_assy(self) -> int:
        return int(self.field.mesh.n_tets) - int(np.unique(np.asarray(self.conductor_tets)).size)

    def mesh_footprint(self) -> int:
        """Device bytes of the mesh entry: coordinates, tets, tetids, status,
        topology (during the build), plan and its workspace, pattern; each
        rounded up to the arena alignment."""
        m = self.field.mesh
        nT, nN, E, F = m.n_tets, m.n_nodes, m.n_edges, m.n_tris
        nA = self._n_assy()
        p = L.Plan()
        L.check(L.lib().emg_plan_init(nT, nA, E, F, L.ctypes.byref(p)))
        sizes = [24 * nN, 16 * nT, 4 * nA, 16, 24 * nT, 16 * nT, p.plan_bytes, p.workspace_bytes,
                 4 * (2 * E + 2 * F + 1), 4 * nnz_of(nT, E, F)]
        return int(sum(-(-x // ARENA_ALIGN) * ARENA_ALIGN for x in sizes))

    def job_footprint(self, precision: int, slots: int) -> int:
        """Device bytes of the job's own arrays: materials (full tensors
        assumed), the element-value workspaces of K and M, K, M and the
        output slots, and its status word."""
        m = self.field.mesh
        nT, E, F = m.n_tets, m.n_edges, m.n_tris
        nnz = nnz_of(nT, E, F)
        ws = L.lib().emg_assemble_workspace_size(self._n_assy(), precision)
        sizes = [144 * nT, 144 * nT, ws, ws, 16] + [16 * nnz] * (2 + slots)
        return int(sum(-(-x // ARENA_ALIGN) * ARENA_ALIGN for x in sizes))

    def footprint(self, precision: int, slots: int) -> int:
        """Upper bound of the device bytes the job needs on a cold cache."""
        return self.mesh_footprint() + self.job_footprint(precision, slots)


ARENA_ALIGN = 256


class DeviceArena:
    """One device buffer allocated when the server starts, carved into one
    contiguous block per admitted job (first fit, freed blocks coalesce).
    Serving then calls no cudaMalloc / cudaFree, which would synchronise the
    device, and admission is exact: a job starts when its block fits."""

    def __init__(self, nbytes: int, device):
        self.size = -(-int(nbytes) // ARENA_ALIGN) * ARENA_ALIGN
        self.buf = torch.empty(max(self.size, ARENA_ALIGN), dtype=torch.uint8, device=device)
        self._free = [(0, self.size)]  # (offset, bytes), sorted by offset
        self.in_use = 0
        self.peak = 0

    def reserve(self, nbytes: int):
        """Offset of a free block of nbytes (rounded up), or None."""
        n = -(-int(nbytes) // ARENA_ALIGN) * ARENA_ALIGN
        for i, (off, sz) in enumerate(self._free):
            if sz >= n:
                if sz == n:
                    self._free.pop(i)
                else:
                    self._free[i] = (off + n, sz - n)
                self.in_use += n
                self.peak = max(self.peak, self.in_use)
                return ArenaBlock(self, off, n)
        return None

    def release(self, block: "ArenaBlock") -> None:
        off, n = block.off, block.n
        i = 0
        while i < len(self._free) and self._free[i][0] < off:
            i += 1
        self._free.insert(i, (off, n))
        if i + 1 < len(self._free) and self._free[i][0] + self._free[i][1] == self._free[i + 1][0]:
            self._free[i] = (off, n + self._free.pop(i + 1)[1])
        if i > 0 and self._free[i - 1][0] + self._free[i - 1][1] == self._free[i][0]:
            self._free[i - 1] = (self._free[i - 1][0], self._free[i - 1][1] + self._free.pop(i)[1])
        self.in_use -= n


class ArenaBlock:
    """A job's block; calling it hands out aligned tensors front to back."""

    def __init__(self, arena: DeviceArena, off: int, n: int):
        self.arena, self.off, self.n, self.top = arena, off, n, 0

    def __call__(self, numel: int, dtype: torch.dtype) -> torch.Tensor:
        nbytes = int(numel) * dtype.itemsize
        start = self.top
        self.top = start + -(-max(nbytes, 1) // ARENA_ALIGN) * ARENA_ALIGN
        if self.top > self.n:
            raise MemoryError("job block overflow (footprint bound violated)")
        o = self.off + start
        return self.arena.buf[o:o + nbytes].view(dtype)


def nnz_of(n_tets: int, n_edges: int, n_tris: int) -> int:
    """Nonzeros of the Nedelec-2 pattern of a conforming mesh with every tet
    assembled. Entity pairs that share a tet: edge-edge E + 2(3F + 3T) (pairs
    sharing a vertex lie in one face, opposite pairs in one tet), edge-face
    2(3F + 12T), face-face F + 2*6T; each entity pair carries 2x2 DoFs."""
    return 4 * (n_edges + 13 * n_tris + 42 * n_tets)


class _MeshEntry:
    """A resident mesh: its device arrays and plan (one arena block), shared
    by the admitted jobs on that mesh."""

    def __init__(self, key, block: "ArenaBlock"):
        self.key, self.block = key, block
        self.dmesh = None
        self.cmap = None
        self.users = 0  # admitted jobs holding it
        self.last_used = 0.0
        self.ready = threading.Event()
        self.error: BaseException | None = None


class _Active:
    """Device state of an admitted job."""

    def __init__(self, job: AssemblyJob, slots: int):
        self.job = job
        self.cmap = None
        self.dmat = None
        self.K = self.M = None
        self.ws_K = self.ws_M = None
        self.status = None
        self.out = []
        self.free_slots = deque(range(slots))
        self.next_f = 0
        self.n_done = 0


class AssemblyServer:
    """Continuous-batching assembly server (see module docstring)."""

    def __init__(self, device=0, budget_bytes: float = 120e9, setup_workers: int = 3, precision: str = "mixed",
                 slots_per_job: int = 4, max_items: int = 512, use_graph: bool = True, max_batch_nnz: int = 1 << 28,
                 max_assembly_jobs: int = 64):
        self.dev = torch.device("cuda", device)
        self.budget = int(budget_bytes)
        self.precision = _prec(precision)
        self.slots = slots_per_job
        self.max_items = max_items
        self.use_graph = use_graph
        self.max_batch_nnz = int(max_batch_nnz)
        self._lock = threading.Lock()
        self._pending: deque[AssemblyJob] = deque()
        self.arena = DeviceArena(self.budget, self.dev)
        self.peak_in_use = 0
        self._setup_q: queue.Queue = queue.Queue()
        self._meshes: dict = {}  # mesh key -> _MeshEntry
        self._ready_km: list[_Active] = []  # set up, waiting for the batched K/M assembly
        self._active: list[_Active] = []
        self.n_km_batches = 0
        self.n_mesh_builds = 0
        # job table of the batched K/M assembly (two entries per job): pinned
        # host copy and device copy, sized once
        self.max_km = int(max_assembly_jobs)
        tb = int(L.lib().emg_assemble_batch_table_bytes(2 * self.max_km))
        self._km_h = torch.zeros(tb, dtype=torch.uint8, pin_memory=True)
        self._km_d = torch.zeros(tb, dtype=torch.uint8, device=self.dev)
        self._km_desc = (L.AssemblyJobDesc * (2 * self.max_km))()
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
            # descriptor copies + the batch launch are captured once
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
        self.arena = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def in_use(self) -> int:
        return self.arena.in_use

    def drop_mesh_cache(self) -> None:
        """Evict every resident mesh no admitted job uses."""
        with self._lock:
            for key, e in list(self._meshes.items()):
                if e.users == 0 and e.ready.is_set():
                    del self._meshes[key]
                    e.dmesh = e.cmap = None
                    self.arena.release(e.block)

    # ------------------------------------------------------------ admission
    def _reserve(self, sizes):
        """Arena blocks of the given sizes, evicting resident meshes no job
        uses (least recently used first) until they fit; None if they do not
        fit even then. Called with the lock held."""
        while True:
            blocks = []
            for n in sizes:
                b = self.arena.reserve(n)
                if b is None:
                    break
                blocks.append(b)
            if len(blocks) == len(sizes):
                return blocks
            for b in blocks:
                self.arena.release(b)
            idle = [e for e in self._meshes.values() if e.users == 0 and e.ready.is_set()]
            if not idle:
                return None
            victim = min(idle, key=lambda e: e.last_used)
            del self._meshes[victim.key]
            victim.dmesh = victim.cmap = None
            self.arena.release(victim.block)

    def _admit(self) -> None:
        admitted = []
        with self._lock:
            while self._pending:
                j = self._pending[0]
                key = j.mesh_key
                entry = self._meshes.get(key)
                need_j = j.job_footprint(self.precision, self.slots)
                need_m = 0 if entry is not None else j.mesh_footprint()
                if need_j + need_m > self.arena.size:
                    self._pending.popleft()
                    j.error = MemoryError(f"job {j.job_id} needs {need_j + need_m} B, over the "
                                          f"{self.arena.size} B budget")
                    j.done.set()
                    continue
                blocks = self._reserve([need_j] + ([need_m] if need_m else []))
                if blocks is None:
                    break  # FIFO: wait for memory
                self._pending.popleft()
                if entry is None:
                    entry = _MeshEntry(key, blocks[1])
                    self._meshes[key] = entry
                    j._build_entry = True
                else:
                    j._build_entry = False
                entry.users += 1
                entry.last_used = time.perf_counter()
                self.peak_in_use = max(self.peak_in_use, self.arena.in_use)
                j._block, j._entry = blocks[0], entry
                j.t_admitted = time.perf_counter()
                admitted.append(j)
        for j in admitted:
            self._setup_q.put(j)

    def _drop(self, j: AssemblyJob) -> None:
        """Return a job's block and its hold on the mesh entry (lock held)."""
        if getattr(j, "_block", None) is not None:
            self.arena.release(j._block)
            j._block = None
        e = getattr(j, "_entry", None)
        if e is not None:
            e.users -= 1
            e.last_used = time.perf_counter()
            if e.error is not None and e.users == 0 and self._meshes.get(e.key) is e:
                del self._meshes[e.key]  # a failed build is not kept
                self.arena.release(e.block)
            j._entry = None

    def _release(self, act: _Active) -> None:
        j = act.job
        act.K = act.M = act.cmap = act.dmat = act.ws_K = act.ws_M = act.status = None
        act.out = []
        with self._lock:
            self._drop(j)
            if act in self._active:
                self._active.remove(act)
        j.t_done = time.perf_counter()
        self.completed.append(j)
        j.done.set()
        self._admit()

    # ------------------------------------------------------------ setup workers
    def _setup_loop(self) -> None:
        torch.cuda.set_device(self.dev)
        # setup copies and plan kernels take the GPU ahead of queued batch tiles
        stream = torch.cuda.Stream(self.dev, priority=-1)
        while not self._stop.is_set():
            j = self._setup_q.get()
            if j is None:
                return
            act = _Active(j, self.slots)
            entry = j._entry
            try:
                with torch.cuda.stream(stream):
                    tp = [time.perf_counter()]
                    if j._build_entry:
                        try:
                            dmesh = DeviceMesh(j.field, j.conductor_tets, self.dev, alloc=entry.block)
                            cmap = GpuCSCMapping(dmesh)
                            stream.synchronize()
                            dmesh.check_status()
                            entry.dmesh, entry.cmap = dmesh, cmap
                            self.n_mesh_builds += 1
                        except BaseException as e:
                            entry.error = e
                        finally:
                            entry.ready.set()
                    else:
                        entry.ready.wait()
                    if entry.error is not None:
                        raise entry.error
                    tp.append(time.perf_counter())
                    blk = j._block
                    cmap = entry.cmap
                    er, ur = j.materials()
                    act.dmat = DeviceMaterial(er, ur, j.n_tets, self.dev, alloc=blk)
                    nnz = max(cmap.nnz, 1)
                    ws = int(L.lib().emg_assemble_workspace_size(cmap.n_assy, self.precision))
                    act.K = blk(nnz, torch.complex128)
                    act.M = blk(nnz, torch.complex128)
                    act.ws_K = blk(max(ws, 1), torch.uint8)
                    act.ws_M = blk(max(ws, 1), torch.uint8)
                    act.status = blk(2, torch.int64)
                    act.out = [blk(nnz, torch.complex128) for _ in range(self.slots)]
                    act.cmap = cmap
                    stream.synchronize()
                    tp.append(time.perf_counter())
                    j.setup_parts = dict(zip(("mesh", "material"), np.diff(tp)))
            except BaseException as e:  # reported on the job, the server keeps serving
                j.error = e
                stream.synchronize()
                with self._lock:
                    self._drop(j)
                j.done.set()
                self._admit()
                continue
            with self._lock:
                self._ready_km.append(act)
            self._wake.set()

    # ------------------------------------------------------------ batcher
    def _collect(self):
        """Items of the next batch: jobs with the least remaining work first
        (short jobs finish in the first batches), at most max_items items and
        about max_batch_nnz nonzeros, so that a batch stays short and setup
        work on the other streams gets the GPU between batches."""
        batch, work = [], 0
        with self._lock:
            order = sorted(self._active, key=lambda a: (len(a.job.freqs) - a.next_f) * a.cmap.nnz)
            for act in order:
                j = act.job
                while (act.free_slots and act.next_f < len(j.freqs) and len(batch) < self.max_items
                       and (not batch or work + act.cmap.nnz <= self.max_batch_nnz)):
                    batch.append((act, act.next_f, act.free_slots.popleft()))
                    act.next_f += 1
                    work += act.cmap.nnz
        return batch

    def _launch(self, batch) -> None:
        tiles = 0
        self._h_tiles[0] = 0
        lead = 0  # first item of the current run of one job's frequencies (formed together)
        for i, (act, fi, slot) in enumerate(batch):
            k0 = 2 * np.pi * float(act.job.freqs[fi]) / C0
            it = self._items_view[i]
            it.K, it.M, it.P = act.K.data_ptr(), act.M.data_ptr(), None
            it.out = act.out[slot].data_ptr()
            it.nnz = act.cmap.nnz
            it.coef[:] = (1.0, 0.0, -k0 * k0, 0.0, 0.0, 0.0)
            if i > 0 and batch[i - 1][0] is act:
                it.group = 0
                self._items_view[lead].group += 1
            else:
                lead = i
                it.group = 1
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

    def _assemble_km(self, acts) -> None:
        """K and M of every job set up since the last pass: for each material
        kind, groups of up to max_assembly_jobs jobs, each group one element
        launch and one gather launch over a job table (emg_assemble_batch,
        two entries per job: K = alpha 1, beta 0; M = alpha 0, beta 1)."""
        t0 = time.perf_counter()
        lib = L.lib()
        h = L.ctypes.c_void_p(self._batch_stream.cuda_stream)
        by_kind: dict = {}
        for act in acts:
            by_kind.setdefault(act.dmat.kind, []).append(act)
        failed = []
        with torch.cuda.stream(self._batch_stream):
            for kind, group in by_kind.items():
                for g0 in range(0, len(group), self.max_km):
                    part = group[g0:g0 + self.max_km]
                    for i, act in enumerate(part):
                        act.status.zero_()
                        dm = act.cmap.dmesh
                        for k, (a, b, ws, out) in enumerate(((1.0, 0.0, act.ws_K, act.K), (0.0, 1.0, act.ws_M, act.M))):
                            d = self._km_desc[2 * i + k]
                            d.plan = L.ctypes.pointer(act.cmap.plan)
                            d.d_plan, d.d_indptr = act.cmap.d_plan.data_ptr(), act.cmap.d_indptr.data_ptr()
                            d.d_nodes, d.n_nodes, d.d_tets = dm.nodes.data_ptr(), dm.n_nodes, dm.tets.data_ptr()
                            d.d_tetids = dm.tetids.data_ptr() if dm.tetids is not None else None
                            d.mat = act.dmat.struct()
                            d.alpha_re, d.alpha_im, d.beta_re, d.beta_im = a, 0.0, b, 0.0
                            d.d_values, d.d_A, d.d_status = ws.data_ptr(), out.data_ptr(), act.status.data_ptr()
                    L.check(lib.emg_assemble_batch(self._km_desc, 2 * len(part), self.precision,
                                                   L.ptr(self._km_h), L.ptr(self._km_d), self._km_h.numel(), h))
                    self._batch_stream.synchronize()  # the pinned table is reused by the next group
                    self.n_km_batches += 1
                    for act in part:
                        st = act.status.cpu()
                        if int(st[0]):
                            failed.append((act, L.EmgMeshError(L.EMG_EMESH, f"status flags {int(st[0])} at "
                                                                                f"assembled index {int(st[1])}")))
        t1 = time.perf_counter()
        bad = {id(a) for a, _ in failed}
        for act, err in failed:
            act.job.error = err
            self._release(act)
        with self._lock:
            for act in acts:
                if id(act) in bad:
                    continue
                act.job.setup_parts["K_M"] = t1 - t0
                act.job.t_setup = t1
                act.ws_K = act.ws_M = None
                self._active.append(act)

    def _batch_loop(self) -> None:
        torch.cuda.set_device(self.dev)
        while not self._stop.is_set():
            with self._lock:
                km, self._ready_km = self._ready_km, []
            if km:
                try:
                    self._assemble_km(km)
                except BaseException as e:
                    for act in km:
                        act.job.error = e
                        self._release(act)
            batch = self._collect()
            if not batch:
                if not km:
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
    """Latency percentiles (arrival -> last A(f) ready), and the same split
    into admission wait, setup (upload, pattern, K, M) and forming."""
    lat = np.array([j.latency for j in jobs]) * 1e3
    out = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "jobs": int(lat.size)}
    for name, a, b in (("wait", "arrival", "t_admitted"), ("setup", "t_admitted", "t_setup"),
                       ("form", "t_setup", "t_done")):
        d = np.array([getattr(j, b) - getattr(j, a) for j in jobs]) * 1e3
        out[f"{name}_p50_ms"] = float(np.percentile(d, 50))
        out[f"{name}_p99_ms"] = float(np.percentile(d, 99))
    parts = [j.setup_parts for j in jobs if j.setup_parts]
    if parts:
        out["setup_parts_mean_ms"] = {k: 1e3 * float(np.mean([p[k] for p in parts])) for k in parts[0]}
    return out


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
    tan(delta) ~ U[0,1e-2] per 8x8x8-cell block (a per-tet scalar), mu_r = 1,
    a U{n_freq}
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
        er = eps[blk]  # isotropic: per-tet scalar eps_r, mu_r = 1
        nf = int(rng.integers(n_freq[0], n_freq[1] + 1))
        freqs = np.sort(rng.uniform(freq_hz[0], freq_hz[1], nf))
        jobs.append(AssemblyJob(field, er, None, freqs, job_id=i))
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
           "km_batches": server.n_km_batches, "mesh_builds": server.n_mesh_builds,
           "arrival_span_s": float(arrivals[-1]) if len(arrivals) else 0.0}
    out.update(latency_summary(jobs))
    return out
