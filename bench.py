"""Benchmark of the B200 Nedelec-2 assembly (EMerge hot path).

One step = one assembly of A = K - k0^2 M (element kernel + column gather) of
the 2,010,000-tet WR-90 dielectric workload with its pattern cached, inputs
resident in HBM (value) and, separately, through the public drop-in API with
host numpy inputs and a host scipy result (e2e).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config wr90_dielectric|wr90_air]

Prints ONE JSON line on rank 0. Under torchrun (N > 1) every rank assembles
its own replica of the workload (independent objects, no collective on the
data path): weak scaling, max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tets/s assembled (A = K - k0^2 M values, pattern cached), mixed vs plain FP64"
UNIT = "tets/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="wr90_dielectric", choices=["wr90_dielectric", "wr90_air"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-tets", type=int, default=200000,
                    help="tets of the bounded CPU samples of the --sweep / --pml / --heat / --shard modes")
    ap.add_argument("--cpu-chunk-tets", type=int, default=100000,
                    help="tets per chunk of the reference arm's whole-workload assembly")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=None, help="hex grid nx,ny,nz of the dielectric box (default 100,50,67)")
    ap.add_argument("--forms", default="fp64,mixed", help="comma list of forms to time (fp64, mixed, exact)")
    ap.add_argument("--sweep", action="store_true",
                    help="resident frequency sweep: 201 frequencies 8-12 GHz with the two port terms on the workload")
    ap.add_argument("--sweep-conductive", action="store_true",
                    help="the sweep with a conductivity per block (K, M1, P resident; the reference reassembles "
                         "every frequency for such materials)")
    ap.add_argument("--sweep-freqs", type=int, default=201)
    ap.add_argument("--sweep-batch", type=int, default=12, help="frequencies formed per launch (outputs resident; 12 x 8.9 GB)")
    ap.add_argument("--pml", action="store_true",
                    help="anisotropic PML shell + 2%% slivers (1,008,000 tets): speed and mixed-vs-FP64 errors")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: one assembly column-sharded over the ranks instead of one replica per rank")
    ap.add_argument("--heat", action="store_true",
                    help="Lagrange-2 heat-conduction assembly (stiffness + capacity, COO -> CSC) on a 2.01M-tet box")
    ap.add_argument("--heat-grid", default="100,50,67")
    ap.add_argument("--shard-emulate", default="",
                    help="with --shard on one GPU: comma list of shard counts N; each N's shards are assembled one "
                         "after another and timed (an estimate of N-GPU strong scaling, not a measurement of it)")
    ap.add_argument("--serving", action="store_true",
                    help="serving stream instead: Poisson arrivals of assembly jobs (5k-500k tets, 1-64 frequencies)")
    ap.add_argument("--serving-jobs", type=int, default=1000)
    ap.add_argument("--no-serving", action="store_true",
                    help="leave the serving stream out of the default line (it runs at N = 1)")
    ap.add_argument("--serving-rate", type=float, default=50.0, help="mean arrivals per second")
    ap.add_argument("--serving-budget-gb", type=float, default=120.0)
    ap.add_argument("--serving-workers", type=int, default=3, help="setup worker threads")
    ap.add_argument("--serving-batch-nnz", type=float, default=2 ** 28, help="nonzeros per form batch (cap)")
    return ap.parse_args()


def make_workload(name, seed_offset=0, grid=None):
    from emerge_b200 import workloads as W

    if name == "wr90_air":
        return W.wr90_air(seed=0 + seed_offset)
    n = tuple(int(x) for x in grid.split(",")) if grid else (100, 50, 67)
    return W.wr90_dielectric(n=n, seed=1 + seed_offset)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.window = "the timed region with its warm-up"
        # nvidia-smi numbers GPUs physically; map a visible-device index
        # through CUDA_VISIBLE_DEVICES when that restricts the visible set
        vis = [x.strip() for x in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if x.strip()]
        self.gpu = vis[gpu_index] if 0 <= gpu_index < len(vis) else str(gpu_index)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def preroll(self, step, min_samples: int = 5, max_s: float = 1.5):
        """Untimed steps, right before the timed ones, until the sampler has
        min_samples readings under this load (nvidia-smi reads every 50 ms
        at best, so a timed region of tens of ms alone would give one)."""
        import torch

        if self.proc is None:
            return
        self.window = "untimed pre-roll steps, warm-up and timed steps of the same workload"
        n0, t0 = len(self.lines), time.perf_counter()
        while len(self.lines) - n0 < min_samples and time.perf_counter() - t0 < max_s:
            step()
            torch.cuda.synchronize()

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "window": self.window}


# ---------------------------------------------------------------- CPU baseline (oracle port)
class CpuBaseline:
    """The reference algorithm (C port in oracle/, OpenMP over all host cores)
    on a bounded contiguous sample of the workload: element build
    (_matrix_builder) + to_csc of E - k0^2 B, the sample's pattern cached."""

    def __init__(self, wl, sample_tets: int):
        from oracle import oracle as O

        self.O = O
        f = wl.field
        m = f.mesh
        self.n = n = min(sample_tets, f.ntets)
        start = (f.ntets - n) // 2
        self.tetids = np.arange(start, start + n, dtype=np.int64)
        self.cores = os.cpu_count() or 1
        self.args = (m.nodes, m.tets, m.tris, m.edges, f.get_tet_to_field(), m.tet_to_edge, m.tet_to_tri, wl.ur,
                     wl.er, self.tetids)
        dE, dB, rows, cols = O.matrix_builder(*self.args, nthreads=self.cores)
        self.pat = O.CSCPattern.from_rowcol(rows, cols, f.n_field, self.cores)
        del rows, cols, dE, dB
        self.k0 = wl.k0
        self.desc = (f"{n} contiguous tets of the {wl.name} workload ({f.ntets} tets): element build + scatter "
                     f"of E - k0^2 B, pattern cached, {self.cores} threads")

    def step(self):
        t0 = time.perf_counter()
        dE, dB, _, _ = self.O.matrix_builder(*self.args, nthreads=self.cores)
        self.pat.values_lincomb(dE, dB, 1.0, -self.k0 ** 2, self.cores)
        return time.perf_counter() - t0

    def measure(self, reps: int = 3):
        self.step()
        t = float(np.median([self.step() for _ in range(reps)]))
        return {"value": self.n / t, "unit": UNIT, "cores": self.cores, "kind": "port", "sample": self.desc}


class CpuSweepBaseline(CpuBaseline):
    """The reference's cached multi-frequency path (assembler.py:455-494: Evec
    and Bvec built once, to_csc(Evec - Bvec * k0**2) per frequency) on the
    same bounded sample: the per-frequency scatter alone, scaled to the full
    mesh by its tet count. The port term's per-frequency scatter is left out
    (its 20,000 triangles are ~1% of the work)."""

    def __init__(self, wl, sample_tets: int):
        super().__init__(wl, sample_tets)
        self.dE, self.dB, _, _ = self.O.matrix_builder(*self.args, nthreads=self.cores)
        self.scale = self.n / wl.field.ntets
        self.desc = (f"{self.n} contiguous tets of the {wl.name} workload ({wl.field.ntets} tets): per frequency "
                     f"to_csc(E - k0^2 B) with E, B and the pattern cached, {self.cores} threads, scaled to the "
                     f"full mesh by tet count")

    def step(self):
        t0 = time.perf_counter()
        self.pat.values_lincomb(self.dE, self.dB, 1.0, -self.k0 ** 2, self.cores)
        return time.perf_counter() - t0

    def measure(self, reps: int = 5):
        self.step()
        t = float(np.median([self.step() for _ in range(reps)]))
        return {"value": self.scale / t, "unit": "frequencies/s", "cores": self.cores, "kind": "port",
                "sample": self.desc}


def arm_config(wl, nnz):
    """The workload both arms run (the same dict in both lines)."""
    return {"workload": wl.name, "tets": int(wl.n_tets), "hex_grid": list(wl.hex_grid), "nnz": int(nnz),
            "N": int(wl.field.n_field), "freq_hz": wl.freq, "assembled": "A = K - k0^2 M values, pattern cached"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU algorithm (the C port of its
    _matrix_builder + to_csc in oracle/) on all host threads, over the WHOLE
    workload every step: the assembled tets in chunks of --cpu-chunk-tets,
    each chunk's element matrices built and scattered into the one CSC value
    array in the reference scatter's order (bit for bit the one-piece
    result; the full COO, 19.2 KB per tet, would not fit in host memory).
    The pattern and the chunks' scatter orders are built once before the
    timed steps, as the reference caches its CSCMapping. Rank 0 only."""
    if rank != 0:
        return None
    from oracle import oracle as O

    wl = make_workload(args.config, grid=args.grid)
    t0 = time.perf_counter()
    ca = O.ChunkedAssembly(wl.field, wl.er, wl.ur, wl.conductor_tets, chunk_tets=args.cpu_chunk_tets)
    setup_s = time.perf_counter() - t0
    out = np.zeros(ca.nnz, np.complex128)
    beta = -wl.k0 ** 2
    for _ in range(args.warmup):
        ca.step(1.0, beta, out)
    ts = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        ca.step(1.0, beta, out)
        ts.append(time.perf_counter() - t1)
    mean_s = float(np.mean(ts))
    v = wl.n_tets / mean_s
    desc = (f"the whole {wl.name} workload ({wl.n_tets} tets) every step: element build (_matrix_builder) + "
            f"scatter of E - k0^2 B into A in the reference's order, {len(ca.chunks)} chunks of "
            f"<= {ca.chunk_tets} tets, {ca.nthreads} threads, pattern cached")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * mean_s, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": arm_config(wl, ca.nnz),
            "reference_setup_s": setup_s, "step_s": {"min": min(ts), "median": float(np.median(ts)),
                                                     "max": max(ts)},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ca.nthreads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def cpu_baseline_subprocess(args):
    """The reference arm (whole workload, all host threads) in a fresh
    process: 1 warm-up and 2 timed steps. A fresh process keeps the CPU
    timing apart from this process's GPU-side threads, pinned buffers and
    OpenMP runtimes, so both CPU numbers of a run come from the same code in
    the same conditions."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", "2", "--warmup", "1",
           "--config", args.config, "--cpu-chunk-tets", str(args.cpu_chunk_tets)]
    if args.grid:
        cmd += ["--grid", args.grid]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1200, env=env)
    except subprocess.TimeoutExpired:
        return {"value": None, "unavailable": "reference arm timed out"}
    for ln in reversed(r.stdout.strip().splitlines()):
        try:
            d = json.loads(ln)
        except ValueError:
            continue
        cb = dict(d["cpu_baseline"])
        cb["sample"] += "; run as `bench.py --impl reference --steps 2 --warmup 1` in a fresh process"
        return cb
    return {"value": None, "unavailable": f"reference arm failed (rc {r.returncode}): {r.stderr[-300:]}"}


# ---------------------------------------------------------------- GPU arm
L2_BYTES = 126 * 10 ** 6


class L2Guard:
    """Timing hygiene for a step whose data could stay in the 126 MB L2 from
    one step to the next: when the bytes a step reads and writes are below 16
    L2 sizes, a 256 MB buffer is written on the launching stream before every
    timed step or kernel, outside the timed events. Larger steps are timed
    back to back (their inputs are larger than L2)."""

    def __init__(self, footprint, dev):
        import torch

        self.footprint = int(footprint)
        self.buf = None
        if self.footprint < 16 * L2_BYTES:
            self.buf = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=dev)
        self.n = 0

    @property
    def active(self):
        return self.buf is not None

    def flush(self, stream):
        import torch

        if self.buf is not None:
            self.n += 1
            with torch.cuda.stream(stream):
                self.buf.fill_(self.n & 0xFF)

    def text(self):
        if self.buf is None:
            return (f"inputs larger than L2: {self.footprint / 1e9:.2f} GB read or written per step "
                    f"against 126 MB of L2, steps timed back to back")
        return (f"L2 flushed before every timed step and kernel (256 MB written outside the timed events); "
                f"step footprint {self.footprint / 1e6:.0f} MB")


def assembly_footprint(cmap, prec):
    """Bytes one assembly step reads or writes: the element values written
    and read back, the plan read, A written."""
    from emerge_b200 import _lib as L

    ws = int(L.lib().emg_assemble_workspace_size(cmap.n_assy, prec))
    return cmap.d_plan.numel() * cmap.d_plan.element_size() + 2 * ws + 16 * cmap.nnz


def time_steps(fn, steps, warmup, stream, l2=None):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if l2 is not None and l2.active:
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in evs:
            l2.flush(stream)
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / steps
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        fn()
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / steps


def kernel_times(cmap, job, prec, alpha, beta, out, reps, stream, l2=None):
    """Average duration of each kernel of the step, CUDA events on the
    launching stream (L2 flushed before each repetition when the guard
    asks for it)."""
    import torch

    from emerge_b200 import _lib as L

    m = job.mesh
    ws = cmap.workspace(prec)
    mat = job.mat.struct()
    lib = L.lib()
    h = L.ctypes.c_void_p(stream.cuda_stream)
    layout = L.EMG_LAYOUT_BLOCK if cmap.plan.value_layout == L.EMG_LAYOUT_BLOCK else L.EMG_LAYOUT_PACKED
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    te, tg = 0.0, 0.0
    for _ in range(reps):
        if l2 is not None:
            l2.flush(stream)
        ev[0].record(stream)
        L.check(lib.emg_element_values(L.ptr(m.nodes), m.n_nodes, L.ptr(m.tets), m.n_tets, L.ptr(m.tetids),
                                       m.n_assy, L.ctypes.byref(mat), prec, L.EMG_OUT_LINCOMB, layout,
                                       alpha.real, alpha.imag, beta.real, beta.imag, L.ptr(ws), None, h))
        ev[1].record(stream)
        L.check(lib.emg_gather(L.ctypes.byref(cmap.plan), L.ptr(cmap.d_plan), L.ptr(cmap.d_indptr), L.ptr(ws), None,
                               prec, layout, 1.0, 0.0, 0.0, 0.0, L.ptr(out), None, h))
        ev[2].record(stream)
        torch.cuda.synchronize()
        te += ev[0].elapsed_time(ev[1])
        tg += ev[1].elapsed_time(ev[2])
    return te / reps, tg / reps


def load_traffic(workload):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
    except (OSError, ValueError):
        return None
    return d.get(workload)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from emerge_b200 import _lib as L
    from emerge_b200 import workloads as W
    from emerge_b200.assembly import (DeviceMaterial, DeviceMesh, GpuCSCMapping, _Job,
                                      tet_mass_stiffness_matrices)

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    L.check(L.lib().emg_device_check(local_rank))
    wl = make_workload(args.config, seed_offset=0, grid=args.grid)
    f = wl.field
    dmesh = DeviceMesh(f, wl.conductor_tets, dev)
    t0 = time.perf_counter()
    cmap0 = GpuCSCMapping(dmesh)  # entity-pair block layout: 4-byte records, four entries of A each
    torch.cuda.synchronize()
    plan_s = time.perf_counter() - t0
    cmap = cmap0
    dmat = DeviceMaterial(wl.er, wl.ur, f.ntets, dev)
    k0 = wl.k0
    alpha, beta = 1.0 + 0j, complex(-k0 ** 2)
    stream = torch.cuda.current_stream(dev)
    out = torch.empty(cmap.nnz, dtype=torch.complex128, device=dev)
    results = {}
    forms = {"fp64": L.EMG_FP64, "mixed": L.EMG_MIXED, "exact": L.EMG_EXACT}
    for pname in [x for x in ("fp64", "mixed", "exact") if x in args.forms.split(",")]:
        prec = forms[pname]
        job = _Job(dmesh, dmat, prec)
        cmap = cmap0
        cmap.workspace(prec)
        l2 = L2Guard(assembly_footprint(cmap, prec), dev)

        def step():
            cmap.assemble_device(job, alpha, beta, out)

        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local_rank) if pname == "mixed" else None
        if sampler:
            sampler.__enter__()
            sampler.preroll(step)
        ms = time_steps(step, args.steps, args.warmup, stream, l2)
        if sampler:
            sampler.__exit__()
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        dmesh.check_status()
        te, tg = kernel_times(cmap, job, prec, alpha, beta, out, 3, stream, l2)
        results[pname] = {"ms": ms, "k_element_ms": te, "k_gather_ms": tg, "value_layout": cmap.value_layout,
                          "clocks": sampler.summary() if sampler else None, "l2": l2.text()}
        del l2
        torch.cuda.synchronize()
        cmap._ws = None  # element workspace of this form
    cmap = cmap0
    # the mixed form's error against FP64 (which matches the oracle to 1e-12)
    # for K, M and A, relative Frobenius and max entry, on the device
    errors = None
    if "fp64" in results and "mixed" in results:
        def rel(a, b):
            d = a - b
            return {"fro": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b)),
                    "max": float(d.abs().max() / b.abs().max())}

        errors = {}
        for key, ka, kb in (("K", 1.0 + 0j, 0j), ("M", 0j, 1.0 + 0j), ("A", alpha, beta)):
            v64 = cmap.assemble_device(_Job(dmesh, dmat, L.EMG_FP64), ka, kb).clone()
            v32 = cmap.assemble_device(_Job(dmesh, dmat, L.EMG_MIXED), ka, kb)
            errors[key] = rel(v32[: cmap.nnz], v64[: cmap.nnz])
            del v64, v32
        cmap._ws = None
        dmesh.check_status()
    # e2e through the public API (host numpy in, host scipy out), both forms
    def e2e_run(precision):
        nodes_b = f.mesh.nodes.nbytes
        tets_b = f.mesh.tets.shape[1] * 4 * 4
        E, B, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets, cmap, precision=precision,
                                              device=dev)
        A = cmap.to_csc(E - B * k0 ** 2)  # warm
        # the mapping's device tets are reused when the same tet array comes back
        tets_shared = E.job.mesh.tets.data_ptr() == cmap.dmesh.tets.data_ptr()
        h2d = nodes_b + (0 if tets_shared else tets_b) + E.job.mat.h2d_bytes
        del A, E, B
        times = []
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            E, B, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets, cmap, precision=precision,
                                                  device=dev)
            A = cmap.to_csc(E - B * k0 ** 2)
            times.append(time.perf_counter() - t0)
            del A, E, B
        t = float(np.median(times))
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return {"value": world * f.ntets / t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(cmap.nnz * 16), "s_per_step": t, "form": precision,
                "path": "tet_mass_stiffness_matrices(..., cscmap, precision) + GpuCSCMapping.to_csc(E - B*k0**2) "
                        "-> scipy csc_matrix; per step: node coordinates and materials copied in, A copied out"
                        + ("; tets resident in the mapping" if tets_shared else "")}

    e2e = e2e_fp64 = None
    if args.e2e_steps > 0:
        e2e = e2e_run("mixed")
        e2e_fp64 = e2e_run("fp64")
        cmap._ws = None
    line = None
    if rank == 0:
        nT, nnz, nN = f.ntets, cmap.nnz, f.mesh.n_nodes
        balg = W.alg_bytes(nN, nT, nnz, 16)
        bfloor = W.floor_bytes(nN, nT, nnz, 16)
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(pk):
            peaks = json.load(open(pk))
        hbm = peaks.get("hbm_gbs")
        peak_src = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        primary = "mixed" if "mixed" in results else next(iter(results))
        mx = results[primary]
        fp = results.get("fp64", mx)
        traffic = load_traffic(wl.name) or {}

        def roof(r, form):
            """Roofline of the dominant kernel (the gather) on the algorithmic
            bytes of one assembly step: nodes, tets, materials, the int32
            slot -> nonzero map (400 per tet), the segment offsets and A written
            (balg, 7,187 B per tet here) over the gather's CUDA-event time. The
            kernels' own algorithmic bytes -- which count the element values'
            round trip through HBM -- are kept beside it."""
            vb = 8 if form == "mixed" else 16
            vpt = 220 if r.get("value_layout") == "block" else 210
            kb = {"k_element": W.element_alg_bytes(nN, nT, vb, 16, vpt), "k_gather": W.gather_alg_bytes(nT, nnz, vb, vpt)}
            kms = {"k_element": r["k_element_ms"], "k_gather": r["k_gather_ms"]}
            dom = max(kms, key=kms.get)
            kern = {}
            for k in kb:
                ach = kb[k] / (kms[k] * 1e-3) / 1e9
                kern[k] = {"own_alg_bytes": kb[k], "ms": kms[k], "own_achieved": ach, "own_frac": ach / hbm,
                           "traffic": traffic.get(f"{form}_{k}_bytes")}
            ach = balg / (kms[dom] * 1e-3) / 1e9
            step_ach = balg / (r["ms"] * 1e-3) / 1e9
            return {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "unit": "GB/s",
                    "frac": ach / hbm, "traffic": kern[dom]["traffic"], "peak_source": peak_src,
                    "alg_bytes_per_launch": balg,
                    "alg_bytes_rule": "24 nN + 16 nT + 16 nT (er) + 4 x 400 nT + 4 (nnz + 1) + 16 nnz",
                    "kernels": kern,
                    "step": {"alg_bytes": balg, "achieved": step_ach, "frac": step_ach / hbm,
                             "floor_bytes": bfloor, "floor_frac": bfloor / (r["ms"] * 1e-3) / 1e9 / hbm,
                             "traffic": traffic.get(f"{form}_step_bytes")}}

        value = world * nT / (mx["ms"] * 1e-3)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": mx["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 geometry + f32 contraction (mixed), f64 sum", "data": "synthetic",
                "config": arm_config(wl, nnz),
                "form": primary, "l2": mx["l2"],
                "parallelism": f"replicas x{world}" if world > 1 else "1 gpu",
                "alg_bytes_per_step": balg, "floor_bytes_per_step": bfloor, "plan_build_s": plan_s,
                "plain_fp64": {"value": world * nT / (fp["ms"] * 1e-3), "ms_per_step": fp["ms"],
                               "k_element_ms": fp["k_element_ms"], "k_gather_ms": fp["k_gather_ms"],
                               "value_layout": fp["value_layout"], "roofline": roof(fp, "fp64"),
                               "e2e": e2e_fp64},
                "mixed": {"k_element_ms": mx["k_element_ms"], "k_gather_ms": mx["k_gather_ms"]},
                "mixed_over_plain": fp["ms"] / mx["ms"], "mixed_vs_fp64_errors": errors,
                "roofline": roof(mx, primary), "clocks": mx["clocks"], "e2e": e2e,
                # per timed step: the status-word reset, the element kernel and the gather
                "gpu_launches": 3 * args.steps}
    return line, wl


def run_sweep(args, rank, world, local_rank):
    """--sweep: K and M of the workload assembled once and kept in HBM, then
    A(f) = K - k0(f)^2 M + gamma(f) (R_in + R_out) for every frequency (the
    cached multi-frequency path with TE10 port terms, gamma = j beta(f)),
    formed --sweep-batch frequencies per launch into resident outputs."""
    import torch

    from emerge_b200 import workloads as W
    from emerge_b200.assembly import tet_mass_stiffness_matrices
    from emerge_b200.mesh import plane_tris
    from emerge_b200.ranks import max_over_ranks
    from emerge_b200.robin import RobinTerm
    from emerge_b200.sweep import FrequencySweep

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = make_workload(args.config, grid=args.grid)
    f = wl.field
    z = f.mesh.nodes[2]
    t0 = time.perf_counter()
    if args.sweep_conductive:
        # a conductivity per 8x8x8-cell block, 0.1-10 S/m (no loss tangent)
        from emerge_b200.workloads import block_ids

        blk = block_ids(*wl.hex_grid)
        sig = np.random.default_rng(5).uniform(0.1, 10.0, int(blk.max()) + 1)[blk]
        cond = np.zeros((3, 3, f.ntets), np.complex128)
        for d in range(3):
            cond[d, d] = sig
        sw = FrequencySweep.with_conductivity(f, wl.er, np.zeros_like(cond), cond, wl.ur, wl.conductor_tets,
                                              device=dev)
        cmap = sw.cscmap
    else:
        E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets, precision="fp64", device=dev)
    ports = [RobinTerm(f, plane_tris(f.mesh, 2, float(z.min())), cmap),
             RobinTerm(f, plane_tris(f.mesh, 2, float(z.max())), cmap)]
    if args.sweep_conductive:
        sw.robin = ports
        coef_fn = FrequencySweep.conductive_coefficients
    else:
        sw = FrequencySweep(E, B, cmap, robin=ports)
        coef_fn = FrequencySweep.coefficients
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    freqs = np.linspace(8e9, 12e9, args.sweep_freqs)
    gam = np.array([W.rect_port_gamma(x) for x in freqs])
    nb = max(1, min(args.sweep_batch, freqs.size))
    out = torch.empty((nb, cmap.nnz), dtype=torch.complex128, device=dev)
    stream = torch.cuda.current_stream(dev)

    def sweep():
        for i0 in range(0, freqs.size, nb):
            fb = freqs[i0:i0 + nb]
            g = gam[i0:i0 + nb]
            sw.form(coef_fn(fb), out[: fb.size], robin_gamma=np.stack([g, g], axis=1))

    nnz, nf = cmap.nnz, freqs.size
    n_launch = -(-nf // nb)
    n_res = 3 if args.sweep_conductive else 2  # resident matrices read per launch
    bytes_sweep = n_launch * 16 * n_res * nnz + nf * 16 * nnz  # K, M (, P) read per batch; A written per frequency
    l2 = L2Guard(bytes_sweep, dev)
    sampler = ClockSampler(local_rank)
    with sampler:
        ms = time_steps(sweep, args.steps, args.warmup, stream, l2)
    cmap.dmesh.check_status()
    ms = max_over_ranks([ms], dev)[0]
    if rank != 0:
        return None, None
    hbm = (json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
           if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else None) or 6650.0
    ach = bytes_sweep / (ms * 1e-3) / 1e9
    metric = ("resident frequency sweep, conductive materials: A(f) = K - k0^2 M1 - (k0^2/w) P + gamma(f) R_ports "
              "formed per second" if args.sweep_conductive else
              "resident frequency sweep: A(f) = K - k0^2 M + gamma(f) R_ports formed per second")
    return {"metric": metric,
            "value": world * nf / (ms * 1e-3), "unit": "frequencies/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": wl.name + ("_conductive_sweep" if args.sweep_conductive else "_sweep"),
                       "tets": f.ntets, "nnz": nnz, "freqs": nf,
                       "band_hz": [8e9, 12e9], "batch": nb, "port_tris": int(sum(r.n_btris for r in ports)),
                       "K_M_form": "fp64", "setup_s": setup_s, "l2": l2.text(),
                       "step": f"all {nf} frequencies, {n_launch} form launches + {2 * nf} port-term launches"},
            "tet_freqs_per_s": world * f.ntets * nf / (ms * 1e-3),
            "roofline": {"bound": "hbm", "kernel": "k_form_sweep", "achieved": ach, "peak": hbm, "unit": "GB/s",
                         "frac": ach / hbm, "alg_bytes_per_step": bytes_sweep, "traffic": None},
            "clocks": sampler.summary(), "gpu_launches": args.steps * (n_launch + 2 * nf)}, wl


def run_pml(args, rank, world, local_rank):
    """--pml: the 84x50x40 PML + slivers workload (diagonal complex er = ur in
    the outer 10% shell, 2% slivers): assembly speed of both forms and the
    mixed form's relative error against FP64 for K, M, A, also with only one
    diagonal tensor component kept (the others 1), on the device."""
    import torch

    from emerge_b200 import _lib as L
    from emerge_b200 import workloads as W
    from emerge_b200.assembly import DeviceMaterial, DeviceMesh, GpuCSCMapping, _Job
    from emerge_b200.ranks import max_over_ranks

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = W.wr90_pml_slivers()
    f = wl.field
    dm = DeviceMesh(f, wl.conductor_tets, dev)
    cmap = GpuCSCMapping(dm)
    k0 = wl.k0
    alpha, beta = 1.0 + 0j, complex(-k0 ** 2)
    stream = torch.cuda.current_stream(dev)
    dmat = DeviceMaterial(wl.er, wl.ur, f.ntets, dev)
    out = torch.empty(cmap.nnz, dtype=torch.complex128, device=dev)
    times, l2s = {}, {}
    sampler = ClockSampler(local_rank)
    with sampler:
        sampler.preroll(lambda: cmap.assemble_device(_Job(dm, dmat, L.EMG_MIXED), alpha, beta, out))
        for name, prec in (("fp64", L.EMG_FP64), ("mixed", L.EMG_MIXED)):
            job = _Job(dm, dmat, prec)
            l2 = L2Guard(assembly_footprint(cmap, prec), dev)
            times[name] = time_steps(lambda: cmap.assemble_device(job, alpha, beta, out), args.steps, args.warmup,
                                     stream, l2)
            l2s[name] = l2.text()
            del l2
    dm.check_status()
    times = dict(zip(times, max_over_ranks(list(times.values()), dev)))

    def comp(t, c):
        o = np.zeros_like(t)
        for d in range(3):
            o[d, d] = t[d, d] if d == c else 1.0
        return o

    def rel(a, b):
        d = (a - b).abs()
        return {"fro": float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)),
                "max": float(d.max() / b.abs().max())}

    errors = {}
    for cname, c in (("xx", 0), ("yy", 1), ("zz", 2), ("full", None)):
        er = wl.er if c is None else comp(wl.er, c)
        ur = wl.ur if c is None else comp(wl.ur, c)
        mat = DeviceMaterial(er, ur, f.ntets, dev)
        res = {}
        for key, a, b in (("K", 1.0 + 0j, 0j), ("M", 0j, 1.0 + 0j), ("A", alpha, beta)):
            v64 = cmap.assemble_device(_Job(dm, mat, L.EMG_FP64), a, b).clone()
            v32 = cmap.assemble_device(_Job(dm, mat, L.EMG_MIXED), a, b)
            res[key] = rel(v32[: cmap.nnz], v64[: cmap.nnz])
            del v64, v32
        errors[cname] = res
    # both forms against the exact closed form (FP64 on edge-vector geometry,
    # free of the reference's cancellation): on these slivers the reference's
    # own arithmetic, which the FP64 form reproduces, is the larger error
    mat = DeviceMaterial(wl.er, wl.ur, f.ntets, dev)
    vs_exact = {}
    for key, a, b in (("K", 1.0 + 0j, 0j), ("M", 0j, 1.0 + 0j), ("A", alpha, beta)):
        vex = cmap.assemble_device(_Job(dm, mat, L.EMG_EXACT), a, b).clone()
        for pname, prec in (("fp64", L.EMG_FP64), ("mixed", L.EMG_MIXED)):
            v = cmap.assemble_device(_Job(dm, mat, prec), a, b)
            vs_exact.setdefault(pname, {})[key] = rel(v[: cmap.nnz], vex[: cmap.nnz])
            del v
        del vex
    dm.check_status()
    if rank != 0:
        return None, None
    nT, nnz, nN = f.ntets, cmap.nnz, f.mesh.n_nodes
    balg = W.alg_bytes(nN, nT, nnz, 96)
    return {"metric": "tets/s assembled, anisotropic PML + slivers workload (mixed form; FP64 beside)",
            "value": world * nT / (times["mixed"] * 1e-3), "unit": "tets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": times["mixed"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mixed", "data": "synthetic",
            "config": {"workload": wl.name, "tets": nT, "hex_grid": list(wl.hex_grid), "nnz": nnz,
                       "slivers": int(len(wl.slivers)), "material": "diagonal complex er = ur (PML shell)",
                       "alg_bytes_per_step": balg, "l2": l2s["mixed"]},
            "plain_fp64": {"value": world * nT / (times["fp64"] * 1e-3), "ms_per_step": times["fp64"]},
            "mixed_vs_fp64_errors": errors, "errors_vs_exact_form": vs_exact, "clocks": sampler.summary(),
            "gpu_launches": 4 * args.steps}, wl


def run_heat(args, rank, world, local_rank):
    """--heat: the transient heat assembly of assembler.py:123-130 on a
    Lagrange-2 box -- stiffness and capacity element values, each gathered
    into CSC values -- with the field's mesh and COO -> CSC mapping resident.
    Both element forms are timed ('fp64' = the reference's quadrature loop,
    'exact' = the moment form); the line's value is the exact form."""
    import torch

    from emerge_b200 import _lib as L
    from emerge_b200 import workloads as W
    from emerge_b200.heat import _heat_mesh, tet_mass_matrix, tet_stiffness_matrix
    from emerge_b200.ranks import max_over_ranks

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = W.heat_box(n=tuple(int(x) for x in args.heat_grid.split(",")))
    f = wl.field
    t0 = time.perf_counter()
    hm = _heat_mesh(f, dev)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    cm = hm.cmap
    nT, nN, nnz = hm.n_tets, hm.n_nodes, cm.nnz
    d_cond = torch.from_numpy(wl.cond).to(dev)
    d_rho = torch.from_numpy(wl.rho_cp).to(dev)
    vK = torch.empty(100 * nT, dtype=torch.float64, device=dev)
    vM = torch.empty(100 * nT, dtype=torch.float64, device=dev)
    oK = torch.empty(nnz, dtype=torch.float64, device=dev)
    oM = torch.empty(nnz, dtype=torch.float64, device=dev)
    status = torch.zeros(2, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = L.ctypes.c_void_p(stream.cuda_stream)
    lib = L.lib()

    def elem(coef, kind, prec, out):
        L.check(lib.emg_leg2_element(L.ptr(hm.nodes), nN, L.ptr(hm.tets), nT, L.ptr(coef), kind, prec,
                                     L.EMG_LAYOUT_COO_T, L.ptr(out), L.ptr(status), sh))

    def gath(v, out):
        L.check(lib.emg_coo_gather(L.ctypes.byref(cm.desc), L.ptr(cm.d_perm), L.ptr(cm.d_run), 0, 10, L.ptr(v),
                                   L.ptr(out), sh))

    # both element matrices written and read back, the map read twice, K and M written
    l2 = L2Guard(4 * 800 * nT + 2 * (4 * cm.d_perm.numel() + 4 * cm.d_run.numel()) + 16 * nnz, dev)

    def ktime(fn, reps=5):
        fn()
        if l2.active:
            tot = 0.0
            for _ in range(reps):
                l2.flush(stream)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                torch.cuda.synchronize()
                tot += a.elapsed_time(b)
            return tot / reps
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    res = {}
    sampler = ClockSampler(local_rank)
    for pname, prec in (("fp64", L.EMG_FP64), ("exact", L.EMG_EXACT)):
        def step():
            elem(d_cond, 0, prec, vK)
            elem(d_rho, 1, prec, vM)
            gath(vK, oK)
            gath(vM, oM)

        if pname == "exact":
            sampler.__enter__()
            sampler.preroll(step)
        ms = time_steps(step, args.steps, args.warmup, stream, l2)
        if pname == "exact":
            sampler.__exit__()
        ms = max_over_ranks([ms], dev)[0]
        res[pname] = {"ms": ms, "k_stiff_ms": ktime(lambda: elem(d_cond, 0, prec, vK)),
                      "k_mass_ms": ktime(lambda: elem(d_rho, 1, prec, vM)), "k_gather_ms": ktime(lambda: gath(vK, oK))}
    fl, ix = L.ctypes.c_int64(), L.ctypes.c_int64()
    L.check(lib.emg_status_read(L.ptr(status), L.ctypes.byref(fl), L.ctypes.byref(ix), sh))
    if fl.value:
        raise RuntimeError(f"heat workload flagged tet {ix.value}")
    # the two forms agree on this workload
    elem(d_cond, 0, L.EMG_FP64, vK)
    elem(d_cond, 0, L.EMG_EXACT, vM)
    form_diff = float((vK - vM).abs().max() / vK.abs().max())
    # e2e: the public API, host arrays in, host csc_matrix out, field resident
    e2e = None
    if args.e2e_steps > 0:
        def api():
            K, c = tet_stiffness_matrix(f, wl.cond, precision="exact", device=dev)
            A = c.to_csc(K)
            M, c = tet_mass_matrix(f, wl.rho_cp, precision="exact", device=dev)
            B = c.to_csc(M)
            return A, B

        api()
        times = []
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            A, B = api()
            times.append(time.perf_counter() - t1)
            del A, B
        t = max_over_ranks([float(np.median(times))], dev)[0]
        e2e = {"value": world * nT / t, "unit": "tets/s", "h2d_bytes_per_step": int(wl.cond.nbytes + wl.rho_cp.nbytes),
               "d2h_bytes_per_step": int(2 * nnz * 8), "s_per_step": t,
               "path": "tet_stiffness_matrix + to_csc, tet_mass_matrix + to_csc -> scipy csc_matrix (mesh and "
                       "mapping resident)"}
    if rank != 0:
        return None, None
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peaks.get("hbm_gbs") or 6650.0
    src = "measured" if peaks.get("hbm_gbs") else "fallback"

    def roof(r, form):
        kb = {"k_leg2_stiff": W.heat_element_alg_bytes(nN, nT, "stiff"),
              "k_leg2_mass": W.heat_element_alg_bytes(nN, nT, "mass"), "k_coo_gather": W.heat_gather_alg_bytes(nT, nnz)}
        kms = {"k_leg2_stiff": r["k_stiff_ms"], "k_leg2_mass": r["k_mass_ms"], "k_coo_gather": r["k_gather_ms"]}
        tr = load_traffic(wl.name) or {}
        kern = {k: {"alg_bytes": kb[k], "ms": kms[k], "achieved": kb[k] / (kms[k] * 1e-3) / 1e9,
                    "frac": kb[k] / (kms[k] * 1e-3) / 1e9 / hbm, "traffic": tr.get(f"{form}_{k}_bytes")}
                for k in kb}
        dom = max(kms, key=kms.get)
        d = kern[dom]
        return {"bound": "hbm", "kernel": dom, "achieved": d["achieved"], "peak": hbm, "unit": "GB/s",
                "frac": d["frac"], "traffic": d["traffic"], "peak_source": src, "alg_bytes_per_launch": d["alg_bytes"],
                "kernels": kern}

    ex, fp = res["exact"], res["fp64"]
    line = {"metric": "tets/s assembled, Lagrange-2 heat conduction (stiffness + capacity, COO -> CSC)",
            "value": world * nT / (ex["ms"] * 1e-3), "unit": "tets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ex["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "tets": nT, "hex_grid": list(wl.hex_grid), "N": int(f.n_field),
                       "nnz": nnz, "form": "exact", "setup_s": setup_s,
                       "l2": l2.text(),
                       "parallelism": f"replicas x{world}" if world > 1 else "1 gpu"},
            "plain_fp64": {"value": world * nT / (fp["ms"] * 1e-3), "ms_per_step": fp["ms"],
                           "k_stiff_ms": fp["k_stiff_ms"], "k_mass_ms": fp["k_mass_ms"],
                           "note": "the reference's quadrature loop: FP64-issue bound", "roofline": roof(fp, "fp64")},
            "kernels_ms": {k: v for k, v in ex.items() if k != "ms"}, "exact_vs_fp64_max_rel": form_diff,
            "roofline": roof(ex, "exact"), "clocks": sampler.summary(), "e2e": e2e, "gpu_launches": 4 * args.steps}
    return line, wl


class HeatCpuBaseline:
    """The reference's heat assembly restated in C (oracle/, OpenMP over all
    host cores) on a bounded sample of the workload's tets: both element
    builders and the f8 scatter of each into CSC, the sample's pattern
    cached."""

    def __init__(self, wl, sample_tets: int):
        from oracle import oracle as O

        self.O = O
        f = wl.field
        nT = f.mesh.n_tets
        self.n = n = min(sample_tets, nT)
        lo = (nT - n) // 2
        sl = slice(lo, lo + n)
        self.mesh = type("SampleMesh", (), {"nodes": f.mesh.nodes, "tets": np.ascontiguousarray(f.mesh.tets[:, sl])})()
        self.cond = np.ascontiguousarray(wl.cond[:, :, sl])
        self.rho = np.ascontiguousarray(wl.rho_cp[sl])
        self.cores = os.cpu_count() or 1
        rows, cols = O.leg2_rowcol(f.tet_to_field[:, sl])
        self.pat = O.CSCPattern.from_rowcol(rows, cols, f.n_field, self.cores)
        self.desc = (f"{n} contiguous tets of the {wl.name} workload ({nT} tets): stiffness and capacity element "
                     f"builds + f8 scatter of each, pattern cached, {self.cores} threads")

    def step(self):
        t0 = time.perf_counter()
        K = self.O.leg2_values(self.mesh, self.cond, "stiff")
        M = self.O.leg2_values(self.mesh, self.rho, "mass")
        self.pat.values_f8(K, self.cores)
        self.pat.values_f8(M, self.cores)
        return time.perf_counter() - t0

    def measure(self, reps: int = 3):
        self.step()
        t = float(np.median([self.step() for _ in range(reps)]))
        return {"value": self.n / t, "unit": "tets/s", "cores": self.cores, "kind": "port", "sample": self.desc}


def run_shard(args, rank, world, local_rank):
    """--shard: the workload's columns split over the ranks (each rank
    assembles the tets touching its edges/faces, no exchange step); one step
    = every rank assembling its column block; max-over-ranks device time."""
    import torch

    from emerge_b200.partition import ShardedAssembly, shard_of
    from emerge_b200.ranks import max_over_ranks, sum_over_ranks

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = make_workload(args.config, grid=args.grid)
    f = wl.field
    if args.shard_emulate and world == 1:
        return emulate_shards(args, wl, dev)
    t0 = time.perf_counter()
    sh = shard_of(f.mesh, rank, world, wl.conductor_tets)
    sa = ShardedAssembly(f, wl.er, wl.ur, sh, "mixed", dev)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    alpha, beta = 1.0 + 0j, complex(-wl.k0 ** 2)
    out = torch.empty(sa.cmap.nnz, dtype=torch.complex128, device=dev)
    stream = torch.cuda.current_stream(dev)
    l2 = L2Guard(assembly_footprint(sa.cmap, sa.job.precision), dev)
    sampler = ClockSampler(local_rank)
    with sampler:
        ms = time_steps(lambda: sa.assemble(alpha, beta, out), args.steps, args.warmup, stream, l2)
    sa.dmesh.check_status()
    ms, setup_s = max_over_ranks([ms, setup_s], dev)
    own, tets_done = sum_over_ranks([sa.own_nnz, sh.tetids.size], dev)
    if rank != 0:
        return None
    return {"metric": METRIC, "value": f.ntets / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "mixed", "data": "synthetic",
            "config": {"workload": wl.name, "tets": f.ntets, "hex_grid": list(wl.hex_grid),
                       "parallelism": f"column shards x{world}", "owned_nnz_total": int(own),
                       "tets_assembled_total": int(tets_done), "halo_overhead": tets_done / f.ntets - 1.0,
                       "setup_s": setup_s, "l2": l2.text()},
            "clocks": sampler.summary(), "gpu_launches": 2 * args.steps}


def emulate_shards(args, wl, dev):
    """N-way column shards on one GPU, one after another: each shard's step
    time (mixed form, its own tets and halo, its own columns). The shards
    never communicate, so an N-GPU step would take the slowest shard's time;
    that is reported as an estimate, next to the halo overhead."""
    import torch

    from emerge_b200.partition import ShardedAssembly, partition

    f = wl.field
    alpha, beta = 1.0 + 0j, complex(-wl.k0 ** 2)
    stream = torch.cuda.current_stream(dev)
    res = {}
    launches = 0
    for N in [int(x) for x in args.shard_emulate.split(",") if x.strip()]:
        per, tets, own, l2_text = [], 0, 0, []
        parts = partition(f.mesh, N, wl.conductor_tets)
        for r in range(N):
            sh = parts[r]
            launches += 2 * (args.steps + args.warmup)
            sa = ShardedAssembly(f, wl.er, wl.ur, sh, "mixed", dev)
            out = torch.empty(sa.cmap.nnz, dtype=torch.complex128, device=dev)
            l2 = L2Guard(assembly_footprint(sa.cmap, sa.job.precision), dev)
            l2_text.append(l2.text())
            per.append(time_steps(lambda: sa.assemble(alpha, beta, out), args.steps, args.warmup, stream, l2))
            del l2
            sa.dmesh.check_status()
            tets += sh.tetids.size
            own += sa.own_nnz
            del sa, out
            torch.cuda.empty_cache()
        res[str(N)] = {"shard_ms": per, "step_ms_estimate": max(per), "tets_per_s_estimate": f.ntets / (max(per) * 1e-3),
                       "halo_overhead": tets / f.ntets - 1.0, "owned_nnz_total": int(own),
                       "imbalance": max(per) / (sum(per) / N), "l2": l2_text}
    one = res.get("1", {}).get("step_ms_estimate")
    for v in res.values():
        v["speedup_estimate"] = (one / v["step_ms_estimate"]) if one else None
    best = max(res.values(), key=lambda v: v["tets_per_s_estimate"])
    return {"metric": METRIC + " (column shards emulated one after another on one GPU: an estimate)",
            "value": best["tets_per_s_estimate"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["step_ms_estimate"], "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "mixed", "data": "synthetic",
            "config": {"workload": wl.name, "tets": f.ntets, "hex_grid": list(wl.hex_grid),
                       "parallelism": "column shards, emulated sequentially",
                       "l2": "per shard, in emulated_shards[N].l2"},
            "emulated_shards": res, "gpu_launches": launches}


class CpuServingBaseline:
    """The same job list through the CPU port of the reference, in arrival
    order and one job at a time: per job the element build and the pattern,
    then to_csc(E - k0^2 B) per frequency, all host threads; stops after
    about budget_s of work and reports the tet-frequencies completed per
    second."""

    def __init__(self, jobs, budget_s: float = 20.0):
        self.jobs, self.budget = jobs, budget_s
        self.cores = os.cpu_count() or 1

    def measure(self):
        from oracle import oracle as O

        t0 = time.perf_counter()
        tf = n_jobs = 0
        for j in self.jobs:
            f = j.field
            m = f.mesh
            er, ur = j.tensors()
            dE, dB, rows, cols = O.matrix_builder(m.nodes, m.tets, m.tris, m.edges, f.get_tet_to_field(),
                                                  m.tet_to_edge, m.tet_to_tri, ur, er,
                                                  np.arange(f.ntets, dtype=np.int64), nthreads=self.cores)
            pat = O.CSCPattern.from_rowcol(rows, cols, f.n_field, self.cores)
            del rows, cols
            for fr in j.freqs:
                if time.perf_counter() - t0 > self.budget:
                    break
                k0 = 2 * np.pi * fr / 299792458.0
                pat.values_lincomb(dE, dB, 1.0, -k0 ** 2, self.cores)
                tf += f.ntets
            n_jobs += 1
            if time.perf_counter() - t0 > self.budget:
                break
        dt = time.perf_counter() - t0
        return {"value": tf / dt, "unit": "tet-freqs/s", "cores": self.cores, "kind": "port",
                "sample": f"the stream's first {n_jobs} jobs in arrival order, one at a time: element build, "
                          f"pattern and per-frequency scatter ({tf} tet-frequencies in {dt:.1f} s)"}


def serving_stream(args, rank, local_rank, budget_gb=None):
    """One seeded serving stream on this GPU (mixed form): a short warm-up
    stream, then --serving-jobs Poisson arrivals at --serving-rate; returns
    the stream summary (throughput, latency percentiles, clocks) and jobs."""
    import torch

    from emerge_b200.serving import AssemblyServer, run_stream, synthetic_stream

    torch.cuda.set_device(local_rank)
    jobs, arr = synthetic_stream(args.serving_jobs, args.serving_rate, seed=rank)
    warm, warr = synthetic_stream(3, 1000.0, tets=(5_000, 50_000), n_freq=(1, 4), seed=1000 + rank)
    budget = (budget_gb if budget_gb is not None else args.serving_budget_gb) * 1e9
    with AssemblyServer(device=local_rank, budget_bytes=budget, precision="mixed",
                        setup_workers=args.serving_workers, max_batch_nnz=int(args.serving_batch_nnz)) as srv:
        run_stream(srv, warm, warr)
        srv.drop_mesh_cache()  # the measured stream starts cold
        srv.n_batches = srv.n_items = srv.n_km_batches = srv.n_mesh_builds = 0
        srv.peak_in_use = 0
        sampler = ClockSampler(local_rank)
        with sampler:
            r = run_stream(srv, jobs, arr)
    r["clocks"] = sampler.summary()
    r["budget_gb"] = budget / 1e9
    return r, jobs


def run_serving(args, rank, world, local_rank):
    """Serving stream on this rank's GPU (replicas under torchrun: each rank
    serves its own seeded stream). Throughput in tet-frequencies/s."""
    r, jobs = serving_stream(args, rank, local_rank)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([r["makespan_s"], r["p99_ms"]], device=torch.device("cuda", local_rank))
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        r["makespan_s"], r["p99_ms"] = float(t[0]), float(t[1])
    line = {"metric": "serving throughput: tet-frequencies/s assembled (A(f) = K - k0(f)^2 M on the device)",
            "value": world * r["tet_freqs"] / r["makespan_s"], "unit": "tet-freqs/s", "n_gpus": world,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "mixed", "data": "synthetic",
            "config": {"workload": "serving_stream", "jobs": r["jobs"], "rate_per_s": args.serving_rate,
                       "tets": "log-uniform [5k, 500k]", "freqs": "U{1..64} in U[1, 40] GHz",
                       "budget_gb": args.serving_budget_gb, "setup_workers": args.serving_workers,
                       "batch_nnz_cap": int(args.serving_batch_nnz),
                       "alloc_conf": os.environ.get("PYTORCH_CUDA_ALLOC_CONF", ""),
                       "parallelism": f"replicas x{world}"},
            "serving": r, "clocks": r["clocks"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = CpuServingBaseline(jobs).measure()
    return line if rank == 0 else None


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    if args.serving:
        line, wl = run_serving(args, rank, world, local_rank), None
    elif args.shard:
        line, wl = run_shard(args, rank, world, local_rank), None
    elif args.sweep:
        line, wl = run_sweep(args, rank, world, local_rank)
    elif args.pml:
        line, wl = run_pml(args, rank, world, local_rank)
    elif args.heat:
        line, wl = run_heat(args, rank, world, local_rank)
    else:
        line, wl = run_ours(args, rank, world, local_rank)
        if world == 1 and not args.no_serving:
            # the serving stream beside the assembly line (N = 1 only)
            import gc

            import torch

            gc.collect()
            torch.cuda.empty_cache()
            r, _ = serving_stream(args, rank, local_rank, budget_gb=min(args.serving_budget_gb, 100.0))
            line["serving"] = {"metric": "tet-frequencies/s and job latency (arrival -> last A(f) ready)",
                               "rate_per_s": args.serving_rate, **r}
    # the host-core baseline is taken at N = 1 only (rank 0), so that N > 1
    # runs hold their GPUs for the GPU work alone
    if rank == 0 and world == 1 and not args.no_cpu_baseline and wl is not None:
        if args.sweep and args.sweep_conductive:
            cb = CpuBaseline(wl, args.cpu_sample_tets).measure()  # the reference reassembles every frequency
            cb["value"] /= wl.field.ntets
            cb["unit"] = "frequencies/s"
            cb["sample"] += "; per frequency, scaled to the full mesh by tet count (reassembly, as the reference "\
                            "does for conductive materials)"
            line["cpu_baseline"] = cb
        elif args.heat or args.sweep or args.pml:
            base = HeatCpuBaseline if args.heat else (CpuSweepBaseline if args.sweep else CpuBaseline)
            line["cpu_baseline"] = base(wl, args.cpu_sample_tets).measure()
        else:
            line["cpu_baseline"] = cpu_baseline_subprocess(args)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
