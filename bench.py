#!/usr/bin/env python
"""Connected-components benchmark on B200 (one JSON line on rank 0).

Workload (default ``rmat24``): plain single-graph CC on a seeded R-MAT graph,
scale 24 (16,777,216 vertices), edge factor 16, a/b/c/d = .57/.19/.19/.05,
symmetrised with self loops and duplicates removed, uint32 CSR - the
reference's single-GPU headline configuration.  ``grid8192`` is the
8192 x 8192 4-neighbour grid with 10% of edges deleted.

A step is one full solve (labels = min vertex id per component) of the
device-resident graph through ccgpu_local_cc.  ``e2e`` repeats the metric
through the reference-facing call compute_connected_components_pthreads with
pinned host buffers: the CSR copy to HBM and the label copy back are inside
its timed region.  ``cpu_baseline`` and ``--impl reference`` time the
reference's own compute_connected_components_pthreads (compiled unmodified
into oracle/_ref) on this machine's host cores.

Metric: GTEPS = unique undirected edges / solve time (higher is better).
Multi-GPU (torchrun): every rank solves its own graph (seed + rank), no
collective on the data path; value = all ranks' edges / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "rmat24": dict(kind="rmat", scale=24, ef=16),
    "rmat22": dict(kind="rmat", scale=22, ef=16),
    "rmat20": dict(kind="rmat", scale=20, ef=16),
    "grid8192": dict(kind="grid", rows=8192, cols=8192, p=0.1),
    "grid2048": dict(kind="grid", rows=2048, cols=2048, p=0.1),
    # partitioned path (compute_connected_components_mpi_advanced)
    "c3": dict(kind="rmat_big", scale=26, n=65_600_000, undirected=1_800_000_000, parts=4,
               dist=True, ref_runs=1),
    # the reference's own CPU-runnable case: R-MAT scale 18 as a .mat file,
    # mpirun -np 2 -t 8 -c 8192 -e 1 -r 3
    "c1": dict(kind="rmat", scale=18, ef=16, parts=2, dist=True, mat=True, ref_runs=3),
    "rmat24p4": dict(kind="rmat", scale=24, ef=16, parts=4, dist=True),
    "rmat22p4": dict(kind="rmat", scale=22, ef=16, parts=4, dist=True),
    # batched path (ccgpu_batch_*): graphs of log-uniform size, a third each
    # Erdos-Renyi (mean degree 8), R-MAT (edge factor 16), grid (10% deleted)
    "batch4096": dict(kind="batch", graphs=4096, n_min=1_000, n_max=2_000_000, batch=True),
    "batch1024": dict(kind="batch", graphs=1024, n_min=1_000, n_max=200_000, batch=True),
    # served path (ccgpu_server_*): Poisson arrivals drawn from the batched mix
    # plus 5% R-MAT scale-22 requests
    "served": dict(kind="served", pool=512, n_min=1_000, n_max=2_000_000, big_scale=22,
                   big_frac=0.05, seconds=6.0, served=True),
    # the same server on small requests (1k-50k vertices, no large ones),
    # where per-request launch and copy overheads dominate
    "served_small": dict(kind="served", pool=1024, n_min=1_000, n_max=50_000, big_scale=22,
                         big_frac=0.0, seconds=6.0, served=True),
}
L2_BYTES = 126 * 1024 * 1024
ORACLE_MAX_N = 1_000_000  # batched workloads: graphs up to this size are checked by the oracle
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_graph(torch, wl, seed):
    from cc_mpi_b200 import graphs
    spec = WORKLOADS[wl]
    if spec["kind"] == "rmat":
        return graphs.rmat_csr_torch(torch, spec["scale"], spec["ef"], seed=seed)
    if spec["kind"] == "rmat_big":
        return graphs.rmat_csr_big(torch, spec["scale"], spec["n"], spec["undirected"], seed=seed)
    return graphs.grid_csr_torch(torch, spec["rows"], spec["cols"], spec["p"], seed=seed)


def workload_config(wl, n, m):
    spec = dict(WORKLOADS[wl])
    cfg = {"workload": wl, "vertices": n, "undirected_edges": m // 2, "csr_entries": m}
    if spec["kind"] == "rmat":
        cfg.update(graph=f"R-MAT scale {spec['scale']}, edge factor {spec['ef']}, "
                         "a/b/c/d=.57/.19/.19/.05, seeded id permutation")
    elif spec["kind"] == "rmat_big":
        cfg.update(graph=f"R-MAT over 2^{spec['scale']} ids, a/b/c/d=.57/.19/.19/.05, seeded "
                         f"permutation truncated to {spec['n']} vertices, sampled for about "
                         f"{spec['undirected']} distinct undirected edges")
    else:
        cfg.update(graph=f"{spec['rows']}x{spec['cols']} 4-neighbour grid, "
                         f"{int(spec['p'] * 100)}% of edges deleted")
    return cfg


class ClockSampler:
    """Polls NVML (read-only) from a thread while the timed region runs."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
               0x2: "applications_clocks_setting", 0x1: "gpu_idle"}

    def __init__(self, index):
        self.samples, self.reasons = [], 0
        self.max_mhz = None
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # pragma: no cover - depends on the driver
            log("clock sampler unavailable:", e)

    def _reasons(self):
        nv = self.nv
        for fn in ("nvmlDeviceGetCurrentClocksEventReasons",
                   "nvmlDeviceGetCurrentClocksThrottleReasons"):
            if hasattr(nv, fn):
                return getattr(nv, fn)(self.h)
        return 0

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= int(self._reasons())
            except Exception:
                break
            time.sleep(0.001)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        names = [v for k, v in self.REASONS.items() if self.reasons & k and k != 0x1]
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def local_cc_bytes(torch, deg, n, m, opts, finish_rows=None, finish_edges=None, row_bytes=8):
    """Algorithmic bytes of each launch of one local CC solve, by kernel name
    (a list when the launches of one kernel move different bytes).  Per
    launch, what the kernel must move at least: row pointers it reads
    (8 bytes per row), the column entries it reads (4 each), its own label
    read and write (4 each per vertex); neighbour-label gathers are counted
    as cache-served, so the figure is conservative.

    ``deg`` is the device tensor of row lengths of the graph the local CC
    runs on.  Sampling round r reads entry r of every row longer than r.
    With the second-neighbour stash (sampling with min-hooks and a shortcut
    between rounds, at least two rounds, and 8 or more entries per vertex)
    round 0 reads entries 0 and 1 of each row and writes the stash (4n),
    and round 1 reads only the stash (4n).  ``row_bytes``: bytes of row
    bounds per row (8 for a CSR's row pointers, 16 for begin/end pairs)."""
    k = opts.sample_rounds if opts.sample_rounds >= 0 else 2
    hook = opts.hook_mode if opts.hook_mode >= 0 else 12
    stash = (hook & 12) == 12 and k >= 2 and m >= 8 * n

    def longer(r):
        return int((deg > r).sum().item())

    sample = []
    r = 0
    if stash:
        two = int(torch.clamp(deg, max=2).sum().item())
        sample += [row_bytes * n + 4 * two + 4 * n + 4 * n, 4 * n + 4 * n]
        r = 2
    sample += [row_bytes * n + 4 * longer(q) + 4 * n for q in range(r, k)]
    link = 4 * n + row_bytes * n
    if finish_rows is not None:
        link = 4 * n + 8 * int(finish_rows) + 4 * int(finish_edges)
    return {"init": [4 * n], "sample": sample or [0], "compress": [8 * n], "giant": [4 * 1024],
            "link_rows": [link], "link_heavy": [0], "final_compress": [8 * n]}


def per_launch(bytes_lists):
    """Mean bytes per launch of each kernel."""
    return {kk: sum(v) / len(v) for kk, v in bytes_lists.items()}


def step_bytes_of(bytes_lists, per, steps):
    """Algorithmic bytes of one step: every launch the profiler saw, each
    charged its own bytes (kernels launched more than once per step with
    different bytes, like the sampling rounds, are charged their mean)."""
    mean = per_launch(bytes_lists)
    return sum(mean.get(kk, 0) * cnt / steps for kk, (_, cnt) in per.items())


def run_reference_graphs(args, world, spec_w):
    """--impl reference on the batched and served workloads: the reference
    solves one graph per call, so it is timed on the workload's graphs one
    by one (a bounded, seeded sample), reported in graphs per second."""
    import numpy as np
    import torch
    import oracle
    from cc_mpi_b200 import batch
    torch.cuda.set_device(0)
    n_graphs = spec_w.get("graphs", spec_w.get("pool", 512))
    spec = batch.mix_spec(n_graphs, spec_w["n_min"], spec_w["n_max"], seed=args.seed)
    order = np.random.default_rng(args.seed).permutation(len(spec))
    threads = os.cpu_count() or 1
    graphs_h = []
    for g in order[:64]:
        kind, n, seed = spec[g]
        rp_d, col_d = batch.build_one_torch(torch, kind, n, seed)
        graphs_h.append((rp_d.cpu().numpy().view(np.uint64), col_d.cpu().numpy().view(np.uint32)))
    for rp, col in graphs_h[:args.warmup]:
        oracle.ref_pthreads_labels(rp, col, threads, 8192)
    t_all, done, edges = 0.0, 0, 0
    for _ in range(args.steps):
        for rp, col in graphs_h:
            t0 = time.perf_counter()
            oracle.ref_pthreads_labels(rp, col, threads, 8192)
            t_all += time.perf_counter() - t0
            done += 1
            edges += len(col) // 2
        if t_all > 60.0:
            break
    gps = done / t_all
    line = {
        "impl": "reference", "metric": "batched CC graphs/s" if spec_w.get("batch")
        else "served CC graphs/s", "value": gps, "unit": "graphs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_all / max(done, 1) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": args.workload, "graphs_timed": done, "gteps": edges / t_all / 1e9},
        "cpu_baseline": {"value": gps, "unit": "graphs/s", "cores": threads,
                         "kind": "reference" if oracle.have_ref() else "port",
                         "sample": f"{len(graphs_h)} graphs of the workload's mix in seeded "
                                   f"random order, solved one by one, {args.steps} rounds"},
        "e2e": {"value": gps, "unit": "graphs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU code on this host.  Plain
    single-graph workloads time compute_connected_components_pthreads with
    every host thread; partitioned workloads time the reference's own MPI
    path (mpi_cc_benchmark at the workload's rank count, its CLI's per-run
    time) - a bounded number of full solves, ``--ref-runs``."""
    if rank != 0:
        return 0
    spec_w = WORKLOADS[args.workload]
    if spec_w.get("batch") or spec_w.get("served"):
        return run_reference_graphs(args, world, spec_w)
    import numpy as np
    import torch
    import oracle
    torch.cuda.set_device(0)
    rp_d, col_d = make_graph(torch, args.workload, args.seed)
    rp = rp_d.cpu().numpy().view(np.uint64)
    col = col_d.cpu().numpy().view(np.uint32)
    del rp_d, col_d
    torch.cuda.empty_cache()
    n, m = len(rp) - 1, int(rp[-1])
    threads = os.cpu_count() or 1
    cfg = workload_config(args.workload, n, m)
    if spec_w.get("dist"):
        parts = args.parts or spec_w["parts"]
        runs = args.ref_runs or spec_w.get("ref_runs", 1)
        base, why = ref_mpi_baseline(rp, col, parts, args.chunk, args.exchange, runs,
                                     mat=spec_w.get("mat", False))
        if base is None:
            print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
            return 0
        gteps = base["value"]
        cfg.update(partitions=parts, chunk_size=args.chunk, exchange_interval=args.exchange,
                   components=base["components"], rounds=base["rounds"])
        line = {
            "impl": "reference", "metric": "CC GTEPS", "value": gteps, "unit": "GTEPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": base["seconds_per_solve"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": cfg, "cpu_baseline": base,
            "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "timing": f"the reference CLI's own per-run times of {runs} full solve(s); the "
                      f"--steps/--warmup counts are not repeated on the CPU (minutes per solve)",
        }
        print(json.dumps(line), flush=True)
        return 0
    for _ in range(args.warmup):
        oracle.ref_pthreads_labels(rp, col, threads, 8192)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.ref_pthreads_labels(rp, col, threads, 8192)
        times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    gteps = (m / 2) / t / 1e9
    line = {
        "impl": "reference", "metric": "CC GTEPS", "value": gteps, "unit": "GTEPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": threads, "kind": "reference",
                         "path": "compute_connected_components_pthreads",
                         "sample": f"full graph, {args.steps} solves, chunk 8192"},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(rp, col, budget_s=20.0):
    """The reference's compute_connected_components_pthreads (compiled
    unmodified into oracle/_ref) on all host threads, chunk 8192: up to 3
    solves within ``budget_s``.  Returns (baseline dict, labels of the last
    solve) - the labels are the parity check of the GPU result."""
    import oracle
    threads = os.cpu_count() or 1
    m = int(rp[-1])
    times = []
    t_start = time.perf_counter()
    labels = None
    if oracle.have_ref():
        kind = "reference"
        while len(times) < 3 and time.perf_counter() - t_start < budget_s:
            t0 = time.perf_counter()
            labels = oracle.ref_pthreads_labels(rp, col, threads, 8192)
            times.append(time.perf_counter() - t0)
        sample = f"full graph, {len(times)} solves, {threads} threads, chunk 8192"
        used = threads
    else:
        kind = "port"
        t0 = time.perf_counter()
        labels, _ = oracle.lp_labels(rp, col)
        times.append(time.perf_counter() - t0)
        sample = "full graph, 1 solve, 1 thread (oracle label propagation)"
        used = 1
    t = min(times)
    return ({"value": (m / 2) / t / 1e9, "unit": "GTEPS", "cores": used, "kind": kind,
             "path": "compute_connected_components_pthreads", "sample": sample,
             "seconds_per_solve": t}, labels)


def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def ref_mpi_memory(n, m, parts, boundary_raw=None, freed=0):
    """(fits, reason): whether this host can hold the reference's own
    partitioned run.  Peak host bytes: rank 0 holds the whole CSR while the
    partitions fill (2x the CSR), then the partitions plus 8 bytes per cut
    entry of the boundary arrays and ~13 bytes per vertex of per-vertex
    arrays.  ``freed``: bytes the caller releases before the run."""
    csr = 8 * (n + 1) + 4 * m
    raw = boundary_raw if boundary_raw is not None else m
    need = max(2 * csr, csr + 8 * raw + 13 * n) + (2 << 30)
    have = host_mem_available() + freed
    if host_mem_available() and need > have:
        return False, (f"host has {have / 2**30:.1f} GiB available, the reference's "
                       f"{parts}-rank run needs about {need / 2**30:.1f} GiB")
    return True, None


def ref_mpi_write(folder, rp, col, mat):
    """The graph as the reference's CLI input: MAT level 5 (struct Problem,
    sparse field A) when ``mat``, else the CSR binary format under a .mat
    name, which the matio shim serves as one sparse variable."""
    import oracle
    path = os.path.join(folder, "graph.mat")
    t0 = time.perf_counter()
    if mat:
        oracle.write_mat(path, rp, col)
    else:
        oracle.write_csrbin(path, rp, col)
    return path, time.perf_counter() - t0


def ref_mpi_time(path, n, m, parts, chunk, exchange, runs, threads=None, timeout=1500,
                 mat=False):
    """Runs the reference's own partitioned path - its mpi_cc_benchmark CLI
    (src/mpi_cc_benchmark.c, cc_mpi.c, exchange_plan.c, graph_dist.c, ...,
    compiled unmodified over the fakempi / fakematio shims into oracle/_ref)
    at ``parts`` ranks x floor(cores / parts) pthreads, -c chunk -e exchange
    -r runs.  Its time is the CLI's own per-run time (the region around one
    compute_connected_components_mpi_advanced call)."""
    import oracle
    cores = os.cpu_count() or 1
    threads = threads or max(1, cores // parts)
    res = oracle.ref_mpi_run(path, parts, threads=threads, chunk=chunk, exchange=exchange,
                             runs=runs, timeout=timeout)
    runs_out = res["runs"]
    secs = [r["seconds"] for r in runs_out if r["seconds"]]
    t = sum(secs) / len(secs)
    last = runs_out[-1]
    return {"value": (m / 2) / t / 1e9, "unit": "GTEPS", "cores": parts * threads,
            "kind": "reference", "path": "mpi_cc_benchmark (compute_connected_components_"
            "mpi_advanced over fakempi ranks)",
            "sample": f"full graph, {len(secs)} solve(s) of -np {parts} -t {threads} "
                      f"-c {chunk} -e {exchange} -r {runs} ({'MAT v5' if mat else 'CSR binary'}"
                      f" input, loaded once in {res['graph'].get('load_s', 0):.1f} s)",
            "seconds_per_solve": t, "ranks": parts, "threads_per_rank": threads,
            "components": last["components"], "rounds": last["rounds"],
            "bounds": last["bounds"], "boundary_raw": sum(last["raw"].values()),
            "boundary_dedup": sum(last["dedup"].values()),
            "ghosts": sum(last["ghosts"].values())}


def ref_mpi_baseline(rp, col, parts, chunk, exchange, runs, boundary_raw=None, mat=False):
    """ref_mpi_memory + ref_mpi_write + ref_mpi_time on a scratch folder
    (CCB200_SCRATCH or the system temp folder).  Returns (baseline, None) or
    (None, reason)."""
    import tempfile
    import oracle
    if not oracle.have_ref_mpi():
        return None, "reference MPI build (oracle/_ref/mpi_cc_benchmark) absent"
    n, m = len(rp) - 1, int(rp[-1])
    fits, why = ref_mpi_memory(n, m, parts, boundary_raw)
    if not fits:
        return None, why
    with tempfile.TemporaryDirectory(dir=os.environ.get("CCB200_SCRATCH")) as tmp:
        path, write_s = ref_mpi_write(tmp, rp, col, mat)
        base = ref_mpi_time(path, n, m, parts, chunk, exchange, runs, mat=mat)
    base["file_write_s"] = write_s
    return base, None


def local_degrees(torch, rp_d, col_d, bounds, chunk=1 << 26):
    """Row lengths of the partitions' local subgraphs (entries whose target
    lies in the row's own partition, src/cc_mpi.c:252-275), counted on the
    device in chunks of entries (setup work, outside any timed region)."""
    n = rp_d.numel() - 1
    dev = rp_d.device
    ldeg = torch.zeros(n, dtype=torch.int32, device=dev)
    for p in range(len(bounds) - 1):
        b0, b1 = int(bounds[p]), int(bounds[p + 1])
        if b1 <= b0:
            continue
        rows = rp_d[b0:b1 + 1]
        e0, e1 = int(rows[0].item()), int(rows[-1].item())
        for c0 in range(e0, e1, chunk):
            c1 = min(e1, c0 + chunk)
            v = col_d[c0:c1]
            local = (v >= b0) & (v < b1)
            pos = torch.arange(c0, c1, device=dev, dtype=torch.int64)[local]
            r = torch.searchsorted(rows, pos, right=True) - 1 + b0
            ldeg.index_add_(0, r, torch.ones_like(r, dtype=torch.int32))
            del v, local, pos, r
    return ldeg


def dist_bytes(torch, ldeg, n, m, st, chunk):
    """Algorithmic bytes per launch of the partitioned path's kernels (lists
    where one kernel's launches differ).  The local-CC kernels run on the
    partitions' local subgraphs and are counted as in local_cc_bytes over
    the local row lengths; the rest as listed per kernel below.  Two layouts
    of the local subgraphs: read in place as each row's run inside its own
    partition (row_runs: one streaming pass checks the row order and writes
    per-row partition offsets), or a local CSR built by a count and a fill
    pass."""
    from cc_mpi_b200 import _lib
    R, U, G, reps = int(st.sorted_keys), int(st.pair_count), int(st.ghost_count), \
        int(st.rep_count)
    lm = int(st.local_entries)
    P = int(st.parts) if hasattr(st, "parts") else 4
    sorted_rows = bool(st.sorted_rows)
    runs = bool(getattr(st, "row_runs", 0))
    out = local_cc_bytes(torch, ldeg, n, lm, _lib.opts(chunk_size=chunk),
                         row_bytes=16 if runs else 8)
    tiles, wtiles = (m + 4095) // 4096, (m + 511) // 512
    if runs:
        out.update({
            # k_row_scan: every column entry and row pointer in; P offsets
            # and the own run (begin, end) of every row out
            "dist_local_count": [4 * m + 8 * (n + 1) + 4 * P * n + 16 * n],
            # k_emit_ranges: P offsets in, mask out; k_mask_fix: the sorted
            # local-end keys in (the run lengths and masks it touches are few)
            "dist_pairs": [4 * P * n + 4 * n, 8 * R],
        })
    else:
        out.update({
            # k_part_cols (P+1 searches), k_tile_first over 4096- and
            # 512-entry tiles
            "dist_tiles": [0, 8 * (n + 1) + 4 * tiles, 8 * (n + 1) + 4 * wtiles],
            "dist_local_count": [4 * m + 4 * tiles],
            "dist_local_fill": [4 * m + 4 * lm + 16 * (n + 1)],
            "dist_pairs": [8 * (n + 1) + 4 * m + (m // 8 if sorted_rows else n // 8 + 8 * R)],
        })
    out.update({
        "dist_gflag": [4 * n + n // 8],
        "dist_pairs_bitmap": [4 * n + 4 * G],
        "dist_merge_keys": [16 * (R + G)],
        "dist_reps": [4 * n + 12 * reps],
        "dist_pairs_local": [n // 8 + 8 * R],
        "sort_hist": [8 * R], "sort_scatter": [16 * R], "dist_dedup": [8 * R],
        "dist_ghosts": [8 * R + 8 * U + 20 * G], "merge_hook": [12 * U],
        # an exchange reads each ghost's cached rep and its label, the last
        # one sent (8G), and writes the ghost label and delta entry of every
        # changed ghost (8 per sent pair); the first exchange changes all G ghosts,
        # so its hook update is the pull pass over all pairs (12U) whenever
        # G > U/8 - later ones are counted as push (pairs walked not counted)
        "merge_upd": [12 * reps],
        "merge_exchange": [8 * G + 8 * int(st.sent_pairs) // max(int(st.exchanges), 1)],
        "merge_exch_push": [0],
        "merge_exch_pull": [12 * U * (1 if 8 * G > U else 0) // max(int(st.exchanges), 1)],
        "dist_labels": [12 * n], "dist_plan": [0], "dist_bounds": [0], "scan": [0],
        "dist_pairs_heavy": [0], "merge_init": [0],
    })
    return out


# DRAM bytes per launch measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) for the kernels that lead a workload's step, per
# unit of work, so that a capture on a smaller graph scales to the bench's
# graph: "entry" = CSR entries, "vertex" = vertices.  Each figure comes from
# the capture summarised in the named profiles/ file.
NCU_TRAFFIC = {
    # k_sample_stash, rounds 0 and 1 averaged (173.8 MB and 34.2 MB) on R-MAT
    # scale 22 (4,194,304 vertices)
    "sample": {"per": "vertex", "bytes_per_unit": 103_996_544 / 4_194_304,
               "source": "profiles/local_cc_sample_stash_rmat22_ncu.md"},
    # k_row_scan<4> on R-MAT scale 22 with 4 partitions: 671.7 MB moved for
    # 681.0 MB of algorithmic bytes (its traffic follows both n and m, so it
    # scales as a fraction of the launch's algorithmic bytes)
    "dist_local_count": {"per": "algorithmic", "bytes_per_unit": 671_661_568 / 681_006_024,
                         "source": "profiles/dist_row_scan_rmat22p4_ncu.md"},
}


def ncu_traffic(kernel, n, m, algorithmic=0):
    """DRAM bytes per launch of `kernel` from NCU_TRAFFIC, scaled by the
    launch's units: CSR entries, vertices, or its algorithmic bytes."""
    t = NCU_TRAFFIC.get(kernel)
    if not t:
        return None
    units = {"entry": m, "vertex": n, "algorithmic": algorithmic}[t["per"]]
    how = (f"{t['bytes_per_unit']:.3f} x {units} algorithmic bytes" if t["per"] == "algorithmic"
           else f"{t['bytes_per_unit']:.3f} bytes per {t['per']} x {units}")
    return {"bytes_per_launch": t["bytes_per_unit"] * units, "source": t["source"], "scaled": how}


def roofline_dict(dom, achieved, peak, peak_kind, traffic, bytes_per, bytes_lists, per,
                  step_bytes, whole):
    """The line's roofline object for the dominant kernel: achieved =
    algorithmic bytes per launch / mean launch time (CUDA events on the
    launching stream), frac = achieved / measured peak; traffic = ncu DRAM
    bytes per launch (scaled from the capture) or null."""
    b = bytes_per.get(dom, 0)
    d = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
         "frac": achieved / peak, "peak_source": peak_kind,
         "traffic": traffic["bytes_per_launch"] if traffic else None,
         "bytes_per_launch": b, "ms_per_launch": per[dom][0],
         "whole_solve": {"algorithmic_bytes": step_bytes, "achieved": whole,
                         "frac": whole / peak}}
    if len(bytes_lists.get(dom, [])) > 1:
        d["bytes_per_launch_each"] = bytes_lists[dom]
    if traffic:
        d["traffic_over_algorithmic"] = traffic["bytes_per_launch"] / b if b else None
        d["traffic_source"] = traffic["source"]
        d["traffic_scaled"] = traffic["scaled"]
    return d


def release_pinned(torch):
    """Hands torch's cached pinned host blocks back to the system."""
    fn = getattr(torch._C, "_host_emptyCache", None)
    if fn:
        fn()


def run_dist(args, torch, dist_mod, rank, world, dev):
    """Partitioned workloads: a step is one ccgpu_dist_cc solve (all
    partitions device-resident) - the timed region of the reference's
    benchmark, one compute_connected_components_mpi_advanced call.

    Parity, on rank 0: the labels must equal those of the reference's own
    compute_connected_components_pthreads on the same graph (its labels are
    the minimum vertex id of each component, the contract of
    include/cc_mpi.h:26-27), and the component count, partition bounds and
    boundary / dedup / ghost totals must equal what the reference's own MPI
    path prints when it runs as the CPU baseline; graphs the oracle finishes
    in seconds are also checked against its restatement (round and exchange
    counts included)."""
    import numpy as np
    from cc_mpi_b200 import _lib, cc, dist
    spec = WORKLOADS[args.workload]
    L = _lib.lib()
    parts = args.parts or spec["parts"]
    t0 = time.perf_counter()
    rp_d, col_d = make_graph(torch, args.workload, args.seed + rank)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # hand the generator's cached blocks back for the solver's pool
    gen_s = time.perf_counter() - t0
    n, m = rp_d.numel() - 1, col_d.numel()
    log(f"{args.workload}: n={n} m={m} generated in {gen_s:.1f} s")
    lab = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def solve():
        return dist.dist_cc_device(rp_d, col_d, n, m, parts, 1, args.chunk, args.exchange,
                                   d_labels=lab, stream=sptr)

    st, bounds = solve()
    torch.cuda.synchronize()
    # the unpartitioned union-find solve and the device invariants: a check
    # that needs no host copy (it cannot tell merged components apart, the
    # reference comparison below does)
    ref = torch.empty(n, dtype=torch.int32, device=dev)
    cc.local_cc_device(rp_d, col_d, n, m, ref, stream=sptr)
    torch.cuda.synchronize()
    same_as_unpartitioned = bool(torch.equal(ref, lab)) and \
        cc.check_labels_device(rp_d, col_d, n, m, lab) == 0
    del ref
    ldeg = local_degrees(torch, rp_d, col_d, bounds)
    st.parts = parts
    bytes_lists = dist_bytes(torch, ldeg, n, m, st, args.chunk)
    del ldeg
    torch.cuda.empty_cache()
    for _ in range(args.warmup):
        flush.fill_(1)
        st, bounds = solve()  # the last warm solve's statistics are reported
    torch.cuda.synchronize()

    def timed_steps():
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        if world > 1:
            dist_mod.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(i)
            ev[i][0].record(stream)
            solve()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        t = sum(a.elapsed_time(b) for a, b in ev) / args.steps
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist_mod.all_reduce(tt, op=dist_mod.ReduceOp.MAX)
            t = float(tt.item())
        return t

    launches0 = L.ccgpu_ctx_launches(None)
    with ClockSampler(dev.index or 0) as clk:
        t_ms = timed_steps()
    launches = L.ccgpu_ctx_launches(None) - launches0
    k = L.ccgpu_prof_kernels()
    names = [L.ccgpu_prof_name(i).decode() for i in range(k)]
    _lib.check(L.ccgpu_prof_enable(None, 1))
    _lib.check(L.ccgpu_prof_collect(None, None, None))
    t_prof_ms = timed_steps()
    ms = (C.c_double * k)()
    cnt = (C.c_uint64 * k)()
    _lib.check(L.ccgpu_prof_collect(None, ms, cnt))
    _lib.check(L.ccgpu_prof_enable(None, 0))
    per = {names[i]: (ms[i] / cnt[i], int(cnt[i])) for i in range(k) if cnt[i]}
    total_kernel_ms = {kk: v[0] * v[1] / args.steps for kk, v in per.items()}
    dom = max(total_kernel_ms, key=total_kernel_ms.get)
    bytes_per = per_launch(bytes_lists)
    peak, peak_kind = read_peaks()
    achieved = bytes_per.get(dom, 0) / (per[dom][0] / 1e3) / 1e9
    step_bytes = step_bytes_of(bytes_lists, per, args.steps)
    whole = step_bytes / (t_ms / 1e3) / 1e9
    value = (m // 2) * world / (t_ms / 1e3) / 1e9
    traffic = ncu_traffic(dom, n, m, bytes_per.get(dom, 0))

    # e2e through the reference-facing calls with host buffers
    rp_h = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    col_h = torch.empty(m, dtype=torch.int32, pin_memory=True)
    rp_h.copy_(rp_d)
    col_h.copy_(col_d)
    # labels land in pinned memory, like the inputs (a pageable buffer costs
    # about 10 ms more per C3 step: the driver stages the copy)
    lab_pin = torch.empty(n, dtype=torch.int32, pin_memory=True)
    lab_h = lab_pin.numpy().view(np.uint32)
    vp = C.c_void_p
    L.cc_group_create.restype = vp
    L.cc_group_create.argtypes = [C.c_int]
    L.cc_group_set_verbose.argtypes = [vp, C.c_int]
    L.cc_group_free.argtypes = [vp]
    L.dist_csr_from_csr.argtypes = [C.POINTER(_lib.CSRGraph), C.c_int,
                                    C.POINTER(_lib.DistCSRGraph), vp]
    L.free_dist_csr_view.argtypes = [C.POINTER(_lib.DistCSRGraph)]
    L.cc_mpi_solve.argtypes = [C.POINTER(_lib.DistCSRGraph), vp, C.c_int, C.c_int, vp, vp]
    grp = L.cc_group_create(parts)
    L.cc_group_set_verbose(grp, 0)
    g = _lib.CSRGraph()
    g.n, g.m = n, m
    g.row_ptr = C.cast(rp_h.data_ptr(), C.POINTER(C.c_uint64))
    g.col_idx = C.cast(col_h.data_ptr(), C.POINTER(C.c_uint32))
    e2e_t = []
    for _ in range(max(args.e2e_steps, 1) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Gd = _lib.DistCSRGraph()
        if L.dist_csr_from_csr(C.byref(g), 1, C.byref(Gd), grp) != 0:
            raise RuntimeError("dist_csr_from_csr failed: " + L.ccgpu_last_error().decode())
        _lib.check(L.cc_mpi_solve(C.byref(Gd), lab_h.ctypes.data, args.chunk, args.exchange,
                                  grp, None))
        L.free_dist_csr_view(C.byref(Gd))
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e_t[1:])  # host wall clock: the median resists stray slow steps
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        dist_mod.all_reduce(tt, op=dist_mod.ReduceOp.MAX)
        e2e_s = float(tt.item())
    got = lab.cpu().numpy().view(np.uint32)
    e2e_ok = bool((lab_h == got).all())
    L.cc_group_free(grp)

    # parity with the reference, on rank 0
    rp_np, col_np = rp_h.numpy().view(np.uint64), col_h.numpy().view(np.uint32)
    parity = {"same_as_unpartitioned_solve": same_as_unpartitioned}
    pth = None
    if rank == 0 and not args.no_verify:
        pth, ref_labels = cpu_baseline(rp_np, col_np, budget_s=0.0 if world > 1 else 30.0)
        parity["labels_equal_reference_pthreads"] = bool((got == ref_labels).all())
        parity["components_equal_reference_pthreads"] = \
            int(np.count_nonzero(ref_labels == np.arange(n, dtype=np.uint32))) == int(st.roots)
        del ref_labels
        if m < 1_200_000_000:
            import oracle
            want, obounds, ost = oracle.dist_cc(rp_np, col_np, parts, 1, args.exchange)
            parity["oracle_labels_rounds_exchanges"] = bool((got == want).all()) and \
                ost.rounds == st.rounds and ost.exchanges == st.exchanges and \
                [int(x) for x in obounds] == [int(x) for x in bounds]
    cpu = pth
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's partitioned path on the same graph, host memory
        # permitting: the graph file is written from the pinned copies, which
        # are released before the run
        import tempfile
        import oracle
        base, why = None, None
        if not oracle.have_ref_mpi():
            why = "reference MPI build (oracle/_ref/mpi_cc_benchmark) absent"
        else:
            fits, why = ref_mpi_memory(n, m, parts, int(st.boundary_raw),
                                       freed=8 * (n + 1) + 4 * m)
            if fits:
                tmp = tempfile.TemporaryDirectory(dir=os.environ.get("CCB200_SCRATCH"))
                try:
                    path, write_s = ref_mpi_write(tmp.name, rp_np, col_np, spec.get("mat", False))
                    del rp_np, col_np, g
                    rp_h = col_h = None
                    release_pinned(torch)
                    base = ref_mpi_time(path, n, m, parts, args.chunk, args.exchange,
                                        spec.get("ref_runs", 1), mat=spec.get("mat", False))
                    base["file_write_s"] = write_s
                except Exception as e:  # the baseline is reported, never the target
                    base, why = None, f"reference MPI run failed: {e}"
                finally:
                    tmp.cleanup()
        if base is not None:
            parity["mpi_components_equal"] = base["components"] == int(st.roots)
            parity["mpi_bounds_equal"] = base["bounds"] == [int(x) for x in bounds]
            parity["mpi_boundary_counts_equal"] = \
                base["boundary_raw"] == int(st.boundary_raw) and \
                base["boundary_dedup"] == int(st.pair_count) and \
                base["ghosts"] == int(st.ghost_count)
            base["pthreads_baseline"] = pth
            cpu = base
        elif pth is not None:
            cpu = dict(pth, mpi_unavailable=why)
    verified = all(parity.values())
    if rank == 0:
        cfg = workload_config(args.workload, n, m)
        cfg.update(partitions=parts, chunk_size=args.chunk, exchange_interval=args.exchange,
                   bounds=[int(x) for x in bounds], components=int(st.roots),
                   rounds=int(st.rounds), exchanges=int(st.exchanges),
                   boundary_raw=int(st.boundary_raw), sorted_keys=int(st.sorted_keys),
                   sorted_rows=bool(st.sorted_rows),
                   boundary_dedup=int(st.pair_count),
                   ghosts=int(st.ghost_count), reps=int(st.rep_count),
                   local_entries=int(st.local_entries),
                   sent_pairs=int(st.sent_pairs), sort_passes=int(st.sort_passes),
                   phases_ms={"bounds": st.ms_bounds, "local": st.ms_local,
                              "pairs": st.ms_pairs, "sort": st.ms_sort,
                              "ghosts": st.ms_ghosts, "merge": st.ms_merge},
                   l2="2x L2 buffer written between timed steps; col_idx > L2",
                   parallelism=f"{parts} partitions on one device" +
                               (f", replicas{world}" if world > 1 else ""),
                   generate_s=gen_s, verified=verified, verified_by_reference=bool(
                       parity.get("labels_equal_reference_pthreads")),
                   parity=parity, e2e_labels_match=e2e_ok)
        line = {
            "metric": "CC GTEPS", "value": value, "unit": "GTEPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": cfg,
            "roofline": roofline_dict(dom, achieved, peak, peak_kind, traffic, bytes_per,
                                      bytes_lists, per, step_bytes, whole),
            "kernels": {kk: {"ms": round(v[0], 5), "launches": v[1],
                             "gbs": round(bytes_per.get(kk, 0) / (v[0] / 1e3) / 1e9, 1)}
                        for kk, v in per.items()},
            "ms_per_step_kernel_by_kernel": t_prof_ms,
            "cpu_baseline": cpu,
            "e2e": {"value": (m // 2) * world / e2e_s / 1e9, "unit": "GTEPS",
                    "h2d_bytes_per_step": 8 * (n + 1) + 4 * m, "d2h_bytes_per_step": 4 * n,
                    "ms_per_step": e2e_s * 1e3,
                    "ms_steps": [round(x * 1e3, 2) for x in e2e_t[1:]],
                    "api": "dist_csr_from_csr + compute_connected_components_mpi_advanced "
                           "(pinned host CSR, labels to pinned host memory)"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    return 0


def batch_bytes(vo, eo, rounds_by_class, kinds_sampled):
    """Algorithmic bytes per launch of the batched kernels, summed over the
    classes: init writes 4n; a sampling round reads 8(n+G) of row pointers,
    one column entry per vertex with a long enough row and the own label
    (4n); a shortcut reads and writes labels (8n); the finish pass reads the
    own label (4n) and the row bounds of every vertex (8(n+G)) - rows it
    walks are extra and not counted; the final pass reads and writes labels
    (8n)."""
    n, G = int(vo[-1]), len(vo) - 1
    return {
        "batch_init": 4 * n,
        "batch_sample": 8 * (n + G) + 4 * kinds_sampled + 4 * n,
        "batch_compress": 8 * n,
        "batch_giant": 4096 * G,
        "batch_link": 4 * n + 8 * (n + G),
        "batch_heavy": 0,
        "batch_final": 8 * n,
    }


def run_batch(args, torch, dist_mod, rank, world, dev):
    """Batched workload: a step is one solve of the whole batch - one CUDA
    graph replay of the autotuned plan.  The same graphs solved one by one
    with the single-graph kernel (ccgpu_local_cc in a loop) are timed beside
    it and give the reference labels every graph is compared with."""
    import numpy as np
    from cc_mpi_b200 import _lib, batch, cc
    spec_w = WORKLOADS[args.workload]
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    t0 = time.perf_counter()
    spec = batch.mix_spec(spec_w["graphs"], spec_w["n_min"], spec_w["n_max"],
                          seed=args.seed + rank)
    vo, eo, d_rp, d_col, kinds = batch.build_batch_torch(torch, spec)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    gen_s = time.perf_counter() - t0
    G, N, M = len(spec), int(vo[-1]), int(eo[-1])
    log(f"batch: {G} graphs, {N} vertices, {M} entries, built in {gen_s:.1f} s")
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)

    def plain_loop(out):
        for g in range(G):
            a, b = int(vo[g]), int(vo[g + 1])
            n, m = b - a, int(eo[g + 1] - eo[g])
            if n == 0:
                continue
            cc.local_cc_device(d_rp[a + g:], d_col[int(eo[g]):] if m else d_col, n, m,
                               out[a:b], stream=sptr)

    want = torch.empty(N, dtype=torch.int32, device=dev)
    plain_loop(want)
    d_lab = torch.full((N,), -1, dtype=torch.int32, device=dev)
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab)
    t0 = time.perf_counter()
    tuning = plan.autotune(stream=sptr)
    tune_s = time.perf_counter() - t0
    plan.launch(stream=sptr)
    torch.cuda.synchronize()
    comps, done = plan.results(stream=sptr)
    verified = bool(torch.equal(d_lab, want)) and bool((done == 1).all())
    # the same plan as one persistent launch (kb_persist): labels checked too
    ptune = batch.Tuning()
    C.memmove(C.byref(ptune), C.byref(tuning), C.sizeof(batch.Tuning))
    ptune.persistent = 1
    pplan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab, tuning=ptune)
    d_lab.fill_(-1)
    pplan.launch(stream=sptr)
    torch.cuda.synchronize()
    pcomps, pdone = pplan.results(stream=sptr)
    p_verified = bool(torch.equal(d_lab, want)) and bool((pdone == 1).all()) and \
        bool((pcomps == comps).all())
    verified = verified and p_verified
    oracle_checked = []
    if rank == 0 and not args.no_verify:
        # every graph of at most ORACLE_MAX_N vertices against the oracle's
        # union-find labels, on the host's cores (the C oracle releases the
        # interpreter lock)
        import oracle
        from concurrent.futures import ThreadPoolExecutor
        lab = d_lab.cpu().numpy().view(np.uint32)
        rp_all = d_rp.cpu().numpy().view(np.uint64)
        small = [g for g in range(G) if int(vo[g + 1] - vo[g]) <= ORACLE_MAX_N]

        def check(g):
            a, n = int(vo[g]), int(vo[g + 1] - vo[g])
            rp = rp_all[a + g:a + g + n + 1]
            col = d_col[int(eo[g]):int(eo[g + 1])].cpu().numpy().view(np.uint32)
            ref = oracle.uf_labels(rp, col)
            return bool((batch.labels_of(lab, vo, g) == ref).all()) and \
                int(comps[g]) == oracle.count_components(ref)

        t0 = time.perf_counter()
        with ThreadPoolExecutor(max(1, os.cpu_count() or 1)) as ex:
            oks = list(ex.map(check, small))
        log(f"batch: {len(small)} graphs checked against the oracle in "
            f"{time.perf_counter() - t0:.1f} s")
        verified = verified and all(oks)
        oracle_checked = small
        del rp_all, lab
    for _ in range(args.warmup):
        flush.fill_(1)
        plan.launch(stream=sptr)
    torch.cuda.synchronize()

    def timed(step_fn, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        if world > 1:
            dist_mod.barrier()
        torch.cuda.synchronize()
        for i in range(steps):
            flush.fill_(i)
            ev[i][0].record(stream)
            step_fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        t = sum(a.elapsed_time(b) for a, b in ev) / steps
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist_mod.all_reduce(tt, op=dist_mod.ReduceOp.MAX)
            t = float(tt.item())
        return t

    for _ in range(args.warmup):
        flush.fill_(1)
        pplan.launch(stream=sptr)
    torch.cuda.synchronize()
    with ClockSampler(dev.index or 0) as clk:
        t_graph_ms = timed(lambda: plan.launch(stream=sptr), args.steps)
        t_pers_ms = timed(lambda: pplan.launch(stream=sptr), args.steps)
    persistent = t_pers_ms <= t_graph_ms if args.batch_launch == "best" else \
        args.batch_launch == "persistent"
    t_ms = t_pers_ms if persistent else t_graph_ms
    launches = (pplan if persistent else plan).kernels() * args.steps
    plain_steps = max(1, min(args.steps, 3))
    t_plain_ms = timed(lambda: plain_loop(want), plain_steps)

    k = L.ccgpu_prof_kernels()
    names = [L.ccgpu_prof_name(i).decode() for i in range(k)]
    _lib.check(L.ccgpu_prof_enable(None, 1))
    _lib.check(L.ccgpu_prof_collect(None, None, None))
    t_prof_ms = timed(lambda: plan.run(stream=sptr), args.steps)
    ms = (C.c_double * k)()
    cnt = (C.c_uint64 * k)()
    _lib.check(L.ccgpu_prof_collect(None, ms, cnt))
    _lib.check(L.ccgpu_prof_enable(None, 0))
    per = {names[i]: (ms[i] / cnt[i], int(cnt[i])) for i in range(k) if cnt[i]}
    tot = {kk: v[0] * v[1] / args.steps for kk, v in per.items()}
    dom = max(tot, key=tot.get)
    deg = (d_rp[1:] - d_rp[:-1])
    sampled = int((deg > 0).sum().item())  # rows with at least one entry (an upper bound
    del deg                                # of the entries one sampling round reads)
    bytes_per = batch_bytes(vo, eo, None, sampled)
    peak, peak_kind = read_peaks()
    achieved = bytes_per.get(dom, 0) / (per[dom][0] / 1e3) / 1e9
    step_bytes = sum(bytes_per.get(kk, 0) * v[1] / args.steps for kk, v in per.items())
    whole = step_bytes / (t_ms / 1e3) / 1e9

    # e2e: host buffers through the one-shot public call ccgpu_batch_cc
    # (plan set-up included), copies in and labels out inside the timed region
    e2e = None
    in_bytes = 8 * (N + G) + 4 * M
    if in_bytes <= (24 << 30):
        rp_h = torch.empty(N + G, dtype=torch.int64, pin_memory=True)
        col_h = torch.empty(max(M, 1), dtype=torch.int32, pin_memory=True)
        lab_h = torch.empty(N, dtype=torch.int32, pin_memory=True)
        rp_h.copy_(d_rp)
        col_h.copy_(d_col[:max(M, 1)])
        Lb = batch._bind()
        b = batch.Batch()
        b.graphs = G
        b.h_vtx_off = vo.ctypes.data_as(C.POINTER(C.c_uint64))
        b.h_edge_off = eo.ctypes.data_as(C.POINTER(C.c_uint64))
        b.d_row_ptr, b.d_col, b.d_labels = d_rp.data_ptr(), d_col.data_ptr(), d_lab.data_ptr()
        t_e2e = []
        for it in range(max(args.e2e_steps, 1) + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d_rp.copy_(rp_h, non_blocking=True)
            d_col[:max(M, 1)].copy_(col_h, non_blocking=True)
            _lib.check(Lb.ccgpu_batch_cc(None, C.byref(b), C.byref(ptune if persistent else tuning),
                                         None, sptr))
            lab_h.copy_(d_lab, non_blocking=True)
            torch.cuda.synchronize()
            t_e2e.append(time.perf_counter() - t0)
        e2e_s = sum(t_e2e[1:]) / len(t_e2e[1:])
        e2e = {"value": G * world / e2e_s, "unit": "graphs/s", "gteps": (M // 2) * world / e2e_s
               / 1e9, "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": 4 * N,
               "ms_per_step": e2e_s * 1e3, "labels_match": bool(torch.equal(lab_h.to(dev), want)),
               "api": "ccgpu_batch_cc (one-shot plan + solve) with pinned host buffers"}
        del rp_h, col_h, lab_h
    else:
        e2e = {"value": None, "unit": "graphs/s", "h2d_bytes_per_step": in_bytes,
               "d2h_bytes_per_step": 4 * N,
               "skipped": "packed batch above 24 GB of pinned host memory"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        threads = os.cpu_count() or 1
        rng = np.random.default_rng(args.seed)
        done_g, edges, t_cpu = 0, 0, 0.0
        for g in rng.permutation(G):
            a, n = int(vo[g]), int(vo[g + 1] - vo[g])
            rp = d_rp[a + g:a + g + n + 1].cpu().numpy().view(np.uint64)
            col = d_col[int(eo[g]):int(eo[g + 1])].cpu().numpy().view(np.uint32)
            t0 = time.perf_counter()
            if oracle.have_ref():
                oracle.ref_pthreads_labels(rp, col, threads, 8192)
            else:
                oracle.lp_labels(rp, col)
            t_cpu += time.perf_counter() - t0
            done_g += 1
            edges += len(col) // 2
            if t_cpu > 20.0:
                break
        cpu = {"value": done_g / t_cpu, "unit": "graphs/s", "gteps": edges / t_cpu / 1e9,
               "cores": threads if oracle.have_ref() else 1,
               "kind": "reference" if oracle.have_ref() else "port",
               "sample": f"{done_g} of {G} graphs in seeded random order, solved one by one "
                         f"(compute_connected_components_pthreads, chunk 8192)"}

    if rank == 0:
        classes = plan.class_graphs()
        cfg = {"workload": args.workload, "graphs": G, "vertices": N, "undirected_edges": M // 2,
               "csr_entries": M, "n_range": [spec_w["n_min"], spec_w["n_max"]],
               "mix": "log-uniform vertex counts; ER mean degree 8 / R-MAT ef 16 / grid 10% "
                      "deleted, one third each",
               "graphs_per_class": [int(x) for x in classes], "tuning": tuning.as_dict(),
               "launch": "one persistent launch (kb_persist)" if persistent else
                         "CUDA graph replay of the per-phase kernels",
               "autotune_s": tune_s, "build_s": gen_s,
               "l2": "2x L2 buffer written between timed steps; packed batch > L2",
               "parallelism": f"replicas{world}" if world > 1 else "single",
               "verified_vs_plain_kernel": verified, "oracle_checked_graphs": len(oracle_checked),
               "oracle_checked": f"every graph of at most {ORACLE_MAX_N} vertices"}
        line = {
            "metric": "batched CC graphs/s", "value": G * world / (t_ms / 1e3),
            "unit": "graphs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": cfg,
            "gteps": (M // 2) * world / (t_ms / 1e3) / 1e9,
            "plain_loop": {"ms_per_step": t_plain_ms, "graphs_per_s": G / (t_plain_ms / 1e3),
                           "speedup_of_batch": t_plain_ms / t_ms,
                           "api": "ccgpu_local_cc once per graph"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": None, "bytes_per_launch": bytes_per.get(dom, 0),
                         "ms_per_launch": per[dom][0],
                         "whole_solve": {"algorithmic_bytes": step_bytes, "achieved": whole,
                                         "frac": whole / peak}},
            "kernels": {kk: {"ms": round(v[0], 5), "launches": v[1],
                             "gbs": round(bytes_per.get(kk, 0) / (v[0] / 1e3) / 1e9, 1)}
                        for kk, v in per.items()},
            "ms_per_step_kernel_by_kernel": t_prof_ms,
            "launch_modes": {
                "graph_replay": {"ms_per_step": t_graph_ms, "graphs_per_s": G / (t_graph_ms / 1e3),
                                 "kernels_per_step": plan.kernels()},
                "persistent": {"ms_per_step": t_pers_ms, "graphs_per_s": G / (t_pers_ms / 1e3),
                               "kernels_per_step": pplan.kernels(),
                               "whole_solve_frac": step_bytes / (t_pers_ms / 1e3) / 1e9 / peak}},
            "timing": "value: K solves in the faster launch mode (launch_modes: K replays of "
                      "the CUDA graph of per-phase kernels, K persistent launches); kernels: the "
                      "per-phase kernels launched one by one with events around every launch",
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    plan.close()
    pplan.close()
    return 0


class LabelBuffers:
    """Pinned host label buffers for served requests, reused per pool graph.
    A pageable buffer makes the driver stage each label copy, and the client
    then caps the server at about 33 of the link's 55 GB/s on the served
    mix; pinned ones let it reach about 52.  `reserve` allocates ahead of a
    timed run, so no pinned allocation happens inside it."""

    def __init__(self, torch, pool):
        self.torch = torch
        self.sizes = [len(rp) - 1 for rp, _ in pool]
        self.free = [[] for _ in pool]
        self.keep = []
        self.mu = threading.Lock()

    def _new(self, g):
        import numpy as np
        t = self.torch.empty(max(self.sizes[g], 1), dtype=self.torch.int32, pin_memory=True)
        with self.mu:
            self.keep.append(t)
        return t.numpy().view(np.uint32)[:self.sizes[g]]

    def reserve(self, order):
        import numpy as np
        need = np.bincount(np.asarray(order), minlength=len(self.free))
        for g, k in enumerate(need.tolist()):
            while len(self.free[g]) < k:
                self.free[g].append(self._new(g))

    def get(self, g):
        with self.mu:
            if self.free[g]:
                return self.free[g].pop()
        return self._new(g)

    def put(self, g, a):
        with self.mu:
            self.free[g].append(a)


def serve_run(server, pool, order, rate, seconds, want_comps, want_labels, check_every,
              bufs, closed=False, waiters=16):
    """Feeds requests `order` (pool indices) to `server`: Poisson arrivals at
    `rate` per second for `seconds`, or all at once when `closed`.  Each
    request's labels land in a pinned buffer from `bufs`.  Waiter threads
    collect results (the wait copies labels out of HBM) and check them:
    component count always, full labels every `check_every`-th request.
    Returns latencies (s), achieved throughput, batch sizes and the number of
    mismatches."""
    import queue
    import numpy as np
    rng = np.random.default_rng(12345)
    q = queue.Queue()
    lat, sizes, bad, last = [], [], [0], [0.0]
    mu = threading.Lock()

    def waiter():
        while True:
            item = q.get()
            if item is None:
                return
            i, t, g, lab = item
            _, info = server.wait(t, timeout=600)
            ok = info.components == want_comps[g] and \
                (i % check_every != 0 or bool((lab == want_labels[g]).all()))
            bufs.put(g, lab)
            with mu:
                lat.append(info.t_done - info.t_submit)
                sizes.append(info.batch_graphs)
                bad[0] += not ok
                last[0] = max(last[0], info.t_done)

    th = [threading.Thread(target=waiter, daemon=True) for _ in range(waiters)]
    for t in th:
        t.start()
    t_start = server.now()
    next_t = t_start
    n_sub = 0
    for g in order:
        if not closed:
            next_t += rng.exponential(1.0 / rate)
            if next_t - t_start > seconds:
                break
            d = next_t - server.now()
            if d > 0:
                time.sleep(d)
        rp, col = pool[g]
        lab = bufs.get(g)
        q.put((n_sub, server.submit(rp, col, lab), g, lab))
        n_sub += 1
    for _ in th:
        q.put(None)
    for t in th:
        t.join()
    span = last[0] - t_start
    return {"submitted": n_sub, "graphs_per_s": n_sub / span if span > 0 else None,
            "span_s": span, "latency": lat, "batch_sizes": sizes, "bad": bad[0]}


def run_served(args, torch, dist_mod, rank, world, dev):
    """Served workload: requests drawn from the batched mix (plus 5% R-MAT
    scale-22) arrive as a Poisson stream at 70% and 95% of the measured
    capacity of the continuous-batching server; the same arrival streams
    are replayed against a server that solves one request at a time."""
    import numpy as np
    from cc_mpi_b200 import batch, cc, serve
    spec_w = WORKLOADS[args.workload]
    t0 = time.perf_counter()
    spec = batch.mix_spec(spec_w["pool"], spec_w["n_min"], spec_w["n_max"],
                          seed=args.seed + rank)
    nbig = 4 if spec_w["big_frac"] > 0 else 0
    spec += [("rmat", 1 << spec_w["big_scale"], args.seed + 1000 + i) for i in range(nbig)]
    pool, want_comps, want_labels = [], [], []
    for kind, n, seed in spec:
        rp_d, col_d = batch.build_one_torch(torch, kind, n, seed)
        lab_d = torch.empty(rp_d.numel() - 1, dtype=torch.int32, device=dev)
        st = cc.local_cc_device(rp_d, col_d, rp_d.numel() - 1, col_d.numel(), lab_d, stats=True)
        rp_h = torch.empty(rp_d.numel(), dtype=torch.int64, pin_memory=True)
        col_h = torch.empty(max(col_d.numel(), 1), dtype=torch.int32, pin_memory=True)
        rp_h.copy_(rp_d)
        col_h[:col_d.numel()].copy_(col_d)
        pool.append((rp_h.numpy().view(np.uint64), col_h.numpy().view(np.uint32)[:col_d.numel()]))
        want_comps.append(int(st.components))
        want_labels.append(lab_d.cpu().numpy().view(np.uint32))
        del rp_d, col_d, lab_d
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    gen_s = time.perf_counter() - t0
    P = len(spec) - nbig
    rng = np.random.default_rng(args.seed)
    # request order: a mix graph, or with probability big_frac a scale-22 R-MAT
    nreq = 400000
    big = rng.random(nreq) < spec_w["big_frac"]
    order = np.where(big, P + rng.integers(0, max(nbig, 1), nreq), rng.integers(0, P, nreq))
    seconds = spec_w["seconds"]
    entries = np.array([len(c) for _, c in pool])
    log(f"served: pool of {len(pool)} graphs built in {gen_s:.1f} s")

    def pct(x, q):
        return float(np.percentile(np.array(x) * 1e3, q)) if x else None

    bufs = LabelBuffers(torch, pool)
    cap_n = 1500 * (8 if spec_w["n_max"] <= 100_000 else 1)
    bufs.reserve(order[64:64 + cap_n])
    bufs.reserve(np.arange(len(pool)))  # one per graph for the Poisson runs

    def measure(srv_kw):
        srv = serve.Server(**srv_kw)
        # warm-up and capacity: a closed loop of requests submitted at once
        serve_run(srv, pool, order[:64], 0, 0, want_comps, want_labels, 16, bufs, closed=True)
        # the same requests for both servers, so the capacities compare
        cap = serve_run(srv, pool, order[64:64 + cap_n], 0, 0, want_comps, want_labels, 16,
                        bufs, closed=True)
        out = {"capacity_graphs_per_s": cap["graphs_per_s"], "capacity_bad": cap["bad"]}
        srv.close()
        return out, cap["graphs_per_s"]

    def poisson(srv_kw, rate, offset):
        srv = serve.Server(**srv_kw)
        r = serve_run(srv, pool, order[offset:], rate, seconds, want_comps, want_labels, 16,
                      bufs)
        st = srv.stats()
        srv.close()
        sub = order[offset:offset + r["submitted"]]
        return {"offered_per_s": rate, "submitted": r["submitted"],
                "graphs_per_s": r["graphs_per_s"],
                "gteps": float(entries[sub].sum() / 2 / r["span_s"] / 1e9) if r["span_s"] else None,
                "p50_ms": pct(r["latency"], 50), "p99_ms": pct(r["latency"], 99),
                "mean_batch": float(np.mean(r["batch_sizes"])) if r["batch_sizes"] else None,
                "max_in_flight": int(st.max_in_flight), "pool_peak_bytes": int(st.pool_peak),
                "mismatches": r["bad"]}

    kw = dict(hbm_bytes=40 << 30, max_graphs=8192, max_batch=4096, streams=2)
    kw1 = dict(hbm_bytes=40 << 30, max_graphs=8192, max_batch=1, streams=1)
    cap_b, capacity = measure(kw)
    cap_1, _ = measure(kw1)
    runs, runs1 = [], []
    for i, frac in enumerate((0.70, 0.95)):
        rate = frac * capacity
        runs.append(dict(load=frac, **poisson(kw, rate, 20000 + i * 180000)))
        runs1.append(dict(load=frac, **poisson(kw1, rate, 20000 + i * 180000)))
    ok = all(r["mismatches"] == 0 for r in runs + runs1) and cap_b["capacity_bad"] == 0 and \
        cap_1["capacity_bad"] == 0
    if rank == 0:
        top = runs[-1]
        line = {
            "metric": "served CC graphs/s", "value": top["graphs_per_s"], "unit": "graphs/s",
            "n_gpus": world, "steps": len(runs), "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": args.workload, "pool_graphs": len(pool),
                       "request_mix": f"log-uniform {spec_w['n_min']}-{spec_w['n_max']} "
                                      "vertices, ER/R-MAT/grid thirds" +
                                      (f" + {int(spec_w['big_frac'] * 100)}% R-MAT scale "
                                       f"{spec_w['big_scale']}" if nbig else ""),
                       "arrivals": "Poisson at 0.70 and 0.95 x measured capacity",
                       "seconds_per_run": seconds, "server": kw, "build_s": gen_s,
                       "verified": ok},
            "capacity": cap_b, "runs": runs,
            "one_at_a_time": dict(cap_1, runs=runs1, server=kw1),
            "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
            "e2e": {"value": top["graphs_per_s"], "unit": "graphs/s",
                    "note": "host CSR in, host labels out: every request's copies are inside "
                            "its latency"},
            "clocks": None,
        }
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-launch", choices=["best", "graph", "persistent"], default="best",
                    help="batched workloads: launch mode of the headline value")
    ap.add_argument("--hook-mode", type=int, default=-1, help="ccgpu_cc_opts.hook_mode")
    ap.add_argument("--sample-rounds", type=int, default=-1)
    ap.add_argument("--parts", type=int, default=0, help="partitions (partitioned workloads)")
    ap.add_argument("--chunk", type=int, default=8192, help="-c of the partitioned workloads")
    ap.add_argument("--exchange", type=int, default=1, help="-e of the partitioned workloads")
    ap.add_argument("--ref-runs", type=int, default=0,
                    help="full solves the partitioned reference arm times (-r of its CLI)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))

    import torch
    import torch.distributed as dist
    import datetime
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    if args.impl == "reference":
        rc = run_reference(args, rank, world)
        if world > 1:
            dist.destroy_process_group()
        return rc

    import numpy as np
    from cc_mpi_b200 import _lib, cc
    L = _lib.lib()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if WORKLOADS[args.workload].get("served"):
        rc = run_served(args, torch, dist, rank, world, dev)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return rc
    if WORKLOADS[args.workload].get("batch"):
        rc = run_batch(args, torch, dist, rank, world, dev)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return rc
    if WORKLOADS[args.workload].get("dist"):
        rc = run_dist(args, torch, dist, rank, world, dev)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return rc

    rp_d, col_d = make_graph(torch, args.workload, args.seed + rank)
    torch.cuda.synchronize()
    n, m = rp_d.numel() - 1, col_d.numel()
    lab_d = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    opts = _lib.opts(hook_mode=args.hook_mode, sample_rounds=args.sample_rounds)

    # one checked solve: stats + device invariants + oracle on rank 0
    st = cc.local_cc_device(rp_d, col_d, n, m, lab_d, opts, stats=True)
    viol = cc.check_labels_device(rp_d, col_d, n, m, lab_d)
    verified = None
    rp_h = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    col_h = torch.empty(m, dtype=torch.int32, pin_memory=True)
    rp_h.copy_(rp_d)
    col_h.copy_(col_d)
    rp_np = rp_h.numpy().view(np.uint64)
    col_np = col_h.numpy().view(np.uint32)
    if rank == 0 and not args.no_verify:
        import oracle
        want = oracle.uf_labels(rp_np, col_np)
        got = lab_d.cpu().numpy().view(np.uint32)
        verified = bool((got == want).all()) and viol == 0
        if not verified:
            log(f"VERIFY FAILED: {int((got != want).sum())} labels differ, {viol} violations")
    bytes_lists = local_cc_bytes(torch, rp_d[1:] - rp_d[:-1], n, m, opts, st.finish_rows,
                                 st.finish_edges)
    bytes_per = per_launch(bytes_lists)

    for _ in range(args.warmup):
        flush.fill_(1)
        cc.local_cc_device(rp_d, col_d, n, m, lab_d, opts, stream=sptr)
    torch.cuda.synchronize()

    # the whole solve captured once as a CUDA graph (ccgpu_local_cc_plan)
    plan = C.c_void_p()
    _lib.check(L.ccgpu_local_cc_plan(rp_d.data_ptr(), col_d.data_ptr(), n, m, lab_d.data_ptr(),
                                     C.byref(opts), C.byref(plan)))
    plan_kernels = L.ccgpu_plan_kernels(plan)
    for _ in range(args.warmup):
        flush.fill_(1)
        _lib.check(L.ccgpu_plan_launch(plan, sptr))
    torch.cuda.synchronize()

    def timed_steps(step_fn):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(i)  # evicts the labels from L2 between steps (not timed)
            ev[i][0].record(stream)
            step_fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t = sum(a.elapsed_time(b) for a, b in ev) / args.steps
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    # timed region (headline): K graph replays
    with ClockSampler(local) as clk:
        t_ms = timed_steps(lambda: L.ccgpu_plan_launch(plan, sptr))
    launches = plan_kernels * args.steps
    edges_all = (m // 2) * world
    value = edges_all / (t_ms / 1e3) / 1e9

    # the same K steps launched kernel by kernel with the library's launch
    # profiler on: CUDA events on the launching stream around every kernel
    k = L.ccgpu_prof_kernels()
    names = [L.ccgpu_prof_name(i).decode() for i in range(k)]
    _lib.check(L.ccgpu_prof_enable(None, 1))
    _lib.check(L.ccgpu_prof_collect(None, None, None))
    t_prof_ms = timed_steps(lambda: cc.local_cc_device(rp_d, col_d, n, m, lab_d, opts,
                                                       stream=sptr))
    ms = (C.c_double * k)()
    cnt = (C.c_uint64 * k)()
    _lib.check(L.ccgpu_prof_collect(None, ms, cnt))
    _lib.check(L.ccgpu_prof_enable(None, 0))
    L.ccgpu_plan_destroy(plan)

    # per-kernel live timing -> dominant kernel roofline
    per = {names[i]: (ms[i] / cnt[i], int(cnt[i])) for i in range(k) if cnt[i]}
    dom = max(per, key=lambda kk: per[kk][0] * per[kk][1])
    peak, peak_kind = read_peaks()
    achieved = bytes_per.get(dom, 0) / (per[dom][0] / 1e3) / 1e9
    total_bytes = step_bytes_of(bytes_lists, per, args.steps)
    whole = total_bytes / (t_ms / 1e3) / 1e9

    # e2e through the reference-facing call with pinned host buffers
    cc._bind()
    lab_h = torch.empty(n, dtype=torch.int32, pin_memory=True)
    g = _lib.CSRGraph()
    g.n, g.m = n, m
    g.row_ptr = C.cast(rp_h.data_ptr(), C.POINTER(C.c_uint64))
    g.col_idx = C.cast(col_h.data_ptr(), C.POINTER(C.c_uint32))
    L.ccb200_set_exit_on_error(0)
    L.compute_connected_components_pthreads(C.byref(g), lab_h.data_ptr(), 0, 4096)  # warm
    e2e_t = []
    for _ in range(max(args.e2e_steps, 1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.ccgpu_clear_error()
        L.compute_connected_components_pthreads(C.byref(g), lab_h.data_ptr(), 0, 4096)
        e2e_t.append(time.perf_counter() - t0)
        if L.ccgpu_last_error():
            raise RuntimeError(L.ccgpu_last_error().decode())
    e2e_s = sum(e2e_t) / len(e2e_t)
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_ok = bool((lab_h.numpy() == lab_d.cpu().numpy()).all())

    cpu = None
    by_reference = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_labels = cpu_baseline(rp_np, col_np)
        by_reference = bool((lab_d.cpu().numpy().view(np.uint32) == ref_labels).all())
        del ref_labels

    if rank == 0:
        cfg = workload_config(args.workload, n, m)
        cfg.update(components=int(st.components), giant_label=int(st.giant_label),
                   l2="2x L2 buffer written between timed steps; col_idx > L2",
                   opts={"chunk_size": opts.chunk_size, "sample_rounds": opts.sample_rounds,
                         "heavy_degree": opts.heavy_degree, "skip_giant": opts.skip_giant,
                         "hook_mode": opts.hook_mode},
                   parallelism=f"replicas{world}" if world > 1 else "single",
                   verified_vs_oracle=verified, verified_by_reference=by_reference,
                   e2e_labels_match=e2e_ok)
        line = {
            "metric": "CC GTEPS", "value": value, "unit": "GTEPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": cfg,
            "roofline": roofline_dict(dom, achieved, peak, peak_kind, ncu_traffic(dom, n, m, bytes_per.get(dom, 0)),
                                      bytes_per, bytes_lists, per, total_bytes, whole),
            "kernels": {kk: {"ms": round(v[0], 5), "launches": v[1],
                             "gbs": round(bytes_per.get(kk, 0) / (v[0] / 1e3) / 1e9, 1)}
                        for kk, v in per.items()},
            "ms_per_step_kernel_by_kernel": t_prof_ms,
            "timing": "value: K replays of the solve's CUDA graph; kernels/roofline: the same "
                      "K steps launched kernel by kernel with events around every launch",
            "cpu_baseline": cpu,
            "e2e": {"value": (m // 2) * world / e2e_s / 1e9, "unit": "GTEPS",
                    "h2d_bytes_per_step": 8 * (n + 1) + 4 * m, "d2h_bytes_per_step": 4 * n,
                    "ms_per_step": e2e_s * 1e3,
                    "api": "compute_connected_components_pthreads (pinned host CSR)"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
