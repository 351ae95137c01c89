"""Benchmark: neighbor rows/s at 1,048,576 x 1,048,576 3D (exact row set).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

One step is one plain per-call launch of the hot path over one batch: build
the LBVH over the 1,048,576 build points, run fixed-radius neighbors
(radius 0.00287, k_max 64, mean ~28.5 rows per probe) for 1,048,576 probes and
write the exact rows (RtdlFixedRadiusNeighborRow, FP64 distances) to HBM.
Inputs are resident in HBM before timing; L2 is flushed (a 512 MiB write)
between timed steps; each step is timed with CUDA events on the stream the
library launches on, and the job time is the max over ranks.

Multi-GPU (torchrun, one process per GPU): every rank holds a replica of the
build set and answers its own 1,048,576 probes (weak scaling, no data-path
collective); `value` is the rows of all ranks divided by the slowest rank's
time.

`e2e` is the same metric through the C ABI entry point
rtdl_b200_run_fixed_radius_neighbors_3d with pinned host buffers: the timed
region holds the host-to-device copy of both point sets and the device-to-host
copy of the rows.

`--impl reference` times the reference's own CPU implementation of the path
(its native oracle, compiled from its sources into oracle/_ref/, sharded over
all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "neighbor rows/s at 1M x 1M 3D (exact row set)"
UNIT = "rows/s"
RADIUS = 0.00287
K_MAX = 64
N_BUILD = 1 << 20
N_PROBE = 1 << 20
L2_FLUSH_BYTES = 512 << 20


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_traffic(kernel: str, workload: str, probes: int, build: int):
    """DRAM bytes (read + write) of one launch of `kernel`, from the committed ncu capture of the same workload.

    None when no capture of exactly this kernel and size is on record.
    """
    try:
        table = json.loads((ROOT / "profiles" / "dram_traffic.json").read_text())
    except (OSError, ValueError):
        return None
    for e in table.get("entries", []):
        if (e.get("kernel"), e.get("workload"), e.get("probes"), e.get("build")) == (kernel, workload, probes, build):
            return int(e["read_bytes"]) + int(e["write_bytes"])
    return None


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ---------------------------------------------------------------------------
# CPU baselines
# ---------------------------------------------------------------------------

def cpu_baseline_port(probe, build, threads: int, budget_s: float = 10.0) -> dict:
    """The oracle restatement (oracle/nn_oracle.c) on a bounded sample of probes."""
    from oracle import oracle as O

    rng = np.random.default_rng(123)
    n = 64 * threads
    idx = np.sort(rng.choice(len(probe), n, replace=False))
    t0 = time.perf_counter()
    rows = O.fixed_radius_neighbors(probe[idx], build, radius=RADIUS, k_max=K_MAX, threads=threads)
    dt = time.perf_counter() - t0
    scale = max(1.0, min(64.0, budget_s / max(dt, 1e-3)))
    n2 = min(len(probe), int(n * scale))
    if n2 > n:
        idx = np.sort(rng.choice(len(probe), n2, replace=False))
        t0 = time.perf_counter()
        rows = O.fixed_radius_neighbors(probe[idx], build, radius=RADIUS, k_max=K_MAX, threads=threads)
        dt = time.perf_counter() - t0
    return {"value": len(rows) / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(idx)} seeded probes x all {len(build)} build points, {len(rows)} rows in {dt:.2f} s"}


def external_scipy_baseline(probe, build, threads: int, n_sample: int = 50_000) -> dict | None:
    """The reference's external SciPy cKDTree baseline (``external_baselines.py``: ball query, hypot
    distance, sort by (distance, id), first k_max) on a bounded probe sample, all host threads for the
    ball queries.  Its hypot distances are not bit-identical to the reference's rows."""
    try:
        from scipy.spatial import cKDTree
    except Exception:
        return None
    rng = np.random.default_rng(321)
    idx = np.sort(rng.choice(len(probe), min(n_sample, len(probe)), replace=False))
    b = np.stack([build["x"], build["y"], build["z"]], 1)
    q = np.stack([probe["x"][idx], probe["y"][idx], probe["z"][idx]], 1)
    bid = build["id"]
    t0 = time.perf_counter()
    tree = cKDTree(b)
    hits = tree.query_ball_point(q, r=RADIUS, workers=threads)
    rows = 0
    for i, cand in enumerate(hits):
        if not cand:
            continue
        c = np.asarray(cand)
        d = np.hypot(np.hypot(b[c, 0] - q[i, 0], b[c, 1] - q[i, 1]), b[c, 2] - q[i, 2])
        keep = d <= RADIUS
        order = np.lexsort((bid[c][keep], d[keep]))
        rows += min(len(order), K_MAX)
    dt = time.perf_counter() - t0
    return {"value": rows / dt, "unit": UNIT, "cores": threads, "kind": "external (scipy cKDTree)",
            "sample": f"{len(idx)} seeded probes x all {len(build)} build points (tree build included), "
                      f"{rows} rows in {dt:.2f} s"}


def cpu_reference_step(probe_idx, packed_build, probe, threads):
    """One bounded sample of the reference's native oracle, sharded over threads."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O

    shards = np.array_split(probe_idx, threads)
    packed = [O.pack_reference_points(probe[s]) for s in shards if len(s)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        results = list(ex.map(lambda pq: O.reference_fixed_radius_neighbors(pq, packed_build, radius=RADIUS, k_max=K_MAX), packed))
    dt = time.perf_counter() - t0
    return sum(len(r) for r in results), dt


def run_reference_arm(args) -> int:
    rank = _env_int("RANK", 0)
    if rank != 0:
        return 0
    from oracle import oracle as O
    from rtdl_b200 import workloads

    threads = os.cpu_count() or 1
    probe, build = workloads.clustered_3d(N_BUILD, N_PROBE)
    if O.reference_library_available():
        kind = "reference"
        packed_build = O.pack_reference_points(build)
        rng = np.random.default_rng(321)
        # size one step to ~4 s of CPU work: calibrate on a small sample first
        probe_idx = np.sort(rng.choice(len(probe), 8 * threads, replace=False))
        rows, dt = cpu_reference_step(probe_idx, packed_build, probe, threads)
        per_step = int(min(len(probe), max(8 * threads, 8 * threads * (4.0 / max(dt, 1e-3)))))
        samples = []
        for i in range(args.warmup + args.steps):
            idx = np.sort(rng.choice(len(probe), per_step, replace=False))
            rows, dt = cpu_reference_step(idx, packed_build, probe, threads)
            if i >= args.warmup:
                samples.append((rows, dt))
        total_rows = sum(r for r, _ in samples)
        total_t = sum(t for _, t in samples)
        value = total_rows / total_t
        sample = (f"{per_step} seeded probes per step x all {len(build)} build points; reference native oracle "
                  f"(src/native/oracle/rtdl_oracle_api.cpp) sharded over {threads} threads")
    else:
        kind = "port"
        base = cpu_baseline_port(probe, build, threads)
        value, total_t, sample = base["value"], None, base["sample"]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": (total_t / max(1, args.steps) * 1e3) if total_t else None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "clustered_3d_fixed_radius", "build": N_BUILD, "probe": N_PROBE, "radius": RADIUS,
                   "k_max": K_MAX, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# secondary workloads (one GPU): knn k=16 and directed Hausdorff
# ---------------------------------------------------------------------------

def run_secondary(args) -> int:
    import torch

    import rtdl_b200 as rt
    from oracle import oracle as O
    from rtdl_b200 import _native, workloads

    torch.cuda.set_device(0)
    rt.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    if args.workload == "knn":
        probe, build = workloads.clustered_3d()
        k = 16
        units = len(probe) * k
        metric, unit = "knn rows/s at 1M x 1M 3D, k=16 (exact row set)", "rows/s"
    else:
        probe, build = workloads.hausdorff_2d()
        units = len(probe)
        metric, unit = "directed Hausdorff nearest rows/s at 4M x 4M 2D (FP64 max-min)", "rows/s"
    dim = 3 if args.workload == "knn" else 2
    d_build = torch.from_numpy(build.view(np.uint8)).to(dev)
    d_probe = torch.from_numpy(probe.view(np.uint8)).to(dev)
    rows_buf = torch.empty(units * 24, dtype=torch.uint8, device=dev) if args.workload == "knn" else None
    nd = torch.empty(len(probe), dtype=torch.float64, device=dev)
    ni = torch.empty(len(probe), dtype=torch.int32, device=dev)
    result = {}

    def step():
        scene = rt.B200Scene(None, dimension=dim, stream=sh, device_points=(d_build.data_ptr(), len(build)))
        try:
            if args.workload == "knn":
                n = scene.query_device(d_probe.data_ptr(), len(probe), predicate="knn_rows", limit=k,
                                       rows_address=rows_buf.data_ptr(), rows_capacity=units, stream=sh)
                assert n == units
            else:
                result.update(scene.directed_hausdorff_device(d_probe.data_ptr(), len(probe),
                                                              nearest_distance_address=nd.data_ptr(),
                                                              nearest_id_address=ni.data_ptr(), stream=sh))
            return _native.last_phase_timings()
        finally:
            scene.close()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    launches0 = _native.launch_count()
    torch.cuda.synchronize()
    ms, phases = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
        phases.append(step())
        with torch.cuda.stream(stream):
            b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    torch.cuda.synchronize()
    launches = _native.launch_count() - launches0
    clocks = sampler.stop()
    ms_step = sum(ms) / len(ms)
    trav = sum(p.get("traverse", 0.0) for p in phases) / len(phases)
    # exactness against the FP64 oracle on a seeded sample of queries
    rng = np.random.default_rng(99)
    sample = np.sort(rng.choice(len(probe), 256, replace=False))
    if args.workload == "knn":
        got = np.frombuffer(rows_buf.cpu().numpy().tobytes(), dtype=rt.runtime.KNN_ROW_DTYPE).reshape(-1, k)[sample]
        exp = O.knn_rows(probe[sample], build, k=k, threads=os.cpu_count() or 1).reshape(-1, k)
        ids_equal = bool(np.array_equal(got["neighbor_id"], exp["neighbor_id"]))
        max_err = float(np.max(np.abs(got["distance"] - exp["distance"])))
        alg_bytes = len(probe) * 16 + len(build) * 16 + units * 24
    else:
        dist, nid = O.nearest(probe[sample], build, threads=os.cpu_count() or 1)
        got_d = nd.cpu().numpy()[sample]
        ids_equal = bool(np.array_equal(ni.cpu().numpy().view(np.uint32)[sample], nid))
        max_err = float(np.max(np.abs(got_d - dist)))
        alg_bytes = len(probe) * 16 + len(build) * 16 + len(probe) * 12
    try:
        hbm_peak = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except Exception:
        hbm_peak = 6650.0
    achieved = alg_bytes / (trav / 1e3) / 1e9 if trav > 0 else None
    line = {
        "metric": metric, "value": units / (ms_step / 1e3), "unit": unit, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 traversal + f64 band recheck and distances", "data": "synthetic",
        "config": {"workload": args.workload, "build": len(build), "probe": len(probe),
                   "l2": "flushed between steps (512 MiB write)"},
        "phases_ms": {k2: sum(p.get(k2, 0.0) for p in phases) / len(phases) for k2 in ("query_prep", "traverse", "scan", "emit", "reduce")},
        "roofline": {"bound": "hbm", "kernel": "k_pass1 (KNN list traversal)", "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": (achieved / hbm_peak) if achieved else None, "traffic": None,
                     "algorithmic_bytes": alg_bytes},
        "exactness": {"sample_queries": int(len(sample)), "ids_equal_to_oracle": ids_equal,
                      "max_abs_distance_error_vs_fp64_oracle": max_err},
        "hausdorff": result if args.workload == "hausdorff" else None,
        "clocks": clocks, "gpu_launches": launches,
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def _plan_chunks(nb: np.ndarray, nq: np.ndarray, max_build: int, max_probe: int) -> list[tuple[int, int]]:
    """Consecutive problem ranges [a, b) whose build / probe totals stay within one batch's limits."""
    chunks, a, sb, sq = [], 0, 0, 0
    for i in range(len(nb)):
        if i > a and (sb + nb[i] > max_build or sq + nq[i] > max_probe):
            chunks.append((a, i))
            a, sb, sq = i, 0, 0
        sb += int(nb[i])
        sq += int(nq[i])
    chunks.append((a, len(nb)))
    return chunks


def run_batch(args) -> int:
    """2,048 uneven 3D fixed-radius problems: problem batches (one build + one launch sequence per batch)
    against one plain per-call launch per problem, in the same run."""
    import torch

    import rtdl_b200 as rt
    from oracle import oracle as O
    from rtdl_b200 import _native, workloads
    from rtdl_b200.batch import B200ProblemBatch, concat_records

    torch.cuda.set_device(0)
    rt.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    probs = workloads.batched_problems(count=args.problems)
    probes = [p[0] for p in probs]
    builds = [p[1] for p in probs]
    radius = np.array([p[2] for p in probs], dtype=np.float64)
    kmax = np.array([p[3] for p in probs], dtype=np.uint32)
    nb = np.array([len(b) for b in builds], dtype=np.int64)
    nq = np.array([len(q) for q in probes], dtype=np.int64)
    boff = np.zeros(len(probs) + 1, dtype=np.uint64)
    boff[1:] = np.cumsum(nb)
    qoff = np.zeros(len(probs) + 1, dtype=np.uint64)
    qoff[1:] = np.cumsum(nq)
    d_build = torch.from_numpy(concat_records(builds).view(np.uint8)).to(dev)
    d_probe = torch.from_numpy(concat_records(probes).view(np.uint8)).to(dev)
    del probs
    chunks = _plan_chunks(nb, nq, 32 << 20, 8 << 20)
    # autotune (leaf size and block size; batches always walk in warp packets) on the median-size problem
    from dataclasses import asdict

    from rtdl_b200.autotune import Autotuner

    med = int(np.argsort(nb * nq)[len(nb) // 2])
    tuner = Autotuner(repeats=2, traversals=("packet",))
    tune_key, tune_cfg = tuner.tune(d_build.data_ptr() + 32 * int(boff[med]), int(nb[med]),
                                    d_probe.data_ptr() + 32 * int(qoff[med]), int(nq[med]), dimension=3,
                                    radius=float(radius[med]), k_max=int(kmax[med]), stream=sh)

    def batch_step(rows_buf, cap, sizes_out=None):
        total = 0
        for ci, (a, b) in enumerate(chunks):
            ba, qa = int(boff[a]), int(qoff[a])
            with B200ProblemBatch(None, dimension=3, stream=sh,
                                  device_points=(d_build.data_ptr() + 32 * ba, boff[a:b + 1] - boff[a])) as batch:
                offs = batch.fixed_radius_neighbors_device(
                    d_probe.data_ptr() + 32 * qa, qoff[a:b + 1] - qoff[a], radius=radius[a:b], k_max=kmax[a:b],
                    rows_address=rows_buf.data_ptr() if rows_buf is not None else None,
                    rows_capacity=cap, stream=sh)
            if sizes_out is not None:
                sizes_out.append(offs)
            total += int(offs[-1])
        return total

    def plain_step(rows_buf, cap, sizes_out=None):
        total = 0
        for i in range(len(nb)):
            scene = rt.B200Scene(None, dimension=3, stream=sh,
                                 device_points=(d_build.data_ptr() + 32 * int(boff[i]), int(nb[i])))
            try:
                n = scene.query_device(d_probe.data_ptr() + 32 * int(qoff[i]), int(nq[i]),
                                       predicate="fixed_radius_neighbors", radius=float(radius[i]), limit=int(kmax[i]),
                                       rows_address=rows_buf.data_ptr() if rows_buf is not None else None,
                                       rows_capacity=cap, stream=sh)
            finally:
                scene.close()
            if sizes_out is not None:
                sizes_out.append(n)
            total += n
        return total

    chunk_sizes, plain_sizes = [], []
    rows_total = batch_step(None, 0, chunk_sizes)
    max_chunk_rows = max(int(o[-1]) for o in chunk_sizes)
    rows_buf = torch.empty(max_chunk_rows * 16, dtype=torch.uint8, device=dev)
    assert plain_step(None, 0, plain_sizes) == rows_total
    plain_buf = torch.empty(max(plain_sizes) * 16, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        batch_step(rows_buf, max_chunk_rows)
    torch.cuda.synchronize()

    def timed(fn, buf, cap, steps):
        ms = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            fn(buf, cap)
            with torch.cuda.stream(stream):
                b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return ms

    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    launches0 = _native.launch_count()
    ms = timed(batch_step, rows_buf, max_chunk_rows, args.steps)
    launches = _native.launch_count() - launches0
    clocks = sampler.stop()
    plain_ms = timed(plain_step, plain_buf, max(plain_sizes), 1)
    ms_step = sum(ms) / len(ms)

    # exactness: sampled problems, batch rows against the plain call and (small ones) against the oracle
    rng = np.random.default_rng(17)
    sample = sorted(rng.choice(len(nb), 12, replace=False).tolist())
    equal_plain, oracle_checked, equal_oracle = True, 0, True
    for i in sample:
        ci = next(c for c, (a, b) in enumerate(chunks) if a <= i < b)
        a, b = chunks[ci]
        ba, qa = int(boff[a]), int(qoff[a])
        with B200ProblemBatch(None, dimension=3, stream=sh,
                              device_points=(d_build.data_ptr() + 32 * ba, boff[a:b + 1] - boff[a])) as batch:
            offs = batch.fixed_radius_neighbors_device(
                d_probe.data_ptr() + 32 * qa, qoff[a:b + 1] - qoff[a], radius=radius[a:b], k_max=kmax[a:b],
                rows_address=rows_buf.data_ptr(), rows_capacity=max_chunk_rows, stream=sh)
        torch.cuda.synchronize()
        lo, hi = int(offs[i - a]), int(offs[i - a + 1])
        got = np.frombuffer(rows_buf[lo * 16: hi * 16].cpu().numpy().tobytes(), dtype=rt.runtime.FRN_ROW_DTYPE)
        probe_i = np.frombuffer(d_probe[32 * int(qoff[i]): 32 * int(qoff[i + 1])].cpu().numpy().tobytes(),
                                dtype=rt.runtime.POINT3D_DTYPE)
        build_i = np.frombuffer(d_build[32 * int(boff[i]): 32 * int(boff[i + 1])].cpu().numpy().tobytes(),
                                dtype=rt.runtime.POINT3D_DTYPE)
        view = rt.runtime.fixed_radius_neighbors(probe_i, build_i, radius=float(radius[i]), k_max=int(kmax[i]))
        ref = view.to_numpy()
        view.close()
        equal_plain &= bool(len(ref) == len(got) and np.array_equal(ref.view(np.uint8), got.view(np.uint8)))
        if len(probe_i) * len(build_i) <= 2e9:
            exp = O.fixed_radius_neighbors(probe_i, build_i, radius=float(radius[i]), k_max=int(kmax[i]),
                                           threads=os.cpu_count() or 1)
            oracle_checked += 1
            equal_oracle &= bool(np.array_equal(exp["neighbor_id"], got["neighbor_id"]) and
                                 np.array_equal(exp["query_id"], got["query_id"]) and
                                 np.array_equal(exp["distance"].view(np.uint64), got["distance"].view(np.uint64)))
    try:
        hbm_peak = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except Exception:
        hbm_peak = 6650.0
    alg = int(nq.sum()) * 16 + int(nb.sum()) * 16 + rows_total * 16 + int(nq.sum()) * 4
    line = {
        "metric": f"neighbor rows/s, {len(nb)} uneven 3D fixed-radius problems (batched)",
        "value": rows_total / (ms_step / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 traversal + f64 band recheck and distances", "data": "synthetic",
        "config": {"workload": f"{len(nb)} problems, nb and nq log-uniform [1024, 262144] (seed 5), box scaled by "
                               "exp(U[-1,1]) per axis, radius for a mean of U[8, 64] neighbours, k_max 64",
                   "build_points": int(nb.sum()), "probes": int(nq.sum()), "rows": rows_total,
                   "batches": len(chunks), "l2": "flushed between steps (512 MiB write)"},
        "plain_per_call": {"value": rows_total / (plain_ms[0] / 1e3), "unit": "rows/s", "ms": plain_ms[0],
                           "launches": "one scene build + one query per problem"},
        "speedup_vs_plain": plain_ms[0] / ms_step,
        "autotune": {"shape_class": tune_key, "config": asdict(tune_cfg), "candidates_ms": tuner.cache[tune_key]["ms"]},
        "roofline": {"bound": "hbm", "kernel": "whole batched step (build + collect + emit)",
                     "achieved": alg / (ms_step / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": alg / (ms_step / 1e3) / 1e9 / hbm_peak, "traffic": None, "algorithmic_bytes": alg},
        "exactness": {"problems_checked": len(sample), "rows_equal_to_plain_call": equal_plain,
                      "oracle_checked": oracle_checked, "rows_equal_to_oracle": equal_oracle},
        "e2e": None, "cpu_baseline": None, "clocks": clocks, "gpu_launches": launches,
    }
    print(json.dumps(line))
    return 0


def serve_trace(seconds: float, rate: float, scenes: dict, pools: dict, seed: int = 6):
    """Poisson arrivals: (arrival_s, scene, op, queries, radius, limit); probes per request log-uniform
    [100, 1M] taken from the scene's probe pool; op uniform over fixed_radius_neighbors (k_max 64, radius for
    ~32 neighbours at the scene's density) and knn_rows with k in {1, 8, 32}."""
    from rtdl_b200.serve import FRN, KNN

    rng = np.random.default_rng(seed)
    names = sorted(scenes)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            return out
        name = names[rng.integers(len(names))]
        pool = pools[name]
        n = min(len(pool), int(np.exp(rng.uniform(np.log(100), np.log(1 << 20)))))
        a = int(rng.integers(0, len(pool) - n + 1))
        q = pool[a: a + n]
        op = int(rng.integers(4))
        if op == 0:
            out.append((t, name, FRN, q, RADIUS * ((1 << 20) / scenes[name]) ** (1.0 / 3.0), 64))
        else:
            out.append((t, name, KNN, q, 0.0, (1, 8, 32)[op - 1]))


def run_serve(args) -> int:
    """Served loop: resident scenes, Poisson arrivals, continuous batching, p50/p99 against the plain
    per-call path on the same trace."""
    import torch

    import rtdl_b200 as rt
    from rtdl_b200 import _native, workloads
    from rtdl_b200.serve import B200Server, replay, run_plain, same_rows

    torch.cuda.set_device(0)
    rt.set_device(0)
    rng = np.random.default_rng(6)
    c = np.random.default_rng(0).random((64, 3))
    sizes = np.exp(rng.uniform(np.log(100_000), np.log(8_000_000), args.scenes)).astype(np.int64)
    points = {f"scene{i:02d}": workloads.records(workloads._mixture(np.random.default_rng(100 + i), int(n), c))
              for i, n in enumerate(sizes)}
    pools = {name: workloads.records(workloads._mixture(np.random.default_rng(200 + i), 1 << 20, c))
             for i, name in enumerate(points)}
    trace = serve_trace(args.serve_seconds, args.rate, {k: len(v) for k, v in points.items()}, pools)
    with B200Server(memory_budget=120 << 30, streams=4) as server:
        for name, p in points.items():
            server.add_scene(name, p)
        replay(server, trace[: min(len(trace), 32)], keep=set())  # warm-up: allocator pools, pinned buffers
        server.completed.clear()
        sample = set(np.random.default_rng(3).choice(len(trace), min(24, len(trace)), replace=False).tolist())
        sampler = ClockSampler(0)
        sampler.start()
        launches0 = _native.launch_count()
        reqs = replay(server, trace, keep=sample)  # rows of the sampled requests are kept for the check
        launches = _native.launch_count() - launches0
        clocks = sampler.stop()
        served = server.stats()
        failed = [r.error for r in reqs if r.error]
        equal = True
        for i in sorted(sample):  # exactness: the sampled requests against the plain call alone
            r = reqs[i]
            view = server.scenes[r.scene].query(r.queries, predicate=r.op, radius=r.radius, limit=r.limit)
            equal &= same_rows(r.rows, view.to_numpy())
            view.close()
        plain = run_plain(server.scenes, reqs, [t[0] for t in trace])
    line = {
        "metric": f"served neighbor rows/s with continuous batching ({args.scenes} resident 3D scenes, "
                  "Poisson arrivals)",
        "value": served.get("rows_per_s"), "unit": "rows/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": served.get("seconds", 0) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 traversal + f64 band recheck and distances", "data": "synthetic",
        "config": {"workload": f"{args.scenes} scenes, sizes log-uniform [100k, 8M] (clustered mixture), "
                               f"{args.rate:.0f} req/s Poisson for {args.serve_seconds} s (seed 6), probes per "
                               "request log-uniform [100, 1M], op uniform over FRN (k_max 64) and KNN k in "
                               "{1, 8, 32}, 120 GB budget, 4 streams",
                   "requests": len(trace), "scene_points": int(sizes.sum()),
                   "timing": "host wall clock per request (arrival to rows in pinned host memory)"},
        "served": served, "plain_per_call": plain,
        "throughput_vs_plain": (served["rows_per_s"] / plain["rows_per_s"]) if served.get("rows_per_s") else None,
        "exactness": {"requests_checked": len(sample), "rows_equal_to_plain_call": equal, "failed": len(failed)},
        "e2e": None, "cpu_baseline": None, "roofline": None, "clocks": clocks, "gpu_launches": launches,
    }
    print(json.dumps(line))
    return 0


def _time_summary_graph(pts, radius, k_max, flush, args):
    """The same request through the captured batch graph (prepared scene + prepared queries): device
    time of a replay (CUDA events on the graph's stream, L2 flushed before each) and the host time of
    replay() (launch, aggregate read back, status check)."""
    import torch

    import rtdl_b200 as rt

    prep = rt.PreparedB200FixedRadiusNeighbors3D(pts, max_radius=radius)
    pq = rt.PreparedB200FixedRadiusQueryPoints3D(pts)
    graph = prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, [{"radius": radius, "k_max": k_max}])
    try:
        for _ in range(args.warmup):
            graph.replay()
        _, _, _, _, gs = graph.launch_device_partials()
        ext = torch.cuda.ExternalStream(gs)
        torch.cuda.synchronize()
        dev_ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(ext):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(ext)
            graph.launch_device_partials()
            with torch.cuda.stream(ext):
                b.record(ext)
            b.synchronize()
            dev_ms.append(a.elapsed_time(b))
        wall_ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(ext):
                flush.zero_()
            ext.synchronize()
            t0 = time.perf_counter()
            (res,) = graph.replay()
            wall_ms.append((time.perf_counter() - t0) * 1e3)
        agg = {f: res[f] for f in ("query_count", "bounded_neighbor_count", "nearest_id_checksum",
                                   "kth_id_checksum", "sum_distance")}
        return dev_ms, wall_ms, agg
    finally:
        graph.close()
        pq.close()
        prep.close()


def run_summary(args) -> int:
    """The reference's own published GPU benchmark: ranked-summary aggregate of fixed_radius_neighbors
    (r = 0.02, k_max = 50) on its three 262,144-point RTNN sets (queries = search points, float32 inputs,
    prepared scene and resident queries), regenerated with its generator; medians beside its RTX A5000
    medians, aggregates checked against its published values."""
    import torch

    import rtdl_b200 as rt
    from rtdl_b200 import _native, workloads

    torch.cuda.set_device(0)
    rt.set_device(0)
    # these scenes serve only fixed-radius queries: the leaf buckets of a prepared fixed-radius scene
    rt.set_tuning(leaf_size=24)
    golden = json.loads((ROOT / "tests" / "golden" / "rtnn_ranked_summary_262144.json").read_text())
    radius, k_max = golden["radius"], golden["k_max"]
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    results, total_ms, launches = {}, 0.0, 0
    sampler = ClockSampler(0)
    sampler.start()
    for dist_name, g in golden["distributions"].items():
        pts = workloads.rtnn_points(dist_name, g["point_count"], g["seed"])
        for c in ("x", "y", "z"):
            pts[c] = pts[c].astype(np.float32).astype(np.float64)
        d_pts = torch.from_numpy(pts.view(np.uint8).copy()).to(dev)
        scene = rt.B200Scene(None, dimension=3, stream=sh, device_points=(d_pts.data_ptr(), len(pts)))
        queries = rt.B200Queries(None, dimension=3, stream=sh, device_points=(d_pts.data_ptr(), len(pts)))

        def timed(call):
            for _ in range(args.warmup):
                call()
            torch.cuda.synchronize()
            out = []
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                res = call()
                with torch.cuda.stream(stream):
                    b.record(stream)
                b.synchronize()
                out.append(a.elapsed_time(b))
            return out, res

        try:
            l0 = _native.launch_count()
            ms, agg = timed(lambda: scene.ranked_summaries_prepared(queries, radius=radius, k_max=k_max, stream=sh))
            launches += _native.launch_count() - l0
            phases = _native.last_phase_timings()
            ms_device, agg_device = timed(lambda: scene.ranked_summaries_device(
                d_pts.data_ptr(), len(pts), radius=radius, k_max=k_max, stream=sh))
            assert agg_device == agg
            graph_ms, graph_wall_ms, agg_graph = _time_summary_graph(pts, radius, k_max, flush, args)
            assert all(agg_graph[f] == agg[f] for f in agg), (agg_graph, agg)
        finally:
            queries.close()
            scene.close()
        exp = g["exact_aggregate"]
        med = float(np.median(ms))
        total_ms += med
        results[dist_name] = {
            "median_ms": med, "runs_ms": ms, "phases_ms": phases,
            "unprepared_queries_median_ms": float(np.median(ms_device)),
            "graph_replay_median_ms": float(np.median(graph_ms)),
            "graph_replay_host_median_ms": float(np.median(graph_wall_ms)),
            "published_reference_median_ms": g["reference_median_s"] * 1e3,
            "published_reference_gpu": golden.get("gpu") or "RTX A5000",
            "published_cupy_grid_median_ms": g["cupy_grid_median_s"] * 1e3,
            "speedup_vs_published_reference": g["reference_median_s"] * 1e3 / med,
            "aggregate": agg,
            "counts_and_checksums_equal_published": all(agg[f] == exp[f] for f in (
                "bounded_neighbor_count", "nearest_id_checksum", "kth_id_checksum")),
            "sum_distance_rel_diff_vs_published": abs(agg["sum_distance"] - exp["sum_distance"]) / exp["sum_distance"],
        }
    clocks = sampler.stop()
    line = {
        "metric": "ranked-summary aggregate time, 262,144 x 262,144 3D RTNN sets (uniform + clustered + shell), "
                  "r=0.02, k_max=50",
        "value": total_ms, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 traversal + f64 band recheck and distances", "data": "synthetic (reference generator)",
        "config": {"workload": "the reference's published ranked-summary benchmark: prepared scene and prepared "
                               "query set (= search points, float32 inputs), as the published runs; step = "
                               "traversal + emit + summaries + aggregate (unprepared_queries_median_ms adds the "
                               "query preparation)", "l2": "flushed between steps (512 MiB write)"},
        "distributions": results, "e2e": None, "cpu_baseline": None, "roofline": None, "clocks": clocks,
        "gpu_launches": launches,
    }
    print(json.dumps(line))
    return 0


def main(argv=None) -> int:
    global N_PROBE, N_BUILD
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--probes", type=int, default=N_PROBE, help="probe points per GPU (profiling a smaller case)")
    ap.add_argument("--build", type=int, default=N_BUILD, help="build points (profiling a smaller case)")
    ap.add_argument("--workload", choices=("frn", "knn", "hausdorff", "batch", "serve", "summary"), default="frn",
                    help="frn: the headline fixed-radius config; knn: k=16 on the same 3D sets; "
                         "hausdorff: 4,194,304 x 4,194,304 2D directed nearest-distance reduction; "
                         "batch: 2,048 uneven fixed-radius problems, batched vs one call per problem; "
                         "serve: request loop over resident scenes vs the plain per-call path; "
                         "summary: the reference's published ranked-summary benchmark")
    ap.add_argument("--problems", type=int, default=2048, help="problems of the batch workload")
    ap.add_argument("--scenes", type=int, default=16, help="resident scenes of the serve workload")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve workload arrivals per second")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="serve workload trace length")
    ap.add_argument("--traversal", choices=("packet", "lane", "packet_cube"), default=None,
                    help="collect-pass traversal (library default when omitted)")
    ap.add_argument("--leaf-size", type=int, default=None, help="LBVH leaf bucket size (library default when omitted)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    N_PROBE, N_BUILD = args.probes, args.build
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "summary":
        return run_summary(args)
    if args.workload != "frn":
        return run_secondary(args)

    import torch

    import rtdl_b200 as rt
    from rtdl_b200 import _native, workloads

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    rt.set_device(local)
    if args.traversal is not None or args.leaf_size is not None:
        rt.set_tuning(leaf_size=args.leaf_size or 0, traversal=args.traversal or "packet")
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])

    def allreduce(v: float, op) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    # workload: shared build set, per-rank probe set (rank 0 gets the benchmark's own probes)
    c = np.random.default_rng(0).random((64, 3))
    build = workloads.records(workloads._mixture(np.random.default_rng(1), N_BUILD, c))
    probe = workloads.records(workloads._mixture(np.random.default_rng(2 + 1000 * rank), N_PROBE, c))
    dev = torch.device("cuda", local)
    d_build = torch.from_numpy(build.view(np.uint8)).to(dev)
    d_probe = torch.from_numpy(probe.view(np.uint8)).to(dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    overflow = torch.empty(N_PROBE, dtype=torch.uint8, device=dev)

    def one_step(rows_buf, capacity):
        # the plain per-call form on resident records: scene build + query in one call
        n = rt.runtime.fixed_radius_neighbors_device(
            d_probe.data_ptr(), N_PROBE, d_build.data_ptr(), N_BUILD, dimension=3, radius=RADIUS, k_max=K_MAX,
            rows_address=rows_buf.data_ptr() if rows_buf is not None else None, rows_capacity=capacity,
            overflow_address=overflow.data_ptr(), stream=sh)
        return n, _native.last_phase_timings()

    rows_total, _ = one_step(None, 0)
    rows_buf = torch.empty(rows_total * 16, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        one_step(rows_buf, rows_total)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    launches0 = _native.launch_count()
    barrier()
    torch.cuda.synchronize()
    step_ms, phase_log = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
        n, phases = one_step(rows_buf, rows_total)
        with torch.cuda.stream(stream):
            end.record(stream)
        end.synchronize()
        step_ms.append(start.elapsed_time(end))
        phase_log.append(phases)
        assert n == rows_total
    torch.cuda.synchronize()
    barrier()
    launches = _native.launch_count() - launches0
    clocks = sampler.stop()
    local_ms = sum(step_ms)
    job_ms = allreduce(local_ms, dist.ReduceOp.MAX if dist else None)
    all_rows = allreduce(float(rows_total), dist.ReduceOp.SUM if dist else None)
    value = all_rows * args.steps / (job_ms / 1e3)
    ms_per_step = job_ms / args.steps

    # phase (kernel) durations from the library's CUDA events on the launching stream
    def mean_phase(name):
        vals = [p.get(name, 0.0) for p in phase_log]
        return sum(vals) / len(vals)

    traverse_ms, emit_ms, prep_ms, scan_ms = (mean_phase("traverse"), mean_phase("emit"), mean_phase("query_prep"),
                                              mean_phase("scan"))
    # "build" spans the scene build and, on a second stream beside it, the probe set's preparation
    build_ms = mean_phase("build")
    query_ms = mean_phase("total") - build_ms
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        hbm_peak, peak_note = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        hbm_peak, peak_note = 6650.0, "fallback"
    R = rows_total
    # algorithmic bytes (per launch) of the two query phases: the collect kernel reads every probe and build
    # point once and keeps a 4-byte neighbour index per row plus a count and a flag per probe; the emit
    # kernels read those indices back and write 16-byte rows plus per-probe offset/count/flags/point.
    traverse_bytes = N_PROBE * 16 + N_BUILD * 16 + R * 4 + N_PROBE * 5
    emit_bytes = R * 4 + R * 16 + N_PROBE * (4 + 1 + 1 + 8 + 32)
    if traverse_ms >= emit_ms:
        dom, dom_kernel, dom_ms, dom_bytes = ("k_collect_packet (packet LBVH walk, FP32 test + FP64 band)",
                                              "k_collect_packet", traverse_ms, traverse_bytes)
    else:
        dom, dom_kernel, dom_ms, dom_bytes = ("k_emit + k_emit_list (exact FP64 sort and row emission)",
                                              "k_emit", emit_ms, emit_bytes)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = measured_traffic(dom_kernel, "clustered_3d_fixed_radius", N_PROBE, N_BUILD)
    phase_bytes = N_PROBE * 16 + N_BUILD * 16 + R * 16 + N_PROBE * 4 + N_PROBE // 8
    phase_achieved = phase_bytes / (query_ms / 1e3) / 1e9

    # e2e through the C ABI with pinned host buffers
    e2e = None
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else min(args.steps, 5)
    if e2e_steps > 0:
        import ctypes

        h_build = torch.from_numpy(build.view(np.uint8)).pin_memory()
        h_probe = torch.from_numpy(probe.view(np.uint8)).pin_memory()
        lib = _native.load_library()

        def e2e_call():
            rows = ctypes.c_void_p()
            count = ctypes.c_size_t()
            err = _native.error_buffer()
            st = lib.rtdl_b200_run_fixed_radius_neighbors_3d(h_probe.data_ptr(), N_PROBE, h_build.data_ptr(), N_BUILD,
                                                             RADIUS, K_MAX, ctypes.byref(rows), ctypes.byref(count), err,
                                                             len(err))
            _native.check_status(st, err)
            lib.rtdl_b200_free_rows(rows)
            return count.value

        for _ in range(2):
            e2e_call()
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            assert e2e_call() == rows_total
        t_local = time.perf_counter() - t0
        barrier()
        t_job = allreduce(t_local, dist.ReduceOp.MAX if dist else None)
        e2e = {"value": all_rows * e2e_steps / t_job, "unit": UNIT, "h2d_bytes_per_step": (N_BUILD + N_PROBE) * 32,
               "d2h_bytes_per_step": rows_total * 16, "ms_per_step": t_job / e2e_steps * 1e3,
               "entry_point": "rtdl_b200_run_fixed_radius_neighbors_3d (pinned host buffers)"}

    cpu = None
    external = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(probe, build, os.cpu_count() or 1)
        external = external_scipy_baseline(probe, build, os.cpu_count() or 1)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 traversal + f64 band recheck and distances",
            "data": "synthetic",
            "config": {"workload": "clustered_3d_fixed_radius (plain per-call launch: LBVH build + query + exact rows)",
                       "build": N_BUILD, "probe_per_gpu": N_PROBE, "radius": RADIUS, "k_max": K_MAX,
                       "rows_per_gpu": rows_total, "row_bytes": 16, "l2": "flushed between steps (512 MiB write)",
                       "parallelism": f"query-sharded replicas x{world}"},
            "phases_ms": {"build": build_ms, "query_prep": prep_ms, "traverse": traverse_ms, "scan": scan_ms,
                          "emit": emit_ms, "query_total": query_ms},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_note,
                         "algorithmic_bytes": dom_bytes,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one capture of this "
                                           "launch (profiles/dram_traffic.json)" if traffic else None},
            "phase_roofline": {"phase": "query+emit", "achieved": phase_achieved, "peak": hbm_peak, "unit": "GB/s",
                               "frac": phase_achieved / hbm_peak, "algorithmic_bytes": phase_bytes},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "external_baselines": {"scipy_ckdtree": external} if external else None,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
