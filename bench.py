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

def _hbm_peak():
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def full_scale_digests() -> dict:
    """Digests of the complete row sets computed by the oracle (tests/golden/full_scale_digests.json)."""
    try:
        return json.loads((ROOT / "tests" / "golden" / "full_scale_digests.json").read_text())
    except (OSError, ValueError):
        return {}


def _sha(a) -> str:
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def _bits_equal(a, b) -> bool:
    return bool(np.array_equal(np.asarray(a, dtype=np.float64).view(np.uint64),
                               np.asarray(b, dtype=np.float64).view(np.uint64)))


def frn_exactness(rows: np.ndarray, probe, build, sample_n: int = 512) -> dict:
    """The headline's rows against the oracle: every row of a seeded sample of queries (ids and FP64
    distance bits, oracle over the full build set) and the complete row set against the oracle's
    digest of it.  Probe ids are their input indices, so rows come in probe order."""
    from oracle import oracle as O

    rng = np.random.default_rng(99)
    sample = np.sort(rng.choice(len(probe), sample_n, replace=False))
    exp = O.fixed_radius_neighbors(probe[sample], build, radius=RADIUS, k_max=K_MAX, threads=os.cpu_count() or 1)
    starts = np.searchsorted(rows["query_id"], sample, side="left")
    ends = np.searchsorted(rows["query_id"], sample, side="right")
    got = np.concatenate([rows[a:b] for a, b in zip(starts, ends)]) if len(sample) else rows[:0]
    same = (len(got) == len(exp) and np.array_equal(got["query_id"], exp["query_id"])
            and np.array_equal(got["neighbor_id"], exp["neighbor_id"]) and _bits_equal(got["distance"], exp["distance"]))
    err = float(np.max(np.abs(got["distance"] - exp["distance"]))) if same and len(exp) else (0.0 if same else None)
    out = {"sample_queries": int(sample_n), "sample_rows": int(len(exp)), "sample_rows_equal_to_oracle": bool(same),
           "max_abs_distance_error_vs_fp64_oracle": err}
    ref = full_scale_digests().get("frn_1m")
    if ref and len(probe) == N_PROBE == 1 << 20 and len(build) == N_BUILD == 1 << 20:
        out["full_set_rows"] = int(len(rows))
        out["full_set_rows_sha256_equal_to_oracle"] = _sha(rows) == ref["rows_sha256"]
    return out


def secondary_leg(workload: str, steps: int, warmup: int, k: int = 16) -> dict:
    """knn (k=16 unless given) at 1M x 1M 3D, or directed Hausdorff at 4M x 4M 2D: CUDA-event ms per step
    (scene build + query), rows/s, the query kernel's roofline fraction and exactness against the oracle (a
    sample of queries, plus the complete output against the oracle's digest)."""
    import torch

    import rtdl_b200 as rt
    from oracle import oracle as O
    from rtdl_b200 import _native, workloads

    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    knn = workload == "knn"
    if knn:
        probe, build = workloads.clustered_3d(N_BUILD, N_PROBE)  # --build / --probes for a smaller case
        units = len(probe) * k
    else:
        probe, build = workloads.hausdorff_2d()
        units = len(probe)
    dim = 3 if knn else 2
    d_build = torch.from_numpy(build.view(np.uint8)).to(dev)
    d_probe = torch.from_numpy(probe.view(np.uint8)).to(dev)
    rows_buf = torch.empty(units * 24, dtype=torch.uint8, device=dev) if knn else None
    nd = torch.empty(len(probe), dtype=torch.float64, device=dev)
    ni = torch.empty(len(probe), dtype=torch.int32, device=dev)
    result = {}

    def step():
        scene = rt.B200Scene(None, dimension=dim, stream=sh, device_points=(d_build.data_ptr(), len(build)))
        try:
            if knn:
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

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    launches0 = _native.launch_count()
    ms, phases = [], []
    for _ in range(steps):
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
    ms_step = sum(ms) / len(ms)
    trav = sum(p.get("traverse", 0.0) for p in phases) / len(phases)
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(99)
    sample = np.sort(rng.choice(len(probe), 256, replace=False))
    digests = full_scale_digests()
    if knn:
        rows = np.frombuffer(rows_buf.cpu().numpy().tobytes(), dtype=rt.runtime.KNN_ROW_DTYPE)
        got = rows.reshape(-1, k)[sample]
        exp = O.knn_rows(probe[sample], build, k=k, threads=threads).reshape(-1, k)
        ids_equal = bool(np.array_equal(got["neighbor_id"], exp["neighbor_id"])
                         and np.array_equal(got["neighbor_rank"], exp["neighbor_rank"]))
        dist_equal = _bits_equal(got["distance"], exp["distance"])
        max_err = float(np.max(np.abs(got["distance"] - exp["distance"])))
        alg_bytes = len(probe) * 16 + len(build) * 16 + units * 24
        kernel = "k_pass1<KNN> (nearest-list LBVH walk)"
        full = {}
        ref = digests.get("knn16_1m")
        if ref and k == 16 and len(probe) == len(build) == 1 << 20:
            packed = np.zeros(len(rows), dtype=np.dtype({"names": ["query_id", "neighbor_id", "distance", "neighbor_rank"],
                                                         "formats": ["<u4", "<u4", "<f8", "<u4"],
                                                         "offsets": [0, 4, 8, 16], "itemsize": 20}))
            for n in packed.dtype.names:
                packed[n] = rows[n]
            full = {"full_set_rows": int(len(rows)),
                    "full_set_rows_sha256_equal_to_oracle": _sha(packed) == ref["rows_packed_sha256"]}
        extra = {"k": k, "rows": units}
    else:
        dist, nid = O.nearest(probe[sample], build, threads=threads)
        got_d = nd.cpu().numpy()
        got_i = ni.cpu().numpy().view(np.uint32)
        ids_equal = bool(np.array_equal(got_i[sample], nid))
        dist_equal = _bits_equal(got_d[sample], dist)
        max_err = float(np.max(np.abs(got_d[sample] - dist)))
        alg_bytes = len(probe) * 16 + len(build) * 16 + len(probe) * 12
        kernel = "k_pass1<KNN> with k = 1 (nearest LBVH walk)"
        full = {}
        ref = digests.get("hausdorff_4m")
        if ref:
            w = ref["witness"]
            full = {"full_set_nearest_sha256_equal_to_oracle": _sha(got_d) == ref["nearest_distance_sha256"]
                    and _sha(got_i) == ref["nearest_id_sha256"],
                    "witness_equal_to_oracle": (float.fromhex(w["distance_hex"]) == result.get("distance")
                                                and w["source_id"] == result.get("source_id")
                                                and w["target_id"] == result.get("target_id"))}
        extra = {"hausdorff": result, "queries": len(probe)}
    hbm_peak, peak_note = _hbm_peak()
    achieved = alg_bytes / (trav / 1e3) / 1e9 if trav > 0 else None
    return {
        "metric": (f"knn rows/s at 1M x 1M 3D, k={k} (exact row set)" if knn
                   else "directed Hausdorff nearest rows/s at 4M x 4M 2D (FP64 max-min)"),
        "value": units / (ms_step / 1e3), "unit": "rows/s", "ms_per_step": ms_step, "steps": steps, "warmup": warmup,
        "config": {"workload": workload, "build": len(build), "probe": len(probe),
                   "l2": "flushed between steps (512 MiB write)", **extra},
        "phases_ms": {k2: sum(p.get(k2, 0.0) for p in phases) / len(phases)
                      for k2 in ("build", "query_prep", "traverse", "scan", "emit", "reduce")},
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None, "traffic": None,
                     "peak_source": peak_note, "algorithmic_bytes": alg_bytes},
        "exactness": {"sample_queries": int(len(sample)), "ids_equal_to_oracle": ids_equal,
                      "distance_bits_equal_to_oracle": dist_equal,
                      "max_abs_distance_error_vs_fp64_oracle": max_err, **full},
        "gpu_launches": launches,
    }


def run_config1(args) -> int:
    """The reference's CPU-runnable case: 4,096 x 4,096 2D fixed radius (float64 uniform, seed 0, radius
    0.02, no k_max truncation), rows checked against the reference's own rows (tests/golden), GPU
    rows/s through the plain C ABI call beside the CPU runners timed here on one core each."""
    import ctypes

    import torch

    import rtdl_b200 as rt
    from oracle import oracle as O
    from oracle import reference_py
    from rtdl_b200 import _native
    from rtdl_b200.runtime import FRN_ROW_DTYPE, POINT2D_DTYPE

    torch.cuda.set_device(0)
    rt.set_device(0)
    rng = np.random.default_rng(0)
    b, p = rng.random((4096, 2)), rng.random((4096, 2))
    build = np.zeros(4096, dtype=POINT2D_DTYPE)
    probe = np.zeros(4096, dtype=POINT2D_DTYPE)
    for arr, pts in ((build, b), (probe, p)):
        arr["id"] = np.arange(4096, dtype=np.uint32)
        arr["x"], arr["y"] = pts[:, 0], pts[:, 1]
    radius, k_max = 0.02, 4096
    lib = _native.load_library()

    def call():
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        st = lib.rtdl_b200_run_fixed_radius_neighbors(probe.ctypes.data, 4096, build.ctypes.data, 4096, radius,
                                                      k_max, ctypes.byref(rows), ctypes.byref(count), err, len(err))
        _native.check_status(st, err)
        n = count.value
        out = np.frombuffer((ctypes.c_char * (n * 16)).from_address(rows.value), dtype=FRN_ROW_DTYPE).copy()
        lib.rtdl_b200_free_rows(rows)
        return out

    for _ in range(args.warmup):
        call()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    launches0 = _native.launch_count()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rows = call()
    dt = (time.perf_counter() - t0) / args.steps
    launches = _native.launch_count() - launches0
    clocks = sampler.stop()
    golden = ROOT / "tests" / "golden" / "config1_frn_2d.npz"
    exact = None
    if golden.exists():
        z = np.load(golden)
        exact = bool(len(rows) == len(z["query_id"]) and np.array_equal(rows["query_id"], z["query_id"])
                     and np.array_equal(rows["neighbor_id"], z["neighbor_id"])
                     and _bits_equal(rows["distance"], z["distance"]))
    # CPU runners on the same input, one core each
    t = time.perf_counter()
    py_rows = reference_py.fixed_radius_neighbors(reference_py.points(probe), reference_py.points(build),
                                                  radius=radius, k_max=k_max)
    t_py = time.perf_counter() - t
    t = time.perf_counter()
    c_rows = O.fixed_radius_neighbors(probe, build, radius=radius, k_max=k_max, threads=1)
    t_c = time.perf_counter() - t
    ref = None
    if O.reference_library_available():
        pq, pb = O.pack_reference_points(probe), O.pack_reference_points(build)
        t = time.perf_counter()
        ref_rows = O.reference_fixed_radius_neighbors(pq, pb, radius=radius, k_max=k_max)
        t_ref = time.perf_counter() - t
        ref = {"value": len(ref_rows) / t_ref, "unit": "rows/s", "cores": 1, "kind": "reference",
               "sample": f"full set, {len(ref_rows)} rows in {t_ref:.3f} s (the reference's native oracle, "
                         "compiled from its sources)"}
    line = {
        "metric": "fixed-radius neighbor rows/s at 4,096 x 4,096 2D (float64, radius 0.02; exact row set)",
        "value": len(rows) / dt, "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 inputs: f32 traversal + f64 band recheck and distances", "data": "synthetic",
        "config": {"workload": "config1_frn_2d (rng(0) uniform, 4,096 build then 4,096 probe points)",
                   "radius": radius, "k_max": k_max, "rows": int(len(rows)),
                   "timing": "host wall clock around rtdl_b200_run_fixed_radius_neighbors (host records in, "
                             "rows in host memory out)", "l2": "input far below L2 (latency-bound case)"},
        "exactness": {"rows_equal_to_reference_rows": exact, "reference_rows": "tests/golden/config1_frn_2d.npz "
                      "(the reference's cpu_python_reference)"},
        "cpu_baseline": {"value": len(py_rows) / t_py, "unit": "rows/s", "cores": 1, "kind": "port",
                         "sample": f"full set, {len(py_rows)} rows in {t_py:.2f} s (oracle/reference_py.py: the "
                                   "reference's cpu_python_reference algorithm in plain Python)"},
        "cpu_baselines": {"reference_native_oracle": ref,
                          "c_port": {"value": len(c_rows) / t_c, "unit": "rows/s", "cores": 1, "kind": "port",
                                     "sample": f"full set, {len(c_rows)} rows in {t_c:.3f} s (oracle/nn_oracle.c)"}},
        "e2e": {"value": len(rows) / dt, "unit": "rows/s", "h2d_bytes_per_step": 2 * 4096 * 24,
                "d2h_bytes_per_step": int(len(rows)) * 16},
        "clocks": clocks, "gpu_launches": launches,
    }
    print(json.dumps(line))
    return 0


def run_secondary(args) -> int:
    import torch

    import rtdl_b200 as rt

    torch.cuda.set_device(0)
    rt.set_device(0)
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    leg = secondary_leg(args.workload, args.steps, args.warmup, k=args.k)
    clocks = sampler.stop()
    line = {"metric": leg.pop("metric"), "value": leg.pop("value"), "unit": leg.pop("unit"), "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": leg.pop("ms_per_step"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 traversal + f64 band recheck and distances", "data": "synthetic", **leg, "clocks": clocks}
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


def batch_workload(args) -> dict:
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
    from dataclasses import asdict

    from rtdl_b200.autotune import Autotuner

    def one_batch(ci, rows_buf, cap):
        a, b = chunks[ci]
        ba, qa = int(boff[a]), int(qoff[a])
        with B200ProblemBatch(None, dimension=3, stream=sh,
                              device_points=(d_build.data_ptr() + 32 * ba, boff[a:b + 1] - boff[a])) as batch:
            return batch.fixed_radius_neighbors_device(
                d_probe.data_ptr() + 32 * qa, qoff[a:b + 1] - qoff[a], radius=radius[a:b], k_max=kmax[a:b],
                rows_address=rows_buf.data_ptr() if rows_buf is not None else None, rows_capacity=cap, stream=sh)

    def batch_step(rows_buf, cap, sizes_out=None):
        total = 0
        for ci in range(len(chunks)):
            offs = one_batch(ci, rows_buf, cap)
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
    # autotune (leaf size, block size; batches always walk in warp packets) on one whole batch, the largest
    big = int(np.argmax([int(o[-1]) for o in chunk_sizes]))
    tuner = Autotuner(repeats=2, traversals=("packet_hybrid", "packet"))

    tune_key, tune_cfg = tuner.tune_callable(f"problem batch {big} of {len(chunks)}",
                                             lambda: one_batch(big, rows_buf, max_chunk_rows), stream=stream)
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
    if not args.no_graph:
        del plain_buf, rows_buf
        torch.cuda.empty_cache()
        line["graph"] = batch_graph_leg(args, nb, nq, boff, qoff, radius, kmax, d_build, d_probe, stream, flush,
                                        rows_total, sample, alg, hbm_peak)
        g = line["graph"]
        line["speedup_graph_vs_plain"] = plain_ms[0] / g["ms_per_step"]
    return line


def run_batch(args) -> int:
    print(json.dumps(batch_workload(args)))
    return 0


def batch_graph_leg(args, nb, nq, boff, qoff, radius, kmax, d_build, d_probe, stream, flush, rows_total, sample,
                    alg, hbm_peak) -> dict:
    """All problems answered by one replay of the captured graph over prepared problem batches (one persistent
    collect launch per batch, nothing read back inside), rows of every problem into one device buffer."""
    import torch

    import rtdl_b200 as rt
    from rtdl_b200 import _native
    from rtdl_b200.batch import B200ProblemBatch, B200ProblemBatchGraph

    sh = stream.cuda_stream
    chunks = _plan_chunks(nb, nq, (1 << 26) - 1, args.graph_batch_probes)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batches = [B200ProblemBatch(None, dimension=3, stream=sh,
                                device_points=(d_build.data_ptr() + 32 * int(boff[a]), boff[a:b + 1] - boff[a]))
               for a, b in chunks]
    d_rows = torch.empty(rows_total * 16, dtype=torch.uint8, device=d_build.device)
    graph = B200ProblemBatchGraph(batches, d_probe.data_ptr(), qoff, radius=radius, k_max=kmax,
                                  rows_address=d_rows.data_ptr(), rows_capacity=rows_total)
    torch.cuda.synchronize()
    prepare_s = time.perf_counter() - t0
    try:
        off, status = graph.replay()
        assert int(off[-1]) == rows_total and status == 0, (int(off[-1]), rows_total, status)
        for _ in range(args.warmup):
            graph.launch(sh)
        torch.cuda.synchronize()
        launches0 = _native.launch_count()
        ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            graph.launch(sh)
            with torch.cuda.stream(stream):
                b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        launches = _native.launch_count() - launches0
        # sampled problems: graph rows against one plain call per problem
        equal = True
        for i in sample:
            lo, hi = int(off[i]), int(off[i + 1])
            got = np.frombuffer(d_rows[lo * 16: hi * 16].cpu().numpy().tobytes(), dtype=rt.runtime.FRN_ROW_DTYPE)
            probe_i = np.frombuffer(d_probe[32 * int(qoff[i]): 32 * int(qoff[i + 1])].cpu().numpy().tobytes(),
                                    dtype=rt.runtime.POINT3D_DTYPE)
            build_i = np.frombuffer(d_build[32 * int(boff[i]): 32 * int(boff[i + 1])].cpu().numpy().tobytes(),
                                    dtype=rt.runtime.POINT3D_DTYPE)
            view = rt.runtime.fixed_radius_neighbors(probe_i, build_i, radius=float(radius[i]), k_max=int(kmax[i]))
            ref = view.to_numpy()
            view.close()
            equal &= bool(len(ref) == len(got) and np.array_equal(ref.view(np.uint8), got.view(np.uint8)))
        info = graph.info()
    finally:
        graph.close()
        for b in batches:
            b.close()
    ms_step = sum(ms) / len(ms)
    return {"value": rows_total / (ms_step / 1e3), "unit": "rows/s", "ms_per_step": ms_step,
            "step": "one replay of the captured graph over prepared problem batches (queries of all problems)",
            "batches": len(chunks), "persistent_collect_launches": len(chunks), "kernel_nodes": info["kernel_nodes"],
            "prepare_s": prepare_s, "fallback_batches": info["fallbacks"], "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": alg / (ms_step / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                         "frac": alg / (ms_step / 1e3) / 1e9 / hbm_peak, "algorithmic_bytes": alg},
            "exactness": {"problems_checked": len(sample), "rows_equal_to_plain_call": equal}}


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


def serve_workload(args) -> dict:
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
    scene_sizes = {k: len(v) for k, v in points.items()}
    trace = serve_trace(args.serve_seconds, args.rate, scene_sizes, pools)

    def measure(server, trace, sampler=None):
        """Replays a trace through the served loop and the plain path; sampled requests checked."""
        server.completed.clear()
        sample = set(np.random.default_rng(3).choice(len(trace), min(24, len(trace)), replace=False).tolist())
        launches0 = _native.launch_count()
        reqs = replay(server, trace, keep=sample)  # rows of the sampled requests are kept for the check
        launches = _native.launch_count() - launches0
        clocks = sampler.stop() if sampler else None
        served = server.stats()
        failed = [r.error for r in reqs if r.error]
        equal = True
        for i in sorted(sample):  # exactness: the sampled requests against the plain call alone
            r = reqs[i]
            view = server.scenes[r.scene].query(r.queries, predicate=r.op, radius=r.radius, limit=r.limit)
            equal &= same_rows(r.rows, view.to_numpy())
            view.close()
        plain = run_plain(server.scenes, reqs, [t[0] for t in trace])
        return served, plain, {"requests_checked": len(sample), "rows_equal_to_plain_call": equal,
                               "failed": len(failed)}, launches, clocks

    with B200Server(memory_budget=120 << 30, streams=4) as server:
        for name, p in points.items():
            server.add_scene(name, p)
        replay(server, trace[: min(len(trace), 32)], keep=set())  # warm-up: allocator pools, pinned buffers
        sampler = ClockSampler(0)
        sampler.start()
        served, plain, exact, launches, clocks = measure(server, trace, sampler)
        sustained = None
        if args.sustained_rate > 0:  # a rate the loop keeps up with: latencies are service times, not queueing
            strace = serve_trace(args.serve_seconds, args.sustained_rate, scene_sizes, pools, seed=7)
            s_served, s_plain, s_exact, _, _ = measure(server, strace)
            sustained = {"rate_req_per_s": args.sustained_rate, "requests": len(strace), "served": s_served,
                         "plain_per_call": s_plain, "exactness": s_exact,
                         "throughput_vs_plain": (s_served["rows_per_s"] / s_plain["rows_per_s"])
                         if s_served.get("rows_per_s") and s_plain.get("rows_per_s") else None}
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
        "exactness": exact,
        "sustained": sustained,
        "e2e": None, "cpu_baseline": None, "roofline": None, "clocks": clocks, "gpu_launches": launches,
    }
    return line


def run_serve(args) -> int:
    print(json.dumps(serve_workload(args)))
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
    ap.add_argument("--no-secondary", action="store_true",
                    help="leave out the exactness check and the knn16 / hausdorff_4m / batch_2048 / serve legs of "
                         "the headline line")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--probes", type=int, default=N_PROBE, help="probe points per GPU (profiling a smaller case)")
    ap.add_argument("--build", type=int, default=N_BUILD, help="build points (profiling a smaller case)")
    ap.add_argument("--workload", choices=("frn", "knn", "hausdorff", "batch", "serve", "summary", "config1"),
                    default="frn",
                    help="frn: the headline fixed-radius config; knn: k=16 on the same 3D sets; "
                         "hausdorff: 4,194,304 x 4,194,304 2D directed nearest-distance reduction; "
                         "batch: 2,048 uneven fixed-radius problems, batched vs one call per problem; "
                         "serve: request loop over resident scenes vs the plain per-call path; "
                         "summary: the reference's published ranked-summary benchmark; "
                         "config1: 4,096 x 4,096 2D fixed radius beside the reference's CPU runners")
    ap.add_argument("--k", type=int, default=16, help="knn workload: neighbours per query")
    ap.add_argument("--problems", type=int, default=2048, help="problems of the batch workload")
    ap.add_argument("--no-graph", action="store_true", help="batch workload: leave out the captured-graph leg")
    ap.add_argument("--graph-batch-probes", type=int, default=24 << 20,
                    help="batch workload: probes per prepared batch of the captured graph")
    ap.add_argument("--scenes", type=int, default=16, help="resident scenes of the serve workload")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve workload arrivals per second")
    ap.add_argument("--sustained-rate", type=float, default=250.0,
                    help="serve workload: a second trace at a rate the loop keeps up with (0: none)")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="serve workload trace length")
    ap.add_argument("--traversal", choices=("packet", "lane", "packet_cube", "packet_points", "packet_hybrid"),
                    default=None,
                    help="collect-pass traversal (library default when omitted)")
    ap.add_argument("--leaf-size", type=int, default=None, help="LBVH leaf bucket size (library default when omitted)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    N_PROBE, N_BUILD = args.probes, args.build
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.traversal is not None or args.leaf_size is not None:
        import rtdl_b200 as rt

        rt.set_tuning(leaf_size=args.leaf_size or 0, traversal=args.traversal or "packet_hybrid")
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "summary":
        return run_summary(args)
    if args.workload == "config1":
        return run_config1(args)
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
    hbm_peak, peak_note = _hbm_peak()
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

        for _ in range(max(3, args.warmup)):
            e2e_call()
        barrier()
        calls_ms = []
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            tc = time.perf_counter()
            assert e2e_call() == rows_total
            calls_ms.append((time.perf_counter() - tc) * 1e3)
        t_local = time.perf_counter() - t0
        barrier()
        t_job = allreduce(t_local, dist.ReduceOp.MAX if dist else None)
        e2e = {"value": all_rows * e2e_steps / t_job, "unit": UNIT, "h2d_bytes_per_step": (N_BUILD + N_PROBE) * 32,
               "d2h_bytes_per_step": rows_total * 16, "ms_per_step": t_job / e2e_steps * 1e3,
               "calls_ms": [round(v, 3) for v in calls_ms],
               "entry_point": "rtdl_b200_run_fixed_radius_neighbors_3d (pinned host buffers)"}

    # exactness of the timed rows against the oracle, then the KNN and Hausdorff legs (one GPU only)
    exactness = knn16 = hausdorff4m = batch2048 = serve = None
    if rank == 0 and world == 1 and not args.no_secondary:
        from rtdl_b200.runtime import FRN_ROW_DTYPE

        rows_np = np.frombuffer(rows_buf.cpu().numpy().tobytes(), dtype=FRN_ROW_DTYPE)
        del rows_buf, flush
        torch.cuda.empty_cache()
        exactness = frn_exactness(rows_np, probe, build)
        del rows_np
        knn16 = secondary_leg("knn", steps=5, warmup=3)
        hausdorff4m = secondary_leg("hausdorff", steps=5, warmup=3)
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = 3, 3
        b = batch_workload(sub)
        rt.set_tuning()  # the batch leg's autotuner leaves its winner set
        batch2048 = {"metric": b["metric"], "value": b["value"], "unit": b["unit"], "ms_per_step": b["ms_per_step"],
                     "step": "one build + query per batch of problems", "config": b["config"],
                     "plain_per_call": b["plain_per_call"], "speedup_vs_plain": b["speedup_vs_plain"],
                     "graph": b.get("graph"), "speedup_graph_vs_plain": b.get("speedup_graph_vs_plain"),
                     "exactness": b["exactness"], "roofline": b["roofline"], "gpu_launches": b["gpu_launches"],
                     "autotune": {"tuned_on": b["autotune"]["shape_class"], "config": b["autotune"]["config"]}}
        v = serve_workload(sub)
        serve = {"metric": v["metric"], "value": v["value"], "unit": v["unit"], "config": v["config"],
                 "served": v["served"], "plain_per_call": v["plain_per_call"],
                 "throughput_vs_plain": v["throughput_vs_plain"], "sustained": v["sustained"],
                 "exactness": v["exactness"], "gpu_launches": v["gpu_launches"]}

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
            "exactness": exactness,
            "knn16": knn16,
            "hausdorff_4m": hausdorff4m,
            "batch_2048": batch2048,
            "serve": serve,
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
