"""Seeded synthetic workloads with the shapes of the neighbor-path benchmarks.

No public dataset is needed: each generator reproduces the distribution named
by the benchmark configuration it stands for.

* ``uniform_2d``: 4,096 x 4,096 float64 points uniform in [0,1]^2, seed 0
  (build drawn first, then probe from the same generator), radius 0.02.
* ``clustered_3d``: 1,048,576 build and 1,048,576 probe points; 64 centres
  uniform in the unit cube (seed 0); 90% of points N(centre, 0.01^2 I), 10%
  uniform; clamped to [0,1]; float32 values (build seed 1, probe seed 2).
  The radius 0.00287 gives a mean of ~32 in-radius neighbors per probe.
* ``hausdorff_2d``: A uniform in [0,1]^2 (4,194,304 float32 points, seed 3);
  B = A + N(0, 1e-3) jitter with 1% of B displaced uniformly (seed 4).
* ``batched_problems``: independent 3D fixed-radius problems with build and
  probe counts log-uniform in [1,024, 262,144] (seed 5), points uniform in
  boxes of random aspect ratio, per-problem radius for a mean of 8-64
  neighbors.
"""
from __future__ import annotations

import numpy as np

CLUSTERED_RADIUS = 0.00287


def records(points: np.ndarray, ids: np.ndarray | None = None) -> np.ndarray:
    """(n, 2|3) float array -> RtdlPoint / RtdlPoint3D structured records."""
    from .runtime import POINT2D_DTYPE, POINT3D_DTYPE

    n, dim = points.shape
    out = np.zeros(n, dtype=POINT3D_DTYPE if dim == 3 else POINT2D_DTYPE)
    out["id"] = np.arange(n, dtype=np.uint32) if ids is None else ids
    out["x"] = points[:, 0]
    out["y"] = points[:, 1]
    if dim == 3:
        out["z"] = points[:, 2]
    return out


def uniform_2d(n: int = 4096, seed: int = 0):
    rng = np.random.default_rng(seed)
    build = rng.random((n, 2))
    probe = rng.random((n, 2))
    return records(probe), records(build)


def _mixture(rng, n, centres, sigma=0.01, background=0.1):
    which = rng.integers(0, len(centres), n)
    pts = centres[which] + rng.normal(0.0, sigma, (n, 3))
    bg = rng.random(n) < background
    pts[bg] = rng.random((int(bg.sum()), 3))
    return np.clip(pts, 0.0, 1.0).astype(np.float32).astype(np.float64)


def clustered_3d(n_build: int = 1 << 20, n_probe: int = 1 << 20, centres: int = 64):
    c = np.random.default_rng(0).random((centres, 3))
    build = _mixture(np.random.default_rng(1), n_build, c)
    probe = _mixture(np.random.default_rng(2), n_probe, c)
    return records(probe), records(build)


def hausdorff_2d(n: int = 1 << 22):
    a = np.random.default_rng(3).random((n, 2)).astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(4)
    b = a + rng.normal(0.0, 1e-3, (n, 2))
    moved = rng.random(n) < 0.01
    b[moved] = rng.random((int(moved.sum()), 2))
    b = b.astype(np.float32).astype(np.float64)
    return records(a), records(b)


def batched_problems(count: int = 2048, seed: int = 5, lo: int = 1024, hi: int = 262144):
    """Returns a list of (probe_records, build_records, radius, k_max)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nb = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        nq = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        scale = np.exp(rng.uniform(-1.0, 1.0, 3))
        build = (rng.random((nb, 3)) * scale).astype(np.float32).astype(np.float64)
        probe = (rng.random((nq, 3)) * scale).astype(np.float32).astype(np.float64)
        mean = rng.uniform(8.0, 64.0)
        volume = float(np.prod(scale))
        radius = (mean * volume / (nb * 4.0 / 3.0 * np.pi)) ** (1.0 / 3.0)
        out.append((records(probe), records(build), float(radius), 64))
    return out


def rtnn_points(distribution: str, n: int = 262_144, seed: int | None = None) -> np.ndarray:
    """The reference's RTNN-style 3D point sets, regenerated point for point.

    Restates the generator of the reference's published ranked-summary runs
    (``scripts/goal2348_rtnn_v2_2_external_runner.py:19-103``): Python's
    ``random.Random(seed)``; ``uniform``: x, y, z = three ``random()`` draws;
    ``clustered``: 8 centres drawn first (each axis ``uniform(0.12, 0.88)``),
    point i takes centre i mod 8 and each axis ``gauss(centre, 0.035)`` clamped
    to [0, 1]; ``shell``: the same 8 centre draws, then per point an angle
    ``random() * 2 pi``, ``z = uniform(-1, 1)`` and a shell radius
    ``gauss(0.34, 0.025)`` clamped to [0, 0.49] around (0.5, 0.5, 0.5).  Every
    coordinate passes through the 9-decimal text form the reference writes
    (``"%.9f"``) and reads back.  Ids are the point indices.  Default seeds are
    those of the published runs: 2800, 2801, 2802.
    """
    import math
    import random

    seeds = {"uniform": 2800, "clustered": 2801, "shell": 2802}
    if distribution not in seeds:
        raise ValueError("distribution must be uniform, clustered or shell")
    rng = random.Random(seeds[distribution] if seed is None else seed)
    xyz = np.empty((n, 3), dtype=np.float64)
    if distribution == "uniform":
        for i in range(n):
            xyz[i, 0] = rng.random()
            xyz[i, 1] = rng.random()
            xyz[i, 2] = rng.random()
    else:
        centres = [tuple(rng.uniform(0.12, 0.88) for _ in range(3)) for _ in range(8)]
        for i in range(n):
            if distribution == "clustered":
                c = centres[i % 8]
                for a in range(3):
                    xyz[i, a] = min(1.0, max(0.0, rng.gauss(c[a], 0.035)))
            else:
                theta = rng.random() * 6.283185307179586
                z = rng.uniform(-1.0, 1.0)
                radial = math.sqrt(max(0.0, 1.0 - z * z))
                r = min(0.49, max(0.0, rng.gauss(0.34, 0.025)))
                xyz[i, 0] = 0.5 + r * radial * math.cos(theta)
                xyz[i, 1] = 0.5 + r * radial * math.sin(theta)
                xyz[i, 2] = 0.5 + r * z
    xyz = np.array([float(f"{v:.9f}") for v in xyz.ravel()], dtype=np.float64).reshape(n, 3)
    return records(xyz)
