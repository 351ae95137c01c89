"""The oracle's uniform-grid candidate generator gives the brute-force rows bit for bit.

The full-size fixtures (tests/golden/full_scale_digests.json) are computed with
the grid; these cases pin it to the brute-force restatement, which the
reference's own rows pin in test_oracle_golden.py: clustered 3D sets, an
integer lattice whose spacing puts many points exactly on the radius and at
equal distances (ties broken by id, then input order), duplicates, queries
outside the search set's box, and 2D sets.
"""
import numpy as np
import pytest

from oracle import oracle as O
from rtdl_b200 import workloads


def _same(a, b):
    if len(a) != len(b) or a.dtype.names != b.dtype.names:
        return False
    for n in a.dtype.names:
        x, y = a[n], b[n]
        if x.dtype == np.float64:
            x, y = x.view(np.uint64), y.view(np.uint64)
        if not np.array_equal(x, y):
            return False
    return True


def _lattice(dim, n, step, dup=2):
    axes = np.meshgrid(*[np.arange(n)] * dim, indexing="ij")
    g = np.stack(axes, -1).reshape(-1, dim).astype(np.float64) * step
    return workloads.records(np.repeat(g, dup, axis=0))


@pytest.mark.parametrize("radius,k_max", [(0.005, 3), (0.01, 8), (0.02, 64), (0.0, 4)])
def test_grid_fixed_radius_equals_brute_force_clustered(radius, k_max):
    probe, build = workloads.clustered_3d(20_000, 4_000)
    for ranked in (False, True):
        a, ca = O.fixed_radius_neighbors(probe, build, radius=radius, k_max=k_max, threads=4, ranked=ranked,
                                         with_counts=True)
        b, cb = O.fixed_radius_neighbors(probe, build, radius=radius, k_max=k_max, threads=4, ranked=ranked,
                                         with_counts=True, grid=True)
        assert _same(a, b) and np.array_equal(ca, cb)


@pytest.mark.parametrize("k", [1, 8, 33])
def test_grid_knn_equals_brute_force_clustered(k):
    probe, build = workloads.clustered_3d(20_000, 3_000)
    assert _same(O.knn_rows(probe, build, k=k, threads=4), O.knn_rows(probe, build, k=k, threads=4, grid=True))


@pytest.mark.parametrize("dim", [2, 3])
def test_grid_on_lattice_ties_and_duplicates(dim):
    search = _lattice(dim, 12 if dim == 3 else 30, 0.25)
    rng = np.random.default_rng(7)
    q = np.asarray(search[["x", "y"] + (["z"] if dim == 3 else [])].tolist())[::5][:400]
    q = q + np.where(rng.random(q.shape) < 0.5, 0.0, 0.125)  # on lattice points and at cell centres
    query = workloads.records(q)
    for radius, k_max in ((0.25, 4), (0.5, 9), (np.sqrt(2) * 0.25, 6)):
        a = O.fixed_radius_neighbors(query, search, radius=radius, k_max=k_max, threads=4)
        b = O.fixed_radius_neighbors(query, search, radius=radius, k_max=k_max, threads=4, grid=True)
        assert len(a) > 0 and _same(a, b)
    for k in (1, 5, 17):
        assert _same(O.knn_rows(query, search, k=k, threads=4), O.knn_rows(query, search, k=k, threads=4, grid=True))


def test_grid_nearest_and_queries_outside_the_box():
    probe, build = workloads.clustered_3d(10_000, 2_000)
    outside = workloads.records(np.random.default_rng(3).random((500, 3)) * 3.0 - 1.0)
    for q in (probe, outside):
        d0, i0 = O.nearest(q, build, threads=4)
        d1, i1 = O.nearest(q, build, threads=4, grid=True)
        assert np.array_equal(d0.view(np.uint64), d1.view(np.uint64)) and np.array_equal(i0, i1)
        assert _same(O.knn_rows(q, build, k=4, threads=4), O.knn_rows(q, build, k=4, threads=4, grid=True))


def test_grid_hausdorff_sets_2d():
    a, b = workloads.hausdorff_2d(20_000)
    d0, i0 = O.nearest(a, b, threads=4)
    d1, i1 = O.nearest(a, b, threads=4, grid=True)
    assert np.array_equal(d0.view(np.uint64), d1.view(np.uint64)) and np.array_equal(i0, i1)
