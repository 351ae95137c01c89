"""Host-side pieces of bench.py, without a GPU: the DRAM-traffic record the
headline line's roofline reads, the batch planner, and the full-scale digests."""
import numpy as np

import bench


def test_traffic_record_covers_the_headline_kernels():
    n = 1 << 20
    for kernel in ("k_collect_packet", "k_emit"):
        traffic = bench.measured_traffic(kernel, "clustered_3d_fixed_radius", n, n)
        assert traffic is not None and traffic > 0
    # another size or kernel has no record: the line reports null instead of a guess
    assert bench.measured_traffic("k_collect_packet", "clustered_3d_fixed_radius", n // 4, n) is None
    assert bench.measured_traffic("k_unknown", "clustered_3d_fixed_radius", n, n) is None


def test_batch_plan_keeps_order_and_limits():
    rng = np.random.default_rng(5)
    nb = rng.integers(1, 1000, 300)
    nq = rng.integers(1, 1000, 300)
    chunks = bench._plan_chunks(nb, nq, 20000, 15000)
    assert chunks[0][0] == 0 and chunks[-1][1] == len(nb)
    for (a, b), (c, _) in zip(chunks, chunks[1:]):
        assert b == c  # consecutive, no gaps
    for a, b in chunks:
        assert b > a
        if b - a > 1:  # a single problem may exceed the limits on its own
            assert nb[a:b].sum() <= 20000 and nq[a:b].sum() <= 15000


def test_full_scale_digests_present():
    d = bench.full_scale_digests()
    for key in ("frn_1m", "knn16_1m", "hausdorff_4m"):
        assert key in d
