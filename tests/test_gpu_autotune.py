"""The autotuner: its choice is one of the candidates and is cached per shape
class, and every candidate configuration gives the same rows."""
import numpy as np
import pytest

import rtdl_b200 as rt
from rtdl_b200 import workloads
from rtdl_b200.autotune import DEFAULT, Autotuner, Config, tune_records

pytestmark = pytest.mark.gpu


def test_every_configuration_gives_the_same_rows(gpu):
    probe, build = workloads.clustered_3d(100_000, 20_000)
    ref = None
    try:
        for leaf in (4, 8, 16):
            for trav in ("packet_hybrid", "packet", "packet_cube", "lane"):
                for bt in (128, 256):
                    Config(leaf, trav, bt).apply()
                    view = rt.runtime.fixed_radius_neighbors(probe, build, radius=0.006, k_max=48)
                    rows = view.to_numpy()
                    view.close()
                    if ref is None:
                        ref = rows
                    assert np.array_equal(rows.view(np.uint8), ref.view(np.uint8)), (leaf, trav, bt)
    finally:
        DEFAULT.apply()


def test_tune_caches_the_fastest_candidate(gpu, tmp_path):
    probe, build = workloads.clustered_3d(60_000, 30_000)
    tuner = Autotuner(tmp_path / "tune.json", repeats=1, leaf_sizes=(8, 16), traversals=("packet", "lane"),
                      block_threads=(128,))
    try:
        key, cfg = tune_records(build, probe, radius=0.008, k_max=32, tuner=tuner)
        assert cfg in tuner.candidates
        entry = tuner.cache[key]
        assert len(entry["ms"]) == 4
        assert min(entry["ms"].values()) == entry["ms"][f"{cfg.leaf_size}/{cfg.traversal}/{cfg.block_threads}"]
        again = Autotuner(tmp_path / "tune.json")
        assert again.lookup(key) == cfg
    finally:
        DEFAULT.apply()
