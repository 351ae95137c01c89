"""Directed/undirected Hausdorff on the device vs the reference app's results."""
import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", G.load_hausdorff(), ids=lambda c: f"copies{c['copies']}")
def test_hausdorff_matches_reference_app(gpu, case):
    a = rt.pack_points(**{("ids" if k == "id" else k): v for k, v in G.points_columns(case["points_a"], 2).items()})
    b = rt.pack_points(**{("ids" if k == "id" else k): v for k, v in G.points_columns(case["points_b"], 2).items()})
    got = rt.hausdorff_distance(a, b)
    for key in ("directed_a_to_b", "directed_b_to_a"):
        exp = case[key]
        assert got[key]["distance"] == float.fromhex(exp["distance"])
        assert (got[key]["source_id"], got[key]["target_id"], got[key]["row_count"]) == (
            exp["source_id"], exp["target_id"], exp["row_count"])
    assert got["hausdorff_distance"] == float.fromhex(case["hausdorff_distance"])
    assert got["witness_direction"] == case["witness_direction"]


def test_directed_hausdorff_and_nearest_match_oracle(gpu):
    from rtdl_b200 import workloads

    a, b = workloads.hausdorff_2d(1 << 15)
    with rt.B200Scene(rt.pack_points(records=b)) as scene:
        got, nd, ni = scene.directed_hausdorff(rt.pack_points(records=a), with_nearest=True)
    dist, nid = O.nearest(a, b, threads=8)
    assert np.array_equal(nd.view(np.uint64), dist.view(np.uint64))
    assert np.array_equal(ni, nid)
    exp = O.directed_hausdorff(a, b, threads=8)
    assert got == exp


def test_hausdorff_rejects_empty_sets(gpu):
    pts = rt.pack_points(ids=[1], x=[0.0], y=[0.0])
    empty = rt.pack_points(ids=np.zeros(0, np.uint32), x=np.zeros(0), y=np.zeros(0))
    with pytest.raises(RuntimeError, match="non-empty"):
        rt.directed_hausdorff(empty, pts)
