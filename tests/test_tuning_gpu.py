"""Launch choices change speed, not results: the filter's team widths give
the same rows."""
import numpy as np
import pytest

from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_filter_team_widths_give_the_same_rows(gpu):
    wl = W.workload("rmat20_mix", count=6)
    dg = gpu.DeviceGraph(wl.graph)
    old = gpu.get_tuning()
    try:
        ref = [gpu.match(dg, q, cap=50_000) for q in wl.queries]
        for ft, et in ((4, 8), (8, 32), (32, 8)):
            gpu.set_tuning(filter_team=ft, explore_team=et)
            assert gpu.get_tuning()["filter_team"] == ft and gpu.get_tuning()["explore_team"] == et
            for q, r in zip(wl.queries, ref):
                o = gpu.match(dg, q, cap=50_000)
                assert o.count == r.count and np.array_equal(o.pos2id, r.pos2id)
                assert np.array_equal(o.rows, r.rows)
    finally:
        gpu.set_tuning(**{k: v for k, v in old.items() if v})
