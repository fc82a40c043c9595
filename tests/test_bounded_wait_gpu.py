"""A bounded device wait that runs out, and the engine afterwards.

Every wait between blocks (the decoupled look-back of the compaction, scan
and join-locate kernels) polls its predecessor at most scan_spin_limit times;
then the kernel raises a device flag, carries on with in-range values, and
the call returns GPSM_ERR_TIMEOUT instead of hanging (the reference has no
such path: its CUDA errors exit the process, match/Match.h:58-65).

Here the wait is made to run out on purpose without faulting anything: a
stray ticket taken from the engine's ticket counter means the first tile of
each scan waits for a tile 0 that no block holds. The GPU must still answer,
and the next query (the engine re-reads the counter) must be exact.
"""
import time

import numpy as np
import pytest

from gpsm_b200 import GpsmError
from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_lookback_wait_runs_out_then_engine_recovers(gpu, lib):
    g = W.rmat_graph(16, 400_000, 4, 1.0, seed=12)  # 2^16 vertices: two compaction tiles per scan
    dg = gpu.DeviceGraph(g)
    q = W.random_walk_query(g, 5, 3, W.MODE_TREE)
    want = gpu.match(dg, q, cap=20_000)
    assert want.count > 0
    old = gpu.get_tuning()["scan_spin_limit"]
    gpu.set_tuning(scan_spin_limit=64)
    try:
        assert lib.gpsm_debug_skew_scan_tickets(None, 1) == 0
        t0 = time.perf_counter()
        with pytest.raises(GpsmError) as err:
            gpu.match(dg, q, cap=20_000)
        assert err.value.code == -6  # GPSM_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 30
    finally:
        gpu.set_tuning(scan_spin_limit=old)
    again = gpu.match(dg, q, cap=20_000)
    assert again.count == want.count
    assert np.array_equal(again.rows, want.rows)
    dg.free()
