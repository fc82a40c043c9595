"""Multi-GPU is replicas only: each rank matches its own batch of the same
shape against its own copy of the graph, and the bench takes the max of the
ranks' step times and the sum of their work. The host side of that runs
here as two gloo ranks on CPU."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, pg = bench.dist_setup()
    assert (r, w) == (rank, world) and pg is not None
    bounds = bench.slice_bounds(4096, 20)
    mine = [bench.slice_of(k, rank, world, len(bounds)) for k in range(10)]
    sizes = [bounds[s][1] - bounds[s][0] for s in mine]
    bench.barrier(pg)
    mx = bench.max_over_ranks(pg, 10.0 + rank)
    sm = bench.sum_over_ranks(pg, sum(sizes))
    q.put((rank, mx, sm, mine, sizes))
    pg.destroy_process_group()


def test_two_gloo_ranks_reduce_and_take_disjoint_equal_sized_slices():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res[0][1] == res[1][1] == 11.0          # max over ranks
    assert res[0][2] == res[1][2] == sum(res[0][4]) + sum(res[1][4])  # total work over ranks
    # ten steps of two ranks cover the twenty slices once, each slice by one rank
    assert sorted(res[0][3] + res[1][3]) == list(range(20))
    assert all(abs(a - b) <= 1 for a, b in zip(res[0][4], res[1][4]))  # weak scaling: equal work per rank


def test_reference_arm_prints_one_json_line_without_the_engine():
    """The reference arm draws its workload through the oracle: libgpsm.so
    is never mapped in its process."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'small_er', "
            "'--steps', '1', '--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
            "print('MAPPED', 'libgpsm' in open('/proc/self/maps').read())")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert "MAPPED False" in out.stdout


def test_ranks_on_one_host_share_the_page_locked_pool_and_sleep_in_waits():
    """Eight ranks on a host with 256 GiB: each gets an eighth of the default
    pool (a quarter of host memory) and sleeping waits; a caller's own
    choices stand; a single rank keeps the library defaults."""
    sys.path.insert(0, ROOT)
    import bench
    s = bench.rank_host_settings(8, {}, 256.0)
    assert s == {"GPSM_HOST_POOL_GB": str(64.0 / 8), "GPSM_BLOCKING_SYNC": "1"}
    s = bench.rank_host_settings(8, {"GPSM_HOST_POOL_GB": "3", "GPSM_BLOCKING_SYNC": "0"}, 256.0)
    assert s == {}
    assert bench.rank_host_settings(1, {}, 256.0) == {}
    assert float(bench.rank_host_settings(64, {}, 64.0)["GPSM_HOST_POOL_GB"]) == 2.0  # at least 2 GiB each
