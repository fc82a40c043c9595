"""gpsm_select_vertices_static: the same selection as gpsm_select_vertices
for callers that must not allocate device memory (a host that owns every
allocation, or a caller that cannot pay for cudaMalloc at call time). Its
scratch is a fixed array inside the library, shared by every call.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _select(lib, fn, lab, off, n, label, d, out, cnt):
    if fn == "static":
        rc = lib.gpsm_select_vertices_static(C.c_void_p(lab.data_ptr()), C.c_void_p(off.data_ptr()), n, label, d,
                                             C.c_void_p(out.data_ptr()), C.c_void_p(cnt.data_ptr()), None)
    else:
        rc = lib.gpsm_select_vertices(None, C.c_void_p(lab.data_ptr()), C.c_void_p(off.data_ptr()), n, label, d,
                                      C.c_void_p(out.data_ptr()), C.c_void_p(cnt.data_ptr()))
    assert rc == 0, rc
    import torch
    torch.cuda.synchronize()
    k = int(cnt.item())
    return out[:k].cpu().numpy().copy()


def test_static_scratch_variant_matches_allocating_entry_point(gpu, lib):
    import torch
    g = W.rmat_graph(18, 1_000_000, 16, 1.0, seed=21)
    lab = torch.from_numpy(g.labels.astype(np.int32)).cuda()
    off = torch.from_numpy(g.offsets.astype(np.int64).astype(np.int32)).cuda()
    out_a = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    out_b = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    cnt_a = torch.zeros(1, dtype=torch.int32, device="cuda")
    cnt_b = torch.zeros(1, dtype=torch.int32, device="cuda")
    deg = np.diff(g.offsets.astype(np.int64))
    # two calls in a row, each checked against the allocating entry point
    for label, d in [(1, 2), (3, 0)]:
        want = _select(lib, "alloc", lab, off, g.n, label, d, out_a, cnt_a)
        got = _select(lib, "static", lab, off, g.n, label, d, out_b, cnt_b)
        assert np.array_equal(got, want)
        assert np.array_equal(want.astype(np.int64), np.flatnonzero((g.labels == label) & (deg >= d)))


def test_static_scratch_variant_at_its_limit_then_small(gpu, lib):
    """n = 2^22 fills the whole static bitmap and uses every compaction tile;
    a smaller graph right after must not see the larger call's bits."""
    import torch
    rng = np.random.default_rng(5)
    for n in (1 << 22, 70_001):
        labels = rng.integers(1, 9, size=n).astype(np.int32)
        deg = rng.integers(0, 6, size=n)
        offsets = np.concatenate([[0], np.cumsum(deg)]).astype(np.int32)
        lab = torch.from_numpy(labels).cuda()
        off = torch.from_numpy(offsets).cuda()
        out_a = torch.zeros(n, dtype=torch.int32, device="cuda")
        out_b = torch.zeros(n, dtype=torch.int32, device="cuda")
        cnt_a = torch.zeros(1, dtype=torch.int32, device="cuda")
        cnt_b = torch.zeros(1, dtype=torch.int32, device="cuda")
        for label, d in [(2, 1), (7, 4)]:
            want = np.flatnonzero((labels == label) & (deg >= d))
            got = _select(lib, "static", lab, off, n, label, d, out_b, cnt_b)
            assert np.array_equal(got.astype(np.int64), want), (n, label, d)
            assert np.array_equal(_select(lib, "alloc", lab, off, n, label, d, out_a, cnt_a), got)


def test_static_scratch_variant_rejects_graphs_over_its_limit(gpu, lib):
    import torch
    lab = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.gpsm_select_vertices_static(C.c_void_p(lab.data_ptr()), C.c_void_p(lab.data_ptr()), (1 << 22) + 1, 1,
                                         0, C.c_void_p(lab.data_ptr()), C.c_void_p(lab.data_ptr()), None)
    assert rc == -5  # GPSM_ERR_BUDGET, nothing queued
