"""binder_grid_neighbors_noalloc — the grid build + 27-cell probe for callers
that cannot allocate device memory (their own pool owns every device byte, or an
allocation would stall a latency-critical loop).  Called through the C ABI with
caller-owned device buffers, it must return exactly what the allocating entry
point binder_grid_neighbors returns (neighbour lists are bit-exact everywhere in
this suite), on two calls in a row that reuse the library's scratch array.

Collected last (file name) so a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn(pkg):
    f = pkg.lib().binder_grid_neighbors_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_void_p]
    return f


def _call(pkg, torch, cell, ag, q, cap):
    dev = torch.device("cuda", 0)
    d_ag = [torch.from_numpy(np.ascontiguousarray(ag[:, k])).to(dev) for k in range(3)]
    d_q = [torch.from_numpy(np.ascontiguousarray(q[:, k])).to(dev) for k in range(3)]
    d_off = torch.full((len(q) + 1,), -7, dtype=torch.int64, device=dev)
    d_idx = torch.full((max(cap, 1),), -7, dtype=torch.int32, device=dev)
    total = C.c_size_t(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ptr = lambda t: t.data_ptr() if t.numel() else None  # noqa: E731 (empty inputs: NULL)
    st = _fn(pkg)(cell, *(ptr(t) for t in d_ag), len(ag), *(ptr(t) for t in d_q), len(q),
                  d_off.data_ptr(), d_idx.data_ptr() if cap else None, cap, C.byref(total), stream)
    torch.cuda.synchronize(dev)
    return st, total.value, d_off.cpu().numpy(), d_idx.cpu().numpy().view(np.uint32)


def test_noalloc_matches_allocating_entry_point_on_two_calls(pkg, ctx):
    import torch
    rng = np.random.default_rng(20251203)
    for call, (cell, n_ag, n_q) in enumerate([(8.0, 2505, 700), (10.0, 300, 1200)]):
        ag = rng.uniform(-25, 25, size=(n_ag, 3)).astype(np.float32)
        q = rng.uniform(-35, 35, size=(n_q, 3)).astype(np.float32)
        q[:50] = ag[:50]
        ref_off, ref_idx = ctx.grid_neighbors(cell, ag[:, 0], ag[:, 1], ag[:, 2], q[:, 0], q[:, 1], q[:, 2])
        st, total, off, idx = _call(pkg, torch, cell, ag, q, cap=len(ref_idx) + 16)
        assert st == 0, (call, st)
        assert total == len(ref_idx)
        assert np.array_equal(off, ref_off), call
        assert np.array_equal(idx[:total], ref_idx), call


def test_noalloc_limits(pkg):
    import torch
    ag = np.zeros((65537, 3), np.float32)
    q = np.zeros((4, 3), np.float32)
    st, *_ = _call(pkg, torch, 10.0, ag, q, cap=16)
    assert st == 1  # BINDER_ERR_ARG: more atoms than the scratch array holds
    ag = np.float32([[0, 0, 0], [1000, 1000, 1000]])
    st, *_ = _call(pkg, torch, 1.0, ag, q, cap=16)
    assert st == 6  # BINDER_ERR_GRID: occupied box beyond the scratch array
    ag = np.float32([[0, 0, 0], [1, 0, 0]])
    st, total, *_ = _call(pkg, torch, 10.0, ag, q, cap=1)
    assert st == 9 and total == 8  # BINDER_ERR_CAPACITY reports the size needed


def test_noalloc_edge_cases_match_allocating_entry_point(pkg, ctx):
    """Empty antigen, empty probes, no neighbours with a NULL index buffer, and a
    NaN antigen coordinate (BINDER_ERR_NAN) followed by a good call: the scratch is
    re-initialised by every call, so nothing of a failed call leaks into the next."""
    import torch
    rng = np.random.default_rng(7)
    ag = rng.uniform(-20, 20, size=(400, 3)).astype(np.float32)
    q = rng.uniform(-30, 30, size=(300, 3)).astype(np.float32)
    far = np.float32([[500, 500, 500], [-500, 0, 0]])
    cases = [(ag[:0], q, 64), (ag, q[:0], 64), (ag, far, 0)]
    for a, p, cap in cases:
        ref_off, ref_idx = ctx.grid_neighbors(8.0, a[:, 0], a[:, 1], a[:, 2], p[:, 0], p[:, 1], p[:, 2])
        st, total, off, idx = _call(pkg, torch, 8.0, a, p, cap=cap)
        assert st == 0 and total == len(ref_idx) == 0, (len(a), len(p), st, total)
        assert np.array_equal(off, ref_off)
    bad = ag.copy()
    bad[17, 1] = np.nan
    with pytest.raises(pkg.BinderError) as e:
        ctx.grid_neighbors(8.0, bad[:, 0], bad[:, 1], bad[:, 2], q[:, 0], q[:, 1], q[:, 2])
    assert e.value.status == 5
    st, *_ = _call(pkg, torch, 8.0, bad, q, cap=1 << 16)
    assert st == 5  # BINDER_ERR_NAN, as the allocating entry point reports
    ref_off, ref_idx = ctx.grid_neighbors(8.0, ag[:, 0], ag[:, 1], ag[:, 2], q[:, 0], q[:, 1], q[:, 2])
    for _ in range(2):
        st, total, off, idx = _call(pkg, torch, 8.0, ag, q, cap=len(ref_idx))
        assert st == 0 and total == len(ref_idx)
        assert np.array_equal(off, ref_off) and np.array_equal(idx[:total], ref_idx)
