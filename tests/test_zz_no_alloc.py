"""The no-allocation entry point against the plan-based deterministic path.

bspk_iaf_exact_run_noalloc serves callers that cannot allocate device memory
(they run inside another framework's memory pool or allocation hooks): the
test plays such a caller, owning every buffer (allocated here with torch) and
passing plain device pointers through the C ABI.  Its output must equal the
plan-based FP64 deterministic path bit for bit (the tolerance of the other
deterministic-mode tests), on two calls in a row, so a second call proves the
shared scratch array is cleared between calls.  This file is collected last
on purpose.
"""
import ctypes as C
import math

import numpy as np
import pytest

from brainpy.state_b200 import _lib

pytestmark = pytest.mark.gpu

PARAMS = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]  # iaf_psc_alpha


def _network(n=300, K=30, seed=3):
    rng = np.random.default_rng(seed)
    pre = rng.integers(0, n, size=(n, K)).reshape(-1)
    post = np.repeat(np.arange(n), K)
    delay = rng.integers(10, 25, size=pre.size)
    w = np.where(pre < int(0.8 * n), 20.68, -103.4)
    order = np.argsort(pre, kind="stable")  # CSR by pre (what the plan takes)
    indptr = np.concatenate([[0], np.cumsum(np.bincount(pre, minlength=n))])
    csr = (indptr, post[order], w[order], delay[order])
    # in-edges per post, ascending pre (stable in CSR order)
    corder = np.lexsort((np.arange(pre.size), pre[order], post[order]))
    cpost = post[order][corder]
    cindptr = np.concatenate([[0], np.cumsum(np.bincount(cpost, minlength=n))])
    cedges = (pre[order][corder].astype(np.uint64) |
              ((delay[order][corder].astype(np.uint64) + 1) << 24)).astype(np.uint32)
    csc = (cindptr, cedges, w[order][corder])
    v0 = rng.uniform(0.0, 20.0, n)
    return n, csr, csc, v0, int(delay.min()), int(delay.max())


def _reference(n, csr, v0, n_steps):
    pl = _lib.Plan(0.1, precision=64, deterministic=True)
    pl.add_pop(n, PARAMS)
    pl.add_poisson(0, 17789.0, 20.68, 15, 77)
    pl.add_csr(0, 0, *csr)
    pl.upload()
    pl.set_state(0, "V_m", v0)
    pl.run(n_steps)
    st, g = pl.spikes()
    return st, g, pl.get_state(0, "V_m")


def _fn():
    L = _lib.lib()
    fn = L.bspk_iaf_exact_run_noalloc
    fn.restype = C.c_int
    vp = C.c_void_p
    fn.argtypes = [C.c_double, vp, C.c_int, C.c_int, vp, vp, vp, C.c_double, C.c_int, C.c_int,
                   C.c_double, C.c_double, C.c_int, C.c_uint32, vp, vp, C.c_int64, vp, vp,
                   C.c_int64, vp, vp, vp]
    return L, fn


def _call(fn, n, csc, v0, dmin, dmax, n_steps, cap):
    """One call with caller-owned torch buffers; returns (rc, status, count,
    steps, gids, V_m) with the spike pairs cut to min(count, cap)."""
    import torch
    dev = torch.device("cuda")
    indptr = torch.tensor(csc[0], dtype=torch.int64, device=dev)
    edges = torch.tensor(csc[1].view(np.int32), dtype=torch.int32, device=dev)
    w = torch.tensor(csc[2], dtype=torch.float64, device=dev)
    params = np.asarray(PARAMS, np.float64)
    state = torch.zeros((6, n), dtype=torch.float64, device=dev)
    state[0] = torch.tensor(v0, dtype=torch.float64)
    refr = torch.zeros(n, dtype=torch.int32, device=dev)
    spk_step = torch.full((max(cap, 1),), -1, dtype=torch.int64, device=dev)
    spk_gid = torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.full((1,), -99, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(0.1, params.ctypes.data_as(C.c_void_p), params.size, n, indptr.data_ptr(),
            edges.data_ptr(), w.data_ptr(), 0.0, dmin, dmax, 17789.0, 20.68, 15, 77,
            state.data_ptr(), refr.data_ptr(), n_steps, spk_step.data_ptr(),
            spk_gid.data_ptr(), cap, count.data_ptr(), status.data_ptr(), stream)
    if rc != 0:
        return rc, None, None, None, None, None
    torch.cuda.synchronize()
    m = int(count.item())
    k = min(m, cap)
    return (rc, int(status.item()), m, spk_step[:k].cpu().numpy(), spk_gid[:k].cpu().numpy(),
            state[0].cpu().numpy())


def test_noalloc_matches_plan_path_twice():
    n, csr, csc, v0, dmin, dmax = _network()
    n_steps = 600
    ref_st, ref_g, ref_v = _reference(n, csr, v0, n_steps)
    assert ref_st.size > 0
    L, fn = _fn()
    for call in range(2):
        rc, status, m, st, g, v = _call(fn, n, csc, v0, dmin, dmax, n_steps, 200000)
        assert rc == 0, L.bspk_last_error()
        assert status == 0
        assert m == ref_st.size
        order = np.lexsort((g, st))
        np.testing.assert_array_equal(st[order], ref_st)
        np.testing.assert_array_equal(g[order], ref_g)
        np.testing.assert_array_equal(v, ref_v)


def test_noalloc_flags_spikes_beyond_capacity():
    """A capacity below the call's spike count: the count is the true total,
    only `cap` pairs are written (each one of the plan path's spikes) and the
    status is the overflow code (2)."""
    n, csr, csc, v0, dmin, dmax = _network()
    ref_st, ref_g, _ = _reference(n, csr, v0, 300)
    L, fn = _fn()
    rc, status, m, st, g, _ = _call(fn, n, csc, v0, dmin, dmax, 300, 5)
    assert rc == 0, L.bspk_last_error()
    assert m == ref_st.size > 5
    assert status == 2
    ref = set(zip(ref_st.tolist(), ref_g.tolist()))
    assert st.size == 5 and all((int(a), int(b)) in ref for a, b in zip(st, g))


def test_noalloc_largest_resident_network():
    """The largest network the cooperative launch keeps resident (256 neurons
    per SM) matches the plan path; one neuron more is refused up front."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n_max = 256 * sms
    n, csr, csc, v0, dmin, dmax = _network(n=n_max, K=20, seed=5)
    n_steps = 60
    ref_st, ref_g, ref_v = _reference(n, csr, v0, n_steps)
    L, fn = _fn()
    rc, status, m, st, g, v = _call(fn, n, csc, v0, dmin, dmax, n_steps, 500000)
    assert rc == 0, L.bspk_last_error()
    assert status == 0 and m == ref_st.size
    order = np.lexsort((g, st))
    np.testing.assert_array_equal(st[order], ref_st)
    np.testing.assert_array_equal(g[order], ref_g)
    np.testing.assert_array_equal(v, ref_v)
    n1, _, csc1, v1, dmin1, dmax1 = _network(n=n_max + 1, K=2, seed=6)
    rc, *_ = _call(fn, n1, csc1, v1, dmin1, dmax1, 10, 1000)
    assert rc == -4
    assert b"co-resident" in L.bspk_last_error()


def test_noalloc_rejects_oversized_network():
    L = _lib.lib()
    fn = L.bspk_iaf_exact_run_noalloc
    fn.restype = C.c_int
    params = np.asarray(PARAMS, np.float64)
    dummy = C.c_void_p(16)
    rc = fn(C.c_double(0.1), params.ctypes.data_as(C.c_void_p), C.c_int(10), C.c_int(70000),
            dummy, dummy, None, C.c_double(0.0), C.c_int(10), C.c_int(20), C.c_double(100.0),
            C.c_double(1.0), C.c_int(15), C.c_uint32(1), dummy, dummy, C.c_int64(10), dummy,
            dummy, C.c_int64(10), dummy, dummy, None)
    assert rc == -1
    assert b"65536" in L.bspk_last_error()
