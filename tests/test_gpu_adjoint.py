"""GPU tests of the hand-written BPTT adjoint (C ABI through the torch wrapper).

  * FP64, hard and relaxed forward, with and without detach_reset: loss,
    spike count and both gradients bit-exact against the float64 oracle (the
    kernels are compiled without FMA contraction and follow its order);
  * checkpoint spacing does not change the result (bitwise);
  * FP32: gradients within 1e-3 relative of the FP64 ones on a short episode;
    the FP32 contraction mode (dense products over (step, trial), the
    default) against the FP32 read-modify-write mode within 1e-4 relative;
  * central finite differences (h = 1e-3) on 64 random weights of the
    gradient-training network (800 + 200 neurons, batch 64) over 200 steps in
    the relaxed forward with refractoriness off (the loss is then smooth in
    the weights): |adjoint - FD| <= 1e-3 relative.  The relaxed soft reset
    multiplies perturbations by up to 1 + slope * (V_th - V_reset) / 2 per
    threshold passage, so over 400+ steps a few weights leave the linear
    range of h = 1e-3 (their FD error then shrinks with h);
  * torch.autograd.Function plumbing.
"""
import numpy as np
import pytest

from brainpy.state_b200.lif_task import make_task

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _small(relaxed=False, detach=False, t_ref=2.0, seed=3, n_steps=120):
    params = [-70.0, 250.0, 10.0, t_ref, -55.0, -70.0, 2.0, 2.0, 0.0]
    return make_task(n_exc=40, n_inh=10, n_in=20, batch=3, n_steps=n_steps, relaxed=relaxed,
                     detach_reset=detach, params=params, w_in_scale=900.0, seed=seed)


def _gpu(T, precision=64, ckpt=50, split=None, contraction=None):
    from brainpy.state_b200.autograd import LifAdjoint
    dt = torch.float64 if precision == 64 else torch.float32
    adj = LifAdjoint(T["cfg"], T["row_ptr"], T["col"], precision=precision, ckpt_every=ckpt)
    if split is not None:
        assert adj.ctas_per_trial == split
    # FP32 handles contract by default, FP64 handles never do
    assert adj.contraction == (precision == 32)
    if contraction is not None:
        adj.contraction = contraction
    w = torch.tensor(T["w"], dtype=dt, device="cuda")
    wi = torch.tensor(T["w_in"], dtype=dt, device="cuda")
    inp = torch.tensor(T["inputs"], dtype=torch.uint8, device="cuda")
    tg = torch.tensor(T["targets"], dtype=dt, device="cuda")
    nsp = torch.zeros((), dtype=torch.int64, device="cuda")
    loss = adj.forward(w, wi, inp, tg, n_spikes=nsp)
    dw, dwi = adj.backward()
    adj.status()
    torch.cuda.synchronize()
    out = (float(loss), dw.double().cpu().numpy(), dwi.double().cpu().numpy(), int(nsp))
    adj.close()
    return out


@pytest.mark.parametrize("relaxed,detach", [(False, False), (False, True), (True, False)])
def test_fp64_adjoint_bitwise_matches_oracle(oracle, relaxed, detach):
    T = _small(relaxed=relaxed, detach=detach)
    L, dw, dwi, nsp = oracle.lif_bptt(T["cfg"], T["row_ptr"], T["col"], T["w"], T["w_in"],
                                      T["inputs"], T["targets"])
    gL, gdw, gdwi, gnsp = _gpu(T)
    assert nsp > 0 and gnsp == nsp
    assert gL == L
    np.testing.assert_array_equal(gdw, dw)
    np.testing.assert_array_equal(gdwi, dwi)


@pytest.mark.parametrize("relaxed", [False, True])
def test_fp64_adjoint_two_cta_clusters_match_oracle(oracle, relaxed):
    """A network of 150 neurons: each trial runs on a cluster of two CTAs that
    own 75 neurons each and exchange spike and adjoint vectors through
    distributed shared memory; still bit-identical to the oracle."""
    params = [-70.0, 250.0, 10.0, 2.0, -55.0, -70.0, 2.0, 2.0, 0.0]
    T = make_task(n_exc=120, n_inh=30, n_in=20, batch=3, n_steps=120, relaxed=relaxed,
                  params=params, w_in_scale=900.0, seed=5)
    L, dw, dwi, nsp = oracle.lif_bptt(T["cfg"], T["row_ptr"], T["col"], T["w"], T["w_in"],
                                      T["inputs"], T["targets"])
    gL, gdw, gdwi, gnsp = _gpu(T, split=2)
    assert nsp > 0 and gnsp == nsp
    assert gL == L
    np.testing.assert_array_equal(gdw, dw)
    np.testing.assert_array_equal(gdwi, dwi)
    # the small network keeps one CTA per trial
    assert _gpu(_small(), split=1)[3] > 0


def test_checkpoint_spacing_is_invisible():
    T = _small(n_steps=130)
    ref = _gpu(T, ckpt=130)
    for ck in (1, 7, 50):
        got = _gpu(T, ckpt=ck)
        assert got[0] == ref[0]
        np.testing.assert_array_equal(got[1], ref[1])
        np.testing.assert_array_equal(got[2], ref[2])


def test_fp32_gradient_tracks_fp64():
    T = _small(n_steps=60)
    L64, dw64, dwi64, n64 = _gpu(T, precision=64)
    L32, dw32, dwi32, n32 = _gpu(T, precision=32)
    assert n32 == n64
    assert abs(L32 - L64) <= 1e-4 * abs(L64)
    for a, b in ((dw32, dw64), (dwi32, dwi64)):
        np.testing.assert_allclose(a, b, rtol=1e-3, atol=1e-3 * np.abs(b).max())


@pytest.mark.parametrize("relaxed", [False, True])
def test_fp32_contraction_matches_read_modify_write(relaxed):
    # the two FP32 ways of forming dL/dw, dL/dw_in differ only in the order
    # of the FP32 additions
    T = _small(relaxed=relaxed, n_steps=150)
    L1, dw1, dwi1, n1 = _gpu(T, precision=32, contraction=True)
    L0, dw0, dwi0, n0 = _gpu(T, precision=32, contraction=False)
    assert (L1, n1) == (L0, n0)
    assert np.abs(dw0).max() > 0 and np.abs(dwi0).max() > 0
    for a, b in ((dw1, dw0), (dwi1, dwi0)):
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-5 * np.abs(b).max())


def test_fp64_handle_refuses_contraction():
    from brainpy.state_b200.autograd import LifAdjoint
    T = _small(n_steps=20)
    adj = LifAdjoint(T["cfg"], T["row_ptr"], T["col"], precision=64)
    with pytest.raises(NotImplementedError):
        adj.contraction = True
    adj.close()


def test_finite_differences_full_workload():
    params = [-70.0, 250.0, 10.0, 0.0, -55.0, -70.0, 2.0, 2.0, 0.0]  # t_ref = 0
    T = make_task(relaxed=True, params=params, n_steps=200)
    from brainpy.state_b200.autograd import LifAdjoint
    dt = torch.float64
    adj = LifAdjoint(T["cfg"], T["row_ptr"], T["col"], precision=64, ckpt_every=50)
    w = torch.tensor(T["w"], dtype=dt, device="cuda")
    wi = torch.tensor(T["w_in"], dtype=dt, device="cuda")
    inp = torch.tensor(T["inputs"], dtype=torch.uint8, device="cuda")
    tg = torch.tensor(T["targets"], dtype=dt, device="cuda")
    adj.forward(w, wi, inp, tg)
    dw, dwi = adj.backward()
    dw, dwi = dw.cpu().numpy(), dwi.cpu().numpy().reshape(-1)

    def loss(w_, wi_):
        return float(adj.forward(w_, wi_, inp, tg))

    rng = np.random.default_rng(7)
    h = 1e-3
    adjv, fdv = [], []
    for q in rng.choice(w.numel(), 32, replace=False):
        wp = w.clone()
        wp[q] += h
        lp = loss(wp, wi)
        wp[q] -= 2 * h
        lm = loss(wp, wi)
        adjv.append(dw[q])
        fdv.append((lp - lm) / (2 * h))
    for q in rng.choice(wi.numel(), 32, replace=False):
        wp = wi.clone().reshape(-1)
        wp[q] += h
        lp = loss(w, wp.reshape(wi.shape))
        wp[q] -= 2 * h
        lm = loss(w, wp.reshape(wi.shape))
        adjv.append(dwi[q])
        fdv.append((lp - lm) / (2 * h))
    adjv, fdv = np.array(adjv), np.array(fdv)
    floor = 1e-3 * np.abs(fdv).max()
    rel = np.abs(adjv - fdv) / np.maximum(np.abs(fdv), floor)
    assert rel.max() <= 1e-3, (rel.max(), adjv[rel.argmax()], fdv[rel.argmax()])
    adj.close()


def test_autograd_function_backward():
    from brainpy.state_b200.autograd import LifAdjoint, LifBpttLoss
    T = _small()
    adj = LifAdjoint(T["cfg"], T["row_ptr"], T["col"], precision=64)
    w = torch.tensor(T["w"], dtype=torch.float64, device="cuda", requires_grad=True)
    wi = torch.tensor(T["w_in"], dtype=torch.float64, device="cuda", requires_grad=True)
    inp = torch.tensor(T["inputs"], dtype=torch.uint8, device="cuda")
    tg = torch.tensor(T["targets"], dtype=torch.float64, device="cuda")
    loss = LifBpttLoss.apply(w, wi, inp, tg, adj)
    (2.0 * loss).backward()
    _, dw, dwi, _ = _gpu(T)
    np.testing.assert_allclose(w.grad.cpu().numpy(), 2.0 * dw, rtol=1e-15, atol=0)
    np.testing.assert_allclose(wi.grad.cpu().numpy(), 2.0 * dwi, rtol=1e-15, atol=0)
    adj.close()


def test_xla_custom_call_targets_match_the_c_abi():
    """Call the XLA targets the way XLA does (stream, buffer array, opaque)."""
    import ctypes as C
    import struct
    from brainpy.state_b200 import _lib
    from brainpy.state_b200.autograd import LifAdjoint
    T = _small()
    adj = LifAdjoint(T["cfg"], T["row_ptr"], T["col"], precision=64)
    dt = torch.float64
    w = torch.tensor(T["w"], dtype=dt, device="cuda")
    wi = torch.tensor(T["w_in"], dtype=dt, device="cuda")
    inp = torch.tensor(T["inputs"], dtype=torch.uint8, device="cuda")
    tg = torch.tensor(T["targets"], dtype=dt, device="cuda")
    loss = torch.zeros((), dtype=dt, device="cuda")
    dw = torch.zeros_like(w)
    dwi = torch.zeros_like(wi)
    st1 = torch.full((), -99, dtype=torch.int32, device="cuda")
    st2 = torch.full((), -99, dtype=torch.int32, device="cuda")
    L = _lib.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    op = struct.pack("<Q", adj._h.value)
    bufs = (C.c_void_p * 6)(*[t.data_ptr() for t in (w, wi, inp, tg, loss, st1)])
    L.bspk_xla_adjoint_forward(st, bufs, op, len(op))
    bufs = (C.c_void_p * 7)(*[t.data_ptr() for t in (w, wi, inp, tg, dw, dwi, st2)])
    L.bspk_xla_adjoint_backward(st, bufs, op, len(op))
    torch.cuda.synchronize()
    ref = _gpu(T)
    assert int(st1) == 0 and int(st2) == 0
    assert float(loss) == ref[0]
    np.testing.assert_array_equal(dw.cpu().numpy(), ref[1])
    np.testing.assert_array_equal(dwi.cpu().numpy(), ref[2])
    # a bad opaque (null handle): status BSPK_ERR_ARG, NaN loss, no hang
    bad = struct.pack("<Q", 0)
    bufs = (C.c_void_p * 6)(*[t.data_ptr() for t in (w, wi, inp, tg, loss, st1)])
    L.bspk_xla_adjoint_forward(st, bufs, bad, len(bad))
    torch.cuda.synchronize()
    assert int(st1) == -1 and torch.isnan(loss).item()
    adj.close()


def test_xla_run_and_step_targets_write_step_and_status():
    """bspk_xla_run / bspk_xla_step as XLA calls them: the step counter and a
    zero status land in device buffers without a host synchronisation; the
    states equal a plan advanced through bspk_run; a null plan gives status
    BSPK_ERR_ARG and step -1."""
    import ctypes as C
    import struct
    from brainpy.state_b200 import _lib
    from tests.netbuild import Net
    L = _lib.lib()
    net = Net()
    a, b = net.to_plan(precision=64), net.to_plan(precision=64)
    step = torch.zeros((), dtype=torch.int64, device="cuda")
    status = torch.full((), -99, dtype=torch.int32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    bufs = (C.c_void_p * 2)(step.data_ptr(), status.data_ptr())
    op = struct.pack("<Qq", a._h.value, 40)
    L.bspk_xla_run(st, bufs, op, len(op))
    torch.cuda.synchronize()
    assert int(step) == 40 and int(status) == 0
    one = struct.pack("<Q", a._h.value)
    for k in range(3):
        L.bspk_xla_step(st, bufs, one, len(one))
    torch.cuda.synchronize()
    assert int(step) == 43 and int(status) == 0
    b.run(43)
    np.testing.assert_array_equal(a.get_state(0, "V_m"), b.get_state(0, "V_m"))
    bad = struct.pack("<Qq", 0, 10)
    L.bspk_xla_run(st, bufs, bad, len(bad))
    torch.cuda.synchronize()
    assert int(step) == -1 and int(status) == -1
