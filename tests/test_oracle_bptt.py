"""CPU checks of the float64 BPTT restatement (the checker of the GPU adjoint).

In the relaxed forward (spikes = the surrogate primitive, soft reset) the
loss is a smooth function of the weights when refractoriness is off, so the
restatement's adjoint must equal central finite differences: this pins the
adjoint arithmetic without any GPU.  The hard forward is piecewise constant
in the weights (its gradient is the surrogate's by definition), so there the
test only checks consistency with the relaxed trajectory's structure.
"""
import numpy as np

from brainpy.state_b200.lif_task import make_task


def _small(relaxed, t_ref=0.0, detach=False, seed=3):
    params = [-70.0, 250.0, 10.0, t_ref, -55.0, -70.0, 2.0, 2.0, 0.0]
    return make_task(n_exc=40, n_inh=10, n_in=20, batch=3, n_steps=120, relaxed=relaxed,
                     detach_reset=detach, params=params, w_in_scale=900.0, seed=seed)


def _loss(oracle, T, w=None, w_in=None):
    return oracle.lif_bptt(T["cfg"], T["row_ptr"], T["col"], T["w"] if w is None else w,
                           T["w_in"] if w_in is None else w_in, T["inputs"], T["targets"],
                           grad=False)[0]


def _fd_check(oracle, T, n=12, h=1e-3, rtol=1e-3):
    L, dw, dwi, nsp = oracle.lif_bptt(T["cfg"], T["row_ptr"], T["col"], T["w"], T["w_in"],
                                      T["inputs"], T["targets"])
    assert nsp > 0
    rng = np.random.default_rng(1)
    adj, fd = [], []
    for q in rng.choice(T["col"].size, n, replace=False):
        w = T["w"].copy()
        w[q] += h
        lp = _loss(oracle, T, w=w)
        w[q] -= 2 * h
        lm = _loss(oracle, T, w=w)
        adj.append(dw[q])
        fd.append((lp - lm) / (2 * h))
    for q in rng.choice(T["w_in"].size, n, replace=False):
        wi = T["w_in"].copy().reshape(-1)
        wi[q] += h
        lp = _loss(oracle, T, w_in=wi.reshape(T["w_in"].shape))
        wi[q] -= 2 * h
        lm = _loss(oracle, T, w_in=wi.reshape(T["w_in"].shape))
        adj.append(dwi.reshape(-1)[q])
        fd.append((lp - lm) / (2 * h))
    adj, fd = np.array(adj), np.array(fd)
    floor = 1e-3 * np.abs(fd).max()
    assert np.all(np.abs(adj - fd) <= rtol * np.maximum(np.abs(fd), floor)), (adj, fd)
    # a random direction over all weights, scaled by their magnitudes
    dirw = rng.standard_normal(T["w"].size) * np.abs(T["w"]).mean()
    diri = rng.standard_normal(T["w_in"].shape) * np.abs(T["w_in"]).mean()
    eps = 1e-4
    lp = _loss(oracle, T, w=T["w"] + eps * dirw, w_in=T["w_in"] + eps * diri)
    lm = _loss(oracle, T, w=T["w"] - eps * dirw, w_in=T["w_in"] - eps * diri)
    ad = float(np.sum(dw * dirw) + np.sum(dwi * diri))
    assert abs(ad - (lp - lm) / (2 * eps)) <= rtol * abs(ad)


def test_relaxed_adjoint_matches_finite_differences(oracle):
    _fd_check(oracle, _small(relaxed=True))


def test_relaxed_adjoint_matches_finite_differences_other_network(oracle):
    _fd_check(oracle, _small(relaxed=True, seed=8))


def test_hard_forward_surrogate_gradient_is_finite_and_nonzero(oracle):
    T = _small(relaxed=False, t_ref=2.0)
    L, dw, dwi, nsp = oracle.lif_bptt(T["cfg"], T["row_ptr"], T["col"], T["w"], T["w_in"],
                                      T["inputs"], T["targets"])
    assert nsp > 0 and np.isfinite(L)
    assert np.all(np.isfinite(dw)) and np.any(dw != 0) and np.any(dwi != 0)
    # detaching the reset changes the gradient, not the loss
    T2 = _small(relaxed=False, t_ref=2.0, detach=True)
    L2, dw2, _, _ = oracle.lif_bptt(T2["cfg"], T2["row_ptr"], T2["col"], T2["w"], T2["w_in"],
                                    T2["inputs"], T2["targets"])
    assert L2 == L and not np.array_equal(dw2, dw)
