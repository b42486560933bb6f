"""The windowed form of the per-step engine against the per-step form and the
float64 oracle.

The windowed form advances W = min(lag, 32, 64 - max lag) steps per launch
sequence and brings each plastic weight up to date at its arrivals; it does
the same floating-point operations on every weight and trace as the per-step
form, so FP64 weights agree to 1e-12 relative and rasters are identical.  The
conductance and current inputs are summed in another order (atomics into the
ring against per-thread sums), hence V_m within 1e-9 mV (iaf) and RKF45
states within 2e-6 (the aeif parity band of the reference's own test).
"""
import math

import numpy as np
import pytest

from brainpy.state_b200 import _lib
from tests.netbuild import random_csr

pytestmark = pytest.mark.gpu

IAF = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]


def _stdp_plan(NE=200, NI=50, KE=20, KI=5, J=20.68, seed=9, delay=15, windowed=True,
               precision=64, semantics=_lib.LEGACY):
    rng = np.random.default_rng(seed)
    pieces = []
    for pre, K, w in ((0, KE, J), (1, KI, -5.0 * J)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            pieces.append((pre, post) + random_csr(rng, n_pre, n_post, K, w, delay))
    v0 = rng.uniform(0.0, 20.0, NE + NI)
    pl = _lib.Plan(0.1, precision=precision, semantics=semantics)
    pl.add_pop(NE, IAF)
    pl.add_pop(NI, IAF)
    pl.add_poisson(0, 17789.0, 20.68, delay, 5)
    pl.add_poisson(1, 17789.0, 20.68, delay, 6)
    ids = [pl.add_csr(pre, post, indptr, idx, w, d) for pre, post, indptr, idx, w, d in pieces]
    pl.attach_stdp(ids[0], 20.0, 20.0, 0.05, 1.0, 1.0, 1.0, 3 * J)
    rec = np.arange(0, NE + NI, 5)
    pl.record_v(rec)
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    if not windowed:
        pl.set_windowed(False)
    return pl, ids


def _raster(pl):
    st, g = pl.spikes()
    return set(zip(st.tolist(), g.tolist()))


def test_windowed_stdp_matches_per_step_over_uneven_runs():
    win, ids = _stdp_plan()
    ref, _ = _stdp_plan(windowed=False)
    assert win.engine == "windowed" and ref.engine == "per_step"
    # windows restart at every run: runs of 37 and 88 steps end in partial
    # windows (W = 15)
    win.run(37)
    r1, v1 = _raster(win), win.v_trace()
    win.run(88)
    r2, v2 = _raster(win), win.v_trace()
    ref.run(125)
    assert len(_raster(ref)) > 50
    # spike lists hold the last run's spikes
    assert r1 | r2 == _raster(ref)
    np.testing.assert_allclose(np.concatenate([v1, v2]), ref.v_trace(), rtol=0, atol=1e-9)
    w_ref = ref.weights(ids[0])
    assert np.any(w_ref != 20.68)
    np.testing.assert_allclose(win.weights(ids[0]), w_ref, rtol=1e-12, atol=0)


def test_windowed_stdp_with_heavy_rows_matches_per_step():
    # in-degrees of about 300 plastic edges and a high rate: many arrivals per
    # (step, post) list and several own spikes owed to each edge per window
    kw = dict(NE=320, NI=80, KE=300, KI=75, J=20.68 * 20 / 300, seed=12, delay=12)
    win, ids = _stdp_plan(**kw)
    ref, _ = _stdp_plan(windowed=False, **kw)
    win.run(300)
    ref.run(300)
    assert _raster(win) == _raster(ref)
    np.testing.assert_allclose(win.weights(ids[0]), ref.weights(ids[0]), rtol=1e-12, atol=0)
    np.testing.assert_allclose(win.v_trace(), ref.v_trace(), rtol=0, atol=1e-9)


def test_weight_recording_runs_per_step_forms_and_agrees():
    win, ids = _stdp_plan()
    win.record_weights(ids[0])
    win.run(60)
    tr = win.weight_trace(ids[0])
    assert tr.shape[0] == 60
    np.testing.assert_array_equal(tr[-1], win.weights(ids[0]))
    ref, _ = _stdp_plan(windowed=False)
    ref.run(60)
    np.testing.assert_allclose(tr[-1], ref.weights(ids[0]), rtol=1e-12, atol=0)


def test_short_lags_stay_per_step():
    # kernel timing: a delay of one step is a lag of one step (W would be 1)
    pl, _ = _stdp_plan(delay=1, semantics=_lib.RING)
    assert pl.engine == "per_step"
    with pytest.raises(NotImplementedError):
        pl.set_windowed(True)


AEIF = [0.0, -60.0, 0.0, 30.0, 281.0, 0.0, -85.0, -70.6, 2.0, 144.0, 4.0, 80.5, -50.4, 0.2,
        2.0, 0.0, 1e-6]


def _aeif_plan(windowed, precision=64, seed=4):
    rng = np.random.default_rng(seed)
    NE, NI = 160, 40
    pl = _lib.Plan(0.1, "aeif_cond_alpha", precision=precision)
    pl.add_pop(NE, AEIF)
    pl.add_pop(NI, AEIF)
    pl.add_poisson(0, 9000.0, 3.0, 5, 31, receptor=0)
    pl.add_poisson(1, 9000.0, 3.0, 5, 32, receptor=0)
    for pre, K, w, rc in ((0, 16, 0.8, 0), (1, 4, 2.5, 1)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            indptr, idx, ww, d = random_csr(rng, n_pre, n_post, K, w,
                                            rng.integers(5, 20, n_post * K))
            pl.add_csr(pre, post, indptr, idx, ww, d, rc)
    v0 = rng.uniform(-70.0, -55.0, NE + NI)
    pl.record_v(np.arange(0, 200, 3))
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    if not windowed:
        pl.set_windowed(False)
    return pl


def test_windowed_aeif_matches_per_step():
    win = _aeif_plan(True)
    ref = _aeif_plan(False)
    assert win.engine == "windowed"  # lags 5..19: W = 5
    win.run(150)
    ref.run(150)
    assert len(_raster(ref)) > 0
    assert _raster(win) == _raster(ref)
    np.testing.assert_allclose(win.v_trace(), ref.v_trace(), rtol=0, atol=2e-6)
    for name in ("w", "g_ex", "g_in"):
        np.testing.assert_allclose(win.get_state(0, name), ref.get_state(0, name), rtol=0, atol=2e-6)
    # the same integrator work, up to acceptances moved at the margin by the
    # input summation order
    n_w, n_r = win.rk_substeps(), ref.rk_substeps()
    assert abs(n_w - n_r) <= 1e-3 * n_r, (n_w, n_r)



def _aeif_stdp_plan(windowed, seed=21):
    """AdEx network with a plastic E->E projection (lag 21 steps; the others
    21-26) and W = 21: posts fire inside windows that still bring them
    arrivals, and the strong drive makes some pres fire twice within one
    window (edges with two arrivals in a window)."""
    rng = np.random.default_rng(seed)
    NE, NI = 160, 40
    pl = _lib.Plan(0.1, "aeif_cond_alpha", precision=64)
    pl.add_pop(NE, AEIF)
    pl.add_pop(NI, AEIF)
    pl.add_poisson(0, 12000.0, 3.5, 5, 31, receptor=0)
    pl.add_poisson(1, 12000.0, 3.5, 5, 32, receptor=0)
    ids = []
    for pre, K, w, rc in ((0, 16, 0.8, 0), (1, 4, 2.5, 1)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            d = 20 if (pre, post) == (0, 0) else rng.integers(20, 26, n_post * K)
            indptr, idx, ww, dd = random_csr(rng, n_pre, n_post, K, w, d)
            ids.append(pl.add_csr(pre, post, indptr, idx, ww, dd, rc))
    pl.attach_stdp(ids[0], 20.0, 20.0, 0.05, 1.0, 1.0, 1.0, 2.4)
    v0 = rng.uniform(-65.0, -52.0, NE + NI)
    pl.record_v(np.arange(0, 200, 3))
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    if not windowed:
        pl.set_windowed(False)
    return pl, ids


def test_windowed_aeif_stdp_matches_per_step():
    """RKF45 neurons with a plastic projection: the windowed form against the
    per-step form, identical rasters and FP64 weights, states within the
    reordered input sums."""
    win, ids = _aeif_stdp_plan(True)
    ref, _ = _aeif_stdp_plan(False)
    assert win.engine == "windowed"
    for n in (140, 230):  # runs end inside windows
        win.run(n)
        ref.run(n)
    r = _raster(ref)
    assert len(r) > 300
    assert _raster(win) == r
    np.testing.assert_allclose(win.weights(ids[0]), ref.weights(ids[0]), rtol=1e-12, atol=0)
    np.testing.assert_allclose(win.v_trace(), ref.v_trace(), rtol=0, atol=2e-6)
    for name in ("w", "g_ex", "g_in"):
        np.testing.assert_allclose(win.get_state(0, name), ref.get_state(0, name), rtol=0, atol=2e-6)
    n_w, n_r = win.rk_substeps(), ref.rk_substeps()
    assert abs(n_w - n_r) <= 1e-3 * n_r, (n_w, n_r)
