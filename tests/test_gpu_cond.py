"""GPU parity of the per-step engine's iaf_cond_exp and iaf_cond_alpha
(adaptive RKF45, receptor ports g_ex / g_in) against the float64 oracle.

Tolerances: FP64 states within 2e-6, the reference test's own band for the
RKF45 trace (_nest_neuron/iaf_cond_alpha_test.py:319-325); spike rasters
identical; FP32 population rate within 5 % of the oracle.
"""
import numpy as np
import pytest

import brainpy.state_b200 as bs
from brainpy.state_b200 import _lib
from brainpy.state_b200.units import Hz, mV, ms, nS
from tests.netbuild import random_csr

pytestmark = pytest.mark.gpu

COND_ORDER = ("E_L", "C_m", "t_ref", "V_th", "V_reset", "E_ex", "E_in", "g_L", "tau_syn_ex",
              "tau_syn_in", "I_e", "gsl_error_tol")
COND = dict(E_L=-70.0, C_m=250.0, t_ref=2.0, V_th=-55.0, V_reset=-60.0, E_ex=0.0, E_in=-85.0,
            g_L=16.6667, tau_syn_ex=0.2, tau_syn_in=2.0, I_e=0.0, gsl_error_tol=1e-3)
DRIVE_NS = {"iaf_cond_exp": 4.0, "iaf_cond_alpha": 2.0}  # about 100 Hz in both models
NE, NI = 160, 40


def _net(target, is_plan, model, seed=4, K=(16, 4), w=(1.0, 3.0)):
    """Excitatory projections into receptor 0 (g_ex), inhibitory into 1 (g_in)."""
    rng = np.random.default_rng(seed)
    p = [COND[k] for k in COND_ORDER]
    add_proj = target.add_csr if is_plan else target.add_proj
    add_drive = target.add_poisson if is_plan else target.add_drive
    target.add_pop(NE, p)
    target.add_pop(NI, p)
    add_drive(0, 9000.0, DRIVE_NS[model], 5, 31, receptor=0)
    add_drive(1, 9000.0, DRIVE_NS[model], 5, 32, receptor=0)
    for pre, Kp, wp, rec in ((0, K[0], w[0], 0), (1, K[1], w[1], 1)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            indptr, idx, ww, d = random_csr(rng, n_pre, n_post, Kp, wp,
                                            rng.integers(5, 20, n_post * Kp))
            add_proj(pre, post, indptr, idx, ww, d, rec)
    return rng.uniform(-70.0, -55.0, NE + NI)


def _pair(oracle, model, precision, rec=None, **net):
    pl = _lib.Plan(0.1, model, precision=precision)
    v0 = _net(pl, True, model, **net)
    if rec is not None:
        pl.record_v(rec)
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    sim = oracle.OracleSim(0.1, model)
    _net(sim, False, model, **net)
    if rec is not None:
        sim.record_v(rec)
    sim.set_state(0, "V_m", v0[:NE])
    sim.set_state(1, "V_m", v0[NE:])
    return pl, sim


@pytest.mark.parametrize("model", ["iaf_cond_exp", "iaf_cond_alpha"])
def test_cond_network_fp64_matches_oracle(oracle, model):
    rec = np.arange(0, NE + NI, 3)
    pl, sim = _pair(oracle, model, 64, rec)
    pl.run(200)
    st, g = pl.spikes()
    ost, og, ov = sim.run(200)
    assert len(ost) > 0
    assert set(zip(st.tolist(), g.tolist())) == set(zip(ost.tolist(), og.tolist()))
    np.testing.assert_allclose(pl.v_trace(), ov, rtol=0, atol=2e-6)
    n_gpu, n_ref = pl.rk_substeps(), sim.rk_substeps
    assert n_ref >= (NE + NI) * 200
    assert abs(n_gpu - n_ref) <= 1e-3 * n_ref, (n_gpu, n_ref)
    names = ("g_ex", "g_in", "h") if model == "iaf_cond_exp" else ("dg_ex", "g_ex", "dg_in",
                                                                    "g_in", "h")
    for pop, n in ((0, NE), (1, NI)):
        for name in names:
            np.testing.assert_allclose(pl.get_state(pop, name), sim.get_state(pop, name, n),
                                       rtol=0, atol=2e-6, err_msg=name)
        np.testing.assert_array_equal(pl.get_state(pop, "r"), sim.get_state(pop, "r", n))


def test_static_rows_wider_than_one_work_item_match_oracle(oracle):
    """In-degrees of 120 excitatory and 80 inhibitory inputs: the I -> E rows
    average 80 * 160 / 40 = 320 edges per pre neuron, so static delivery
    splits them into two 256-edge work items."""
    model = "iaf_cond_alpha"
    pl, sim = _pair(oracle, model, 64, rec=np.arange(0, NE + NI, 7), K=(120, 80),
                    w=(16.0 / 120, 12.0 / 80))
    pl.run(200)
    st, g = pl.spikes()
    ost, og, ov = sim.run(200)
    assert len(ost) > 0
    assert set(zip(st.tolist(), g.tolist())) == set(zip(ost.tolist(), og.tolist()))
    np.testing.assert_allclose(pl.v_trace(), ov, rtol=0, atol=2e-6)


@pytest.mark.parametrize("model", ["iaf_cond_exp", "iaf_cond_alpha"])
def test_cond_fp32_rate_close_to_oracle(oracle, model):
    pl, sim = _pair(oracle, model, 32)
    pl.run(2000)
    st, _ = pl.spikes()
    ost, _, _ = sim.run(2000)
    assert len(ost) > 1000
    assert abs(len(st) - len(ost)) / len(ost) < 0.05


@pytest.mark.parametrize("model", [bs.iaf_cond_exp, bs.iaf_cond_alpha])
def test_cond_simulator_receptor_types(model):
    """Simulator facade: receptor_type 1 feeds g_ex and 2 feeds g_in; an
    excitatory input depolarises, the same input into receptor 2 hyperpolarises."""
    out = []
    for receptor in (1, 2):
        sim = bs.Simulator(dt=0.1 * ms)
        pop = sim.create(model, 2, params=dict(V_th=100.0 * mV))
        gen = sim.create(bs.poisson_generator, rate=20000.0 * Hz)
        sim.connect(gen, pop, weight=2.0 * nS, delay=0.1 * ms, receptor_type=receptor)
        vm = sim.create(bs.voltmeter)
        sim.connect(vm, pop)
        res = sim.simulate(20.0 * ms)
        out.append(res.trace(vm)[-1].mean())
    assert out[0] > -70.0 > out[1]
