"""GPU parity of the per-step engine's iaf_psc_exp_multisynapse (one input
channel per receptor, each with its own synaptic time constant) against the
float64 oracle.

Tolerances: FP64 spike rasters identical and states within 1e-9 (exact
propagators; the GPU contracts multiply-adds, the oracle does not); FP32
population rate within 5 % of the oracle.
"""
import numpy as np
import pytest

import brainpy.state_b200 as bs
from brainpy.state_b200 import _lib
from brainpy.state_b200.units import Hz, mV, ms, pA
from tests.netbuild import random_csr

pytestmark = pytest.mark.gpu

# E_L C_m tau_m t_ref V_th V_reset I_e n_receptors tau_syn[3]
PARAMS = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.0, 3.0, 0.5, 2.0, 5.0]
NE, NI = 200, 50


def _net(target, is_plan, seed=6):
    """Drive into receptor 0, excitation into 1, inhibition (negative) into 2."""
    rng = np.random.default_rng(seed)
    target.add_pop(NE, PARAMS)
    target.add_pop(NI, PARAMS)
    add_drive = target.add_poisson if is_plan else target.add_drive
    add_proj = target.add_csr if is_plan else target.add_proj
    add_drive(0, 17789.0, 35.0, 15, 5, receptor=0)
    add_drive(1, 17789.0, 35.0, 15, 6, receptor=0)
    for pre, K, w, rec in ((0, 20, 0.4 * 20.68, 1), (1, 5, -2.0 * 20.68, 2)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            indptr, idx, ww, d = random_csr(rng, n_pre, n_post, K, w,
                                            rng.integers(10, 25, n_post * K))
            add_proj(pre, post, indptr, idx, ww, d, rec)
    return rng.uniform(0.0, 20.0, NE + NI)


def _pair(oracle, precision, rec=None):
    pl = _lib.Plan(0.1, "iaf_psc_exp_multisynapse", precision=precision)
    v0 = _net(pl, True)
    if rec is not None:
        pl.record_v(rec)
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    sim = oracle.OracleSim(0.1, "iaf_psc_exp_multisynapse")
    _net(sim, False)
    if rec is not None:
        sim.record_v(rec)
    sim.set_state(0, "V_m", v0[:NE])
    sim.set_state(1, "V_m", v0[NE:])
    return pl, sim


def test_multisynapse_network_fp64_matches_oracle(oracle):
    rec = np.arange(0, NE + NI, 4)
    pl, sim = _pair(oracle, 64, rec)
    pl.run(600)
    st, g = pl.spikes()
    ost, og, ov = sim.run(600)
    assert len(ost) > 50
    assert set(zip(st.tolist(), g.tolist())) == set(zip(ost.tolist(), og.tolist()))
    np.testing.assert_allclose(pl.v_trace(), ov, rtol=0, atol=1e-9)
    for pop, n in ((0, NE), (1, NI)):
        for k in range(3):
            np.testing.assert_allclose(pl.get_state(pop, f"i_syn_{k}"),
                                       sim.get_state(pop, f"i_syn_{k}", n), rtol=0, atol=1e-9)
        np.testing.assert_array_equal(pl.get_state(pop, "r"), sim.get_state(pop, "r", n))


def test_multisynapse_fp32_rate_close_to_oracle(oracle):
    pl, sim = _pair(oracle, 32)
    pl.run(3000)
    st, _ = pl.spikes()
    ost, _, _ = sim.run(3000)
    assert len(ost) > 1000
    assert abs(len(st) - len(ost)) / len(ost) < 0.05


def test_multisynapse_simulator_receptor_ports():
    """Simulator facade: the same input into receptor 1 (tau_syn 0.5 ms) and
    receptor 2 (tau_syn 20 ms) carries the same charge per spike in the
    second case 40 times longer, so the slow port depolarises more."""
    out = []
    for receptor in (1, 2):
        sim = bs.Simulator(dt=0.1 * ms)
        pop = sim.create(bs.iaf_psc_exp_multisynapse, 2,
                         params=dict(V_th=100.0 * mV, tau_syn=(0.5, 20.0)))
        gen = sim.create(bs.poisson_generator, rate=5000.0 * Hz)
        sim.connect(gen, pop, weight=5.0 * pA, delay=0.1 * ms, receptor_type=receptor)
        vm = sim.create(bs.voltmeter)
        sim.connect(vm, pop)
        res = sim.simulate(20.0 * ms)
        out.append(res.trace(vm)[-1].mean())
    assert out[1] > out[0] > -70.0
