"""The public Simulator API end to end on the GPU, against the oracle built
from the same description (the reference Brunel script's structure)."""
import math

import numpy as np
import pytest

from brainpy.state_b200 import (Simulator, Uniform, all_to_all, fixed_indegree, iaf_psc_alpha,
                                poisson_generator, spike_recorder, voltmeter)
from brainpy.state_b200.units import Hz, mV, ms, pA, pF

pytestmark = pytest.mark.gpu


def _build(sim, NE=400, NI=100, CE=40, CI=10, J=20.68, rate=17789.0):
    npar = dict(C_m=250.0 * pF, tau_m=20.0 * ms, tau_syn_ex=0.5 * ms, tau_syn_in=0.5 * ms,
                t_ref=2.0 * ms, E_L=0.0 * mV, V_reset=10.0 * mV, V_th=20.0 * mV,
                V_initializer=Uniform(0.0 * mV, 20.0 * mV))
    ne = sim.create(iaf_psc_alpha, NE, params=npar)
    ni = sim.create(iaf_psc_alpha, NI, params=npar)
    noise = sim.create(poisson_generator, rate=rate * Hz)
    esr = sim.create(spike_recorder)
    vm = sim.create(voltmeter)
    sim.connect(noise, ne, weight=J * pA, delay=1.5 * ms, rule=all_to_all)
    sim.connect(noise, ni, weight=J * pA, delay=1.5 * ms, rule=all_to_all)
    sim.connect(ne, ne + ni, weight=J * pA, delay=1.5 * ms, rule=fixed_indegree(CE), seed=1)
    sim.connect(ni, ne + ni, weight=-5 * J * pA, delay=1.5 * ms, rule=fixed_indegree(CI), seed=2)
    sim.connect(ne[:50], esr)
    sim.connect(vm, ne[:20])
    return esr, vm


def _oracle_twin(oracle, sim, NE=400, NI=100):
    pl = sim._plan
    o = oracle.OracleSim(0.1)
    for p in sim._pops:
        o.add_pop(p.n, p.params)
    for op in sim._ops:
        if op[0] == "drive":
            _, pop, rate, w, d, seed, tmin, tmax, rec = op
            o.add_drive(pop, rate, w, d, seed, tmin, tmax)
    for j in range(4):
        indptr, post, d, w = pl.csr(j)
        pre = 0 if j < 2 else 1
        post_pop = j % 2
        o.add_proj(pre, post_pop, indptr, post, w, d)
    return o


def test_simulator_exact_fp64_matches_oracle(oracle):
    sim = Simulator(dt=0.1 * ms, precision=64, deterministic=True)
    esr, vm = _build(sim)
    res = sim.simulate(200.0 * ms)
    assert res.spikes(esr).shape == (2000, 50)
    o = _oracle_twin(oracle, sim)
    o.set_state(0, "V_m", _init_v(sim, 0))
    o.set_state(1, "V_m", _init_v(sim, 1))
    o.record_v(np.arange(20))
    st, g, v = o.run(2000)
    sel = g < 50
    mat = np.zeros((2000, 50))
    mat[st[sel], g[sel]] = 1.0
    np.testing.assert_array_equal(res.spikes(esr), mat)
    np.testing.assert_array_equal(res.trace(vm), v)
    assert res.rate(esr) > 1.0
    # simulate() re-initialises: a second call reproduces the first exactly
    res2 = sim.simulate(200.0 * ms)
    np.testing.assert_array_equal(res2.spikes(esr), res.spikes(esr))
    # cont() continues from the current state
    res3 = sim.cont(100.0 * ms)
    assert res3.times[0] == pytest.approx(200.0)


def _init_v(sim, pop_id):
    return sim.initial_v(pop_id)
