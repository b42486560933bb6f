"""Host-side Simulator logic (no GPU): seeds, delays, validation."""
import numpy as np
import pytest

from brainpy.state_b200 import (Simulator, Uniform, all_to_all, fixed_indegree, iaf_psc_alpha,
                                iaf_psc_exp, poisson_generator, spike_recorder, stdp_synapse)
from brainpy.state_b200.units import Hz, mV, ms, pA
from tests.test_gpu_simulator import _build


def test_simulator_seed_derivation_matches_reference_formula():
    sim = Simulator(dt=0.1 * ms)
    _build(sim)
    seeds = [op[4] for op in sim._ops if op[0] == "fixed_indegree"]
    # connect(ne, ne+ni, seed=1): ordinals 2, 3; connect(ni, ne+ni, seed=2): 4, 5
    assert seeds == [(1 * 1_000_003 + 3) & 0x7FFFFFFF, (1 * 1_000_003 + 4) & 0x7FFFFFFF,
                     (2 * 1_000_003 + 5) & 0x7FFFFFFF, (2 * 1_000_003 + 6) & 0x7FFFFFFF]


def test_nest_delay_rounding():
    # _kernel/delays.py:85-86: [0.0, 0.04, 0.05, 0.15, 1.5] ms -> [0, 0, 1, 2, 15]
    sim = Simulator(dt=0.1 * ms)
    np.testing.assert_array_equal(sim._steps(np.array([0.0, 0.04, 0.05, 0.15, 1.5])),
                                  [0, 0, 1, 2, 15])


def test_validation():
    sim = Simulator(dt=0.1 * ms)
    with pytest.raises(TypeError):
        sim.create(iaf_psc_alpha, 3, params=dict(bogus=1.0))
    sim.create(iaf_psc_alpha, 3)
    with pytest.raises(NotImplementedError):
        sim.create(iaf_psc_exp, 3)
    with pytest.raises(ValueError):
        fixed_indegree(-1)
    with pytest.raises(ValueError):
        stdp_synapse(tau_plus=-1.0 * ms)
    nest = Simulator(dt=0.1 * ms, delivery="nest")
    a = nest.create(iaf_psc_alpha, 3)
    with pytest.raises(ValueError, match="delays"):
        nest.connect(a, a, weight=1.0 * pA, delay=0.0 * ms, rule=all_to_all)


def test_distributed_weights_follow_the_reference_k_w_stream(oracle):
    """connect(weight=Uniform(...), rule=fixed_indegree(K), seed=s): the
    reference draws the weights from k_w = split(key(derived seed), 3)[1] in
    the sampler's post-major edge order, as low + (high - low) * uniform01 in
    float32, and sorts them into CSR order with the edges
    (_nest_network/event_proj.py:147-149, 286-291; _dist.py:66-77).  The
    realised CSR weights must equal the oracle's restatement bit for bit."""
    from brainpy.state_b200.units import pA
    sim = Simulator(dt=0.1 * ms)
    a = sim.create(iaf_psc_alpha, 120)
    sim.connect(a, a, weight=Uniform(10.0 * pA, 30.0 * pA), delay=1.5 * ms,
                rule=fixed_indegree(9), seed=5)
    pl = sim._build(upload=False)
    indptr, post, _, w = pl.csr(0)
    pseed = (5 * 1_000_003 + 0 + 1) & 0x7FFFFFFF
    pre_o, post_o = oracle.fixed_indegree(pseed, 120, 120, 9, pre_is_post=True,
                                          allow_autapses=True)
    order, idx, iptr = oracle.csr_structure(pre_o, post_o, 120)
    k_w = oracle.jax_fold_in(oracle.jax_key(pseed), 1)
    u = oracle.jax_uniform(k_w, pre_o.size, 32, 0.0, 1.0).astype(np.float32)
    w_draw = np.float32(10.0) + np.float32(20.0) * u
    np.testing.assert_array_equal(iptr, indptr)
    np.testing.assert_array_equal(idx, post)
    np.testing.assert_array_equal(w, w_draw[order].astype(np.float64))
