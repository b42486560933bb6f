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
