"""CPU checks of the oracle's stdp_triplet_synapse rule (the checker of the GPU
per-step engine's triplet kernels), restating the reference's rule tests
(_nest_plasticity/stdp_triplet_synapse_rule_test.py:79-158), and of the
host-side spec and attach validation."""
import numpy as np
import pytest

import brainpy.state_b200 as bs
from brainpy.state_b200 import _lib

DEF = dict(Aplus=5e-10, Aplus_triplet=0.0062, Aminus=0.007, Aminus_triplet=0.00023, Wmax=100.0)


def _upd(oracle, w, pre_s, post_s, r, o, **kw):
    p = dict(DEF, **kw)
    return oracle.triplet_update(w, pre_s, post_s, r, o, p["Aplus"], p["Aplus_triplet"],
                                 p["Aminus"], p["Aminus_triplet"], p["Wmax"])


def test_post_spike_potentiates_with_triplet_term(oracle):
    # traces fed with this step's own spike: o = (1.3, 1.4) -> excluded (0.3, 0.4)
    w = _upd(oracle, 5.0, 0.0, 1.0, (0.6, 0.2), (1.3, 1.4), Aplus=0.001, Aplus_triplet=0.01)
    assert w == pytest.approx(5.0 + 0.6 * (0.001 + 0.01 * 0.4), abs=1e-15)
    assert w > 5.0


def test_triplet_term_distinct_from_pair(oracle):
    lo = _upd(oracle, 5.0, 0.0, 1.0, (0.6, 0.0), (1.0, 1.1), Aplus=0.001, Aplus_triplet=0.01)
    hi = _upd(oracle, 5.0, 0.0, 1.0, (0.6, 0.0), (1.0, 1.9), Aplus=0.001, Aplus_triplet=0.01)
    assert hi > lo


def test_pre_spike_depresses_with_triplet_term(oracle):
    w = _upd(oracle, 5.0, 1.0, 0.0, (0.2, 1.3), (0.5, 0.1), Aminus=0.01, Aminus_triplet=0.02)
    assert w == pytest.approx(5.0 - 0.5 * (0.01 + 0.02 * 0.3), abs=1e-15)
    assert w < 5.0


def test_clamps(oracle):
    assert _upd(oracle, 99.5, 0.0, 1.0, (5.0, 0.0), (1.0, 5.0), Aplus=1.0,
                Aplus_triplet=1.0) == 100.0
    assert _upd(oracle, 0.2, 1.0, 0.0, (1.0, 5.0), (5.0, 0.0), Aminus=1.0,
                Aminus_triplet=1.0) == 0.0


def test_simultaneous_spikes_exclude_the_current_step(oracle):
    kw = dict(Aplus=0.01, Aplus_triplet=0.02, Aminus=0.01, Aminus_triplet=0.02)
    assert _upd(oracle, 5.0, 1.0, 1.0, (1.0, 1.0), (1.0, 1.0), **kw) == 5.0
    assert _upd(oracle, 5.0, 0.0, 0.0, (0.7, 0.7), (0.7, 0.7), Aplus=0.01, Aminus=0.01) == 5.0


def test_post_then_pre_order_on_coincident_step(oracle):
    # potentiation first: 5 + 1 * 0.01 = 5.01; then depression: 5.01 - 1 * 0.01
    w = _upd(oracle, 5.0, 1.0, 1.0, (2.0, 1.0), (2.0, 1.0), Aplus=0.01, Aplus_triplet=0.0,
             Aminus=0.01, Aminus_triplet=0.0)
    assert w == pytest.approx(5.0, abs=1e-15)


def test_spec_defaults_and_validation():
    # stdp_triplet_synapse_rule_test.py:57-78
    s = bs.stdp_triplet_synapse()
    assert [s.taus[k] for k in ("tau_plus", "tau_plus_triplet")] == [16.8, 101.0]
    assert [s.taus[k] for k in ("tau_minus", "tau_minus_triplet")] == [20.0, 110.0]
    assert (s.Aplus, s.Aplus_triplet, s.Aminus, s.Aminus_triplet) == (5e-10, 0.0062, 0.007,
                                                                      0.00023)
    assert s.Wmax == 100.0
    for kw in (dict(tau_plus=0.0), dict(tau_plus_triplet=-1.0), dict(tau_minus=0.0),
               dict(tau_minus_triplet=-1.0)):
        with pytest.raises(ValueError):
            bs.stdp_triplet_synapse(**kw)
    assert isinstance(bs.stdp_synapse_hom(), bs.stdp_synapse)


def test_library_attach_validation():
    pl = _lib.Plan(0.1)
    a = pl.add_pop(3, [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -np.inf])
    j = pl.add_csr(a, a, np.array([0, 1, 2, 3]), np.array([1, 2, 0], np.int32), np.ones(3),
                   np.full(3, 5, np.int32))
    with pytest.raises(ValueError, match="'tau_minus_triplet' must be > 0"):
        pl.attach_stdp_triplet(j, tau_minus_triplet=0.0)
    k = pl.add_csr(a, a, np.array([0, 1, 2, 3]), np.array([1, 2, 0], np.int32), np.ones(3),
                   np.array([5, 6, 5], np.int32))
    with pytest.raises(NotImplementedError, match="homogeneous delay"):
        pl.attach_stdp_triplet(k)
    pl.attach_stdp_triplet(j)
