"""CPU checks of the oracle's iaf_psc_exp_multisynapse step (the checker of the
GPU per-step engine's multisynapse model), pinned to the reference's
analytical test (_nest_neuron/iaf_psc_exp_multisynapse_test.py:65-137), and
of the library's parameter and receptor validation (host code, no GPU)."""
import numpy as np
import pytest

from brainpy.state_b200 import _lib

ALPHA = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -np.inf]


def _ms_params(tau_syn, E_L=-70.0, C_m=250.0, tau_m=10.0, t_ref=2.0, V_th=-55.0, V_reset=-70.0,
               I_e=0.0):
    return [E_L, C_m, tau_m, t_ref, V_th, V_reset, I_e, float(len(tau_syn))] + list(tau_syn)


def test_multisynapse_matches_closed_form_psc_and_psp(oracle):
    # four receptors, one spike each at its own time; the exact integration
    # must follow the closed-form current and membrane responses
    tau_syns = np.array([2.0, 20.0, 60.0, 100.0])
    delays = np.array([7.0, 5.0, 2.0, 1.0])
    weights = np.array([30.0, 50.0, 20.0, 10.0])
    c_m, tau_m, spike_time, dt = 250.0, 15.0, 0.1, 0.1
    sim = oracle.OracleSim(dt, "iaf_psc_exp_multisynapse")
    sim.add_pop(1, _ms_params(tau_syns, E_L=0.0, C_m=c_m, tau_m=tau_m, V_th=1500.0,
                              V_reset=0.0))
    sim.set_state(0, "V_m", [0.0])
    steps = 80
    w_step = np.zeros((steps, 4))
    for r, (d, w) in enumerate(zip(delays, weights)):
        # an on-grid event at time T acts in the step that ends at T
        w_step[int(round((spike_time + d - dt) / dt)), r] += w
    i_syn, v = np.zeros((steps, 4)), np.zeros(steps)
    for k in range(steps):
        sim.step_neuron_ms(0, w_step[k])
        i_syn[k] = [sim.get_state(0, f"i_syn_{r}", 1)[0] for r in range(4)]
        v[k] = sim.get_state(0, "V_m", 1)[0]
    t = (np.arange(steps) + 1) * dt
    i_ref = np.zeros((steps, 4))
    v_ref = np.zeros(steps)
    for r, (w, d, ts) in enumerate(zip(weights, delays, tau_syns)):
        s = t - d - spike_time
        m = s > 0
        i_ref[m, r] = w * np.exp(-s[m] / ts)
        v_ref[m] += w / (c_m * (1.0 / ts - 1.0 / tau_m)) * (np.exp(-s[m] / tau_m)
                                                             - np.exp(-s[m] / ts))
    np.testing.assert_allclose(i_syn, i_ref, atol=2e-10, rtol=1e-10)
    np.testing.assert_allclose(v, v_ref, atol=5e-10, rtol=1e-10)


def test_multisynapse_refractory_and_reset(oracle):
    # a large current on receptor 1 fires the neuron, which is then held at
    # V_reset for ceil(t_ref / dt) = 3 steps before it integrates again
    sim = oracle.OracleSim(0.1, "iaf_psc_exp_multisynapse")
    sim.add_pop(1, _ms_params([2.0, 5.0], t_ref=0.3))
    sim.set_state(0, "V_m", [-70.0])
    spikes, v = [], []
    for k in range(12):
        spikes.append(bool(sim.step_neuron_ms(0, [0.0, 40000.0] if k == 0 else [0.0, 0.0])))
        v.append(sim.get_state(0, "V_m", 1)[0])
    first = spikes.index(True)
    assert v[first] == -70.0
    for k in range(first + 1, first + 4):
        assert not spikes[k] and v[k] == -70.0
    assert v[first + 4] > -70.0


def test_multisynapse_validation_errors_match_reference_messages():
    # iaf_psc_exp_multisynapse.py:463-477
    pl = _lib.Plan(0.1, "iaf_psc_exp_multisynapse")
    with pytest.raises(ValueError, match="Membrane and synapse time constants must differ"):
        pl.add_pop(2, _ms_params([2.0, 10.0], tau_m=10.0))
    with pytest.raises(ValueError, match="All synaptic time constants must be strictly positive"):
        pl.add_pop(2, _ms_params([-1.0]))
    with pytest.raises(ValueError, match="Capacitance must be > 0"):
        pl.add_pop(2, _ms_params([2.0], C_m=0.0))
    with pytest.raises(ValueError, match="Reset potential must be smaller than threshold"):
        pl.add_pop(2, _ms_params([2.0], V_reset=-50.0))
    with pytest.raises(NotImplementedError, match="n_receptors"):
        pl.add_pop(2, _ms_params([1.0, 2.0, 3.0, 4.0, 5.0]))
    a = pl.add_pop(2, _ms_params([2.0, 8.0]))
    ip, post = np.array([0, 1, 2]), np.array([1, 0], np.int32)
    pl.add_csr(a, a, ip, post, np.ones(2), np.full(2, 5, np.int32), receptor=1)
    with pytest.raises(ValueError, match="n_receptors"):
        pl.add_csr(a, a, ip, post, np.ones(2), np.full(2, 5, np.int32), receptor=2)
    # the current models still sum every input into one port
    pl2 = _lib.Plan(0.1)
    b = pl2.add_pop(2, ALPHA)
    with pytest.raises(ValueError, match="receptor ports"):
        pl2.add_csr(b, b, ip, post, np.ones(2), np.full(2, 5, np.int32), receptor=1)
