"""CPU checks of the oracle's iaf_cond_exp and iaf_cond_alpha steps (the
checker of the GPU per-step engine's conductance models), pinned to the
reference's own known-answer tests (_nest_neuron/iaf_cond_exp_test.py,
_nest_neuron/iaf_cond_alpha_test.py), and of the library's parameter
validation for both models (host code, no GPU)."""
import math

import numpy as np
import pytest

from brainpy.state_b200 import _lib

COND_ORDER = ("E_L", "C_m", "t_ref", "V_th", "V_reset", "E_ex", "E_in", "g_L", "tau_syn_ex",
              "tau_syn_in", "I_e", "gsl_error_tol")
# NEST defaults (iaf_cond_exp.py:295-318, iaf_cond_alpha.py:307-329)
COND_DEFAULTS = dict(E_L=-70.0, C_m=250.0, t_ref=2.0, V_th=-55.0, V_reset=-60.0, E_ex=0.0,
                     E_in=-85.0, g_L=16.6667, tau_syn_ex=0.2, tau_syn_in=2.0, I_e=0.0,
                     gsl_error_tol=1e-3)


def _params(**kw):
    d = dict(COND_DEFAULTS, **kw)
    return [d[k] for k in COND_ORDER]


def _sim(oracle, model, v0, **kw):
    sim = oracle.OracleSim(0.1, model)
    sim.add_pop(1, _params(**kw))
    sim.set_state(0, "V_m", [v0])
    return sim


# Fehlberg 4(5): stage coefficients, 5th- and 4th-order weights
_A = [[], [1 / 4], [3 / 32, 9 / 32], [1932 / 2197, -7200 / 2197, 7296 / 2197],
      [439 / 216, -8.0, 3680 / 513, -845 / 4104], [-8 / 27, 2.0, -3544 / 2565, 1859 / 4104, -11 / 40]]
_B5 = [16 / 135, 0.0, 6656 / 12825, 28561 / 56430, -9 / 50, 2 / 55]
_B4 = [25 / 216, 0.0, 1408 / 2565, 2197 / 4104, -1 / 5, 0.0]


def _rhs(model, y, refr, i_stim, p):
    if model == "iaf_cond_exp":
        v, ge, gi = y
        dge, dgi = -ge / p["tau_syn_ex"], -gi / p["tau_syn_in"]
    else:
        v, dex, ge, din, gi = y
    if refr:
        dv = 0.0
    else:
        ve = min(v, p["V_th"])
        dv = (-p["g_L"] * (ve - p["E_L"]) + i_stim + p["I_e"] - ge * (ve - p["E_ex"])
              - gi * (ve - p["E_in"])) / p["C_m"]
    if model == "iaf_cond_exp":
        return np.array([dv, dge, dgi])
    return np.array([dv, -dex / p["tau_syn_ex"], dex - ge / p["tau_syn_ex"],
                     -din / p["tau_syn_in"], din - gi / p["tau_syn_in"]])


def _rkf45_dt(model, y, refr, i_stim, dt, h, p, atol=1e-3):
    """The tests' scalar RKF45 over one dt (iaf_cond_exp_test.py:17-97,
    iaf_cond_alpha_test.py:34-87): absolute max-norm error against atol, the
    refractory flag fixed for the whole step, step growth 0.9 (atol/err)^(1/5)
    in [0.2, 5] and shrink 0.9 (atol/err)^(1/4) in [0.2, 1]."""
    min_h, t = 1e-8, 0.0
    h = max(h, min_h)
    y = np.array(y, dtype=np.float64)
    while t < dt:
        h = max(min_h, min(h, dt - t))
        k = []
        for s in range(6):
            ys = y + h * sum(a * kk for a, kk in zip(_A[s], k)) if s else y
            k.append(_rhs(model, ys, refr, i_stim, p))
        y5 = y + h * sum(b * kk for b, kk in zip(_B5, k))
        y4 = y + h * sum(b * kk for b, kk in zip(_B4, k))
        err = float(np.max(np.abs(y5 - y4)))
        if err <= atol or h <= min_h:
            y = y5
            t += h
            fac = 5.0 if err == 0.0 else min(5.0, max(0.2, 0.9 * (atol / err) ** 0.2))
        else:
            fac = min(1.0, max(0.2, 0.9 * (atol / err) ** 0.25))
        h = max(min_h, h * fac)
    return y, h


# ------------------------------------------------------------- iaf_cond_exp

def test_cond_exp_current_input_has_one_step_delay(oracle):
    # iaf_cond_exp_test.py:170-185: 100 pA for one step on 250 pF -> 0.04 mV
    sim = _sim(oracle, "iaf_cond_exp", 0.0, E_L=0.0, g_L=0.0, I_e=0.0, V_th=1e9, V_reset=0.0)
    sim.step_neuron(0, x_next=100.0)
    assert abs(sim.get_state(0, "V_m", 1)[0]) < 1e-12
    sim.step_neuron(0, x_next=0.0)
    assert sim.get_state(0, "V_m", 1)[0] == pytest.approx(0.04, abs=1e-9)


def test_cond_exp_refractory_countdown_and_spike_timing(oracle):
    # iaf_cond_exp_test.py:207-233: spike, three refractory steps, spike
    sim = _sim(oracle, "iaf_cond_exp", 0.0, E_L=0.0, g_L=0.0, C_m=250.0, I_e=10000.0,
               V_th=1.0, V_reset=0.0, t_ref=0.25)
    spikes = [bool(sim.step_neuron(0)) for _ in range(5)]
    assert spikes == [True, False, False, False, True]


def test_cond_signed_weights_split_into_ex_and_in(oracle):
    # iaf_cond_exp_test.py:158-168 and iaf_cond_alpha_test.py:201-221
    sim = _sim(oracle, "iaf_cond_exp", -70.0, V_th=100.0)
    sim.step_neuron(0, w0=5.0, w1=3.0)
    assert sim.get_state(0, "g_ex", 1)[0] == pytest.approx(5.0, abs=1e-12)
    sim_in = sim.get_state(0, "g_in", 1)[0]
    assert sim_in == pytest.approx(3.0, abs=1e-12)
    sim = _sim(oracle, "iaf_cond_alpha", -70.0, V_th=1000.0)
    sim.step_neuron(0, w0=5.0, w1=3.0)
    assert sim.get_state(0, "dg_ex", 1)[0] == pytest.approx(math.e / 0.2 * 5.0, abs=1e-12)
    assert sim.get_state(0, "dg_in", 1)[0] == pytest.approx(math.e / 2.0 * 3.0, abs=1e-12)
    assert sim.get_state(0, "g_ex", 1)[0] == 0.0 and sim.get_state(0, "g_in", 1)[0] == 0.0
    sim.step_neuron(0)
    assert sim.get_state(0, "g_ex", 1)[0] > 0.0 and sim.get_state(0, "g_in", 1)[0] > 0.0


@pytest.mark.parametrize("model", ["iaf_cond_exp", "iaf_cond_alpha"])
def test_cond_excitation_raises_and_inhibition_lowers_v(oracle, model):
    # iaf_cond_exp_test.py:187-205
    out = []
    for w0, w1 in ((0.0, 0.0), (5.0, 0.0), (0.0, 5.0)):
        sim = _sim(oracle, model, -70.0, V_th=100.0)
        sim.step_neuron(0, w0=w0, w1=w1)
        sim.step_neuron(0)
        if model == "iaf_cond_alpha":
            sim.step_neuron(0)
        out.append(sim.get_state(0, "V_m", 1)[0])
    base, exc, inh = out
    assert exc > base > inh


def test_cond_exp_trace_matches_reference_loop(oracle):
    # iaf_cond_exp_test.py:235-329: V within 5e-6, conductances within 1e-6
    kw = dict(E_L=-70.0, C_m=250.0, t_ref=0.25, V_th=-55.0, V_reset=-60.0, E_ex=0.0, E_in=-85.0,
              g_L=16.6667, tau_syn_ex=0.2, tau_syn_in=2.0, I_e=20.0)
    p = dict(COND_DEFAULTS, **kw)
    sim = _sim(oracle, "iaf_cond_exp", -69.5, **kw)
    x_seq = [0.0, 30.0, 0.0, 0.0, -20.0, 0.0, 0.0]
    dg_seq = [[4.0], [], [-2.0], [3.0, -1.0], [], [], [1.5]]
    y, r, h, i_stim = np.array([-69.5, 0.0, 0.0]), 0, 0.1, 0.0
    refr_steps = math.ceil(0.25 / 0.1)
    for x, dgs in zip(x_seq, dg_seq):
        w_ex = sum(v for v in dgs if v >= 0)
        w_in = sum(-v for v in dgs if v < 0)
        sp = bool(sim.step_neuron(0, w0=w_ex, w1=w_in, x_next=x))
        y, h = _rkf45_dt("iaf_cond_exp", y, r > 0, i_stim, 0.1, h, p)
        y[1] += w_ex
        y[2] += w_in
        if r > 0:
            r -= 1
            y[0] = p["V_reset"]
            spike = False
        elif y[0] >= p["V_th"]:
            spike, r, y[0] = True, refr_steps, p["V_reset"]
        else:
            spike = False
        i_stim = x
        assert sp == spike
        assert sim.get_state(0, "V_m", 1)[0] == pytest.approx(y[0], abs=5e-6, rel=0)
        assert sim.get_state(0, "g_ex", 1)[0] == pytest.approx(y[1], abs=1e-6, rel=0)
        assert sim.get_state(0, "g_in", 1)[0] == pytest.approx(y[2], abs=1e-6, rel=0)


# ----------------------------------------------------------- iaf_cond_alpha

def test_cond_alpha_current_input_has_one_step_delay(oracle):
    # iaf_cond_alpha_test.py:182-199
    sim = _sim(oracle, "iaf_cond_alpha", 0.0, E_L=0.0, g_L=0.0, I_e=0.0, V_th=1e9, V_reset=0.0)
    sim.step_neuron(0, x_next=100.0)
    assert abs(sim.get_state(0, "V_m", 1)[0]) < 1e-12
    sim.step_neuron(0, x_next=0.0)
    assert sim.get_state(0, "V_m", 1)[0] == pytest.approx(0.04, abs=1e-9)


def test_cond_alpha_trace_matches_reference_loop(oracle):
    # iaf_cond_alpha_test.py:223-329: every state and h within 2e-6, r and
    # the spike train exact, at least one spike
    kw = dict(E_L=-70.0, C_m=250.0, t_ref=0.25, V_th=-58.0, V_reset=-60.0, E_ex=0.0, E_in=-85.0,
              g_L=16.6667, tau_syn_ex=0.2, tau_syn_in=2.0, I_e=900.0)
    p = dict(COND_DEFAULTS, **kw)
    sim = _sim(oracle, "iaf_cond_alpha", -69.5, **kw)
    x_seq = [0.0, 20.0, 0.0, -30.0, 0.0, 40.0, 0.0, 0.0, -10.0, 0.0, 0.0, 0.0] + [0.0] * 36
    w_seq = [0.0, 5.0, -2.0, 0.0, 4.0, -3.0, 0.0, 0.0, 1.0, 0.0, 0.0, -2.5] + [0.0] * 36
    y, r, h, i_stim = np.array([-69.5, 0.0, 0.0, 0.0, 0.0]), 0, 0.1, 0.0
    names = ["V_m", "dg_ex", "g_ex", "dg_in", "g_in"]
    spikes_o, spikes_r = [], []
    for x, w in zip(x_seq, w_seq):
        spikes_o.append(bool(sim.step_neuron(0, w0=max(w, 0.0), w1=max(-w, 0.0), x_next=x)))
        y, h = _rkf45_dt("iaf_cond_alpha", y, r > 0, i_stim, 0.1, h, p)
        if r > 0:
            r -= 1
            y[0] = p["V_reset"]
            spike = False
        elif y[0] >= p["V_th"]:
            spike, r, y[0] = True, math.ceil(p["t_ref"] / 0.1), p["V_reset"]
        else:
            spike, r = False, 0
        if w >= 0.0:
            y[1] += math.e / p["tau_syn_ex"] * w
        else:
            y[3] += math.e / p["tau_syn_in"] * (-w)
        i_stim = x
        spikes_r.append(spike)
        for i, nm in enumerate(names):
            assert sim.get_state(0, nm, 1)[0] == pytest.approx(y[i], abs=2e-6, rel=0), nm
        assert sim.get_state(0, "r", 1)[0] == r
        assert sim.get_state(0, "h", 1)[0] == pytest.approx(h, abs=2e-6, rel=0)
    assert spikes_o == spikes_r and any(spikes_o)


# ------------------------------------------------- library validation (host)

@pytest.mark.parametrize("model", ["iaf_cond_exp", "iaf_cond_alpha"])
def test_cond_validation_errors_match_reference_messages(model):
    # iaf_cond_exp.py:360-379, iaf_cond_alpha.py:368-385
    pl = _lib.Plan(0.1, model)
    with pytest.raises(ValueError, match="Reset potential must be smaller than threshold"):
        pl.add_pop(2, _params(V_reset=-50.0, V_th=-55.0))
    with pytest.raises(ValueError, match="Capacitance must be strictly positive"):
        pl.add_pop(2, _params(C_m=0.0))
    with pytest.raises(ValueError, match="Refractory time cannot be negative"):
        pl.add_pop(2, _params(t_ref=-0.1))
    with pytest.raises(ValueError, match="time constants must be strictly positive"):
        pl.add_pop(2, _params(tau_syn_in=0.0))
    if model == "iaf_cond_exp":
        with pytest.raises(ValueError, match="gsl_error_tol"):
            pl.add_pop(2, _params(gsl_error_tol=0.0))
    pl.add_pop(2, _params())
