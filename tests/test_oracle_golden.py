"""Pin the float64 oracle against the reference's own golden vectors.

Every expected value below is a constant (or an independent restatement of a
reference test's own reference loop) taken from the reference's test suite;
the citations name the reference test each case comes from.
"""
import math

import numpy as np
import pytest

# iaf_psc_alpha parameter order: E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in I_e V_min
NEST_ALPHA_DEFAULTS = dict(E_L=-70.0, C_m=250.0, tau_m=10.0, t_ref=2.0, V_th=-55.0,
                           V_reset=-70.0, tau_syn_ex=2.0, tau_syn_in=2.0, I_e=0.0,
                           V_min=-math.inf)
ALPHA_ORDER = ["E_L", "C_m", "tau_m", "t_ref", "V_th", "V_reset", "tau_syn_ex",
               "tau_syn_in", "I_e", "V_min"]
EXP_ORDER = ALPHA_ORDER[:-1]
AEIF_ORDER = ["V_peak", "V_reset", "t_ref", "g_L", "C_m", "E_ex", "E_in", "E_L", "Delta_T",
              "tau_w", "a", "b", "V_th", "tau_syn_ex", "tau_syn_in", "I_e", "gsl_error_tol"]
AEIF_DEFAULTS = dict(V_peak=0.0, V_reset=-60.0, t_ref=0.0, g_L=30.0, C_m=281.0, E_ex=0.0,
                     E_in=-85.0, E_L=-70.6, Delta_T=2.0, tau_w=144.0, a=4.0, b=80.5,
                     V_th=-50.4, tau_syn_ex=0.2, tau_syn_in=2.0, I_e=0.0, gsl_error_tol=1e-6)


def _params(order, defaults, **kw):
    d = dict(defaults)
    d.update(kw)
    return [d[k] for k in order]


# ----------------------------------------------------------------- Threefry

def test_threefry_known_answers(oracle):
    # Random123 known-answer vectors for threefry2x32_20 (also asserted by
    # JAX's own random tests).
    assert oracle.threefry2x32((0, 0), (0, 0)) == (0x6B200159, 0x99BA4EFE)
    assert oracle.threefry2x32((0xFFFFFFFF, 0xFFFFFFFF),
                               (0xFFFFFFFF, 0xFFFFFFFF)) == (0x1CB996FC, 0xBB002BE7)
    assert oracle.threefry2x32((0x13198A2E, 0x03707344),
                               (0x243F6A88, 0x85A308D3)) == (0xC4923A9C, 0x483DF7A0)


def test_jax_layer_self_consistency(oracle):
    # split(key, n)[i] == fold_in(key, i) in the partitionable layout, and
    # randint stays in range for both 32- and 64-bit draws.
    k = oracle.jax_key(1234)
    assert list(k) == [0, 1234]
    sp = oracle.jax_split(k, 3)
    for i in range(3):
        assert list(sp[i]) == list(oracle.jax_fold_in(k, i))
    for nbits in (32, 64):
        r = oracle.jax_randint(k, 5000, 0, 17, nbits)
        assert r.min() >= 0 and r.max() < 17
        assert len(np.unique(r)) == 17


def test_fixed_indegree_structure(oracle):
    pre, post = oracle.fixed_indegree(7, 50, 20, 10)
    assert pre.shape == (200,) and np.all((pre >= 0) & (pre < 50))
    np.testing.assert_array_equal(post, np.repeat(np.arange(20), 10))
    pre2, _ = oracle.fixed_indegree(7, 50, 20, 10, pre_is_post=True, allow_autapses=False)
    assert np.all(pre2 != np.repeat(np.arange(20), 10))


# ---------------------------------------------------------------------- CSR

def test_csr_structure_matches_reference_example(oracle):
    # _nest_network/connectivity_test.py:294-301
    pre = np.array([2, 0, 2, 1, 0])
    post = np.array([4, 1, 3, 0, 2])
    order, indices, indptr = oracle.csr_structure(pre, post, 4)
    np.testing.assert_array_equal(pre[order], [0, 0, 1, 2, 2])
    np.testing.assert_array_equal(indices, [1, 2, 0, 4, 3])
    np.testing.assert_array_equal(indptr, [0, 2, 3, 5, 5])
    order, indices, indptr = oracle.csr_structure(np.zeros(0), np.zeros(0), 3)
    assert order.shape == (0,) and indices.shape == (0,)
    np.testing.assert_array_equal(indptr, [0, 0, 0, 0])


# ------------------------------------------------------------ iaf_psc_alpha

def _alpha_reference_p31_p32(tau_syn, tau_m, c_m, h):
    # restatement of _nest_neuron/iaf_psc_alpha_test.py:30-55 (numpy float64
    # scalars so tau_syn == tau_m gives inf/nan like the reference's NumPy path)
    tau_syn, tau_m, c_m = np.float64(tau_syn), np.float64(tau_m), np.float64(c_m)
    with np.errstate(all="ignore"):
        beta = tau_syn * tau_m / (tau_m - tau_syn)
        gamma = beta / c_m
        inv_beta = (tau_m - tau_syn) / (tau_syn * tau_m)
        e_syn = np.exp(-h / tau_syn)
        em1 = np.expm1(h * inv_beta)
        p32 = gamma * e_syn * em1
        h_min = 1e-7 * tau_m * tau_m / abs(tau_m - tau_syn)
    if (not math.isfinite(p32)) or abs(p32) < np.finfo(np.float64).tiny or p32 <= 0.0:
        p32 = h / c_m * math.exp(-h / tau_m)
    if np.isfinite(h_min) and h > h_min:
        p31 = gamma * e_syn * (beta * em1 - h)
    else:
        p31 = 0.5 * h * h / c_m * math.exp(-h / tau_m)
    return p31, p32


@pytest.mark.parametrize("tau_syn", [0.5, 2.0, 10.0, 10.0 + 1e-10, 9.999999])
def test_alpha_propagators_match_reference_helper(oracle, tau_syn):
    got = oracle.alpha_p31_p32(tau_syn, 10.0, 250.0, 0.1)
    exp = _alpha_reference_p31_p32(tau_syn, 10.0, 250.0, 0.1)
    assert got[0] == pytest.approx(exp[0], rel=1e-12, abs=0)
    assert got[1] == pytest.approx(exp[1], rel=1e-12, abs=0)


def test_iaf_psc_alpha_nest_trace(oracle):
    # NEST testsuite trace, _nest_neuron/iaf_psc_alpha_test.py:200-245
    ref = {0.1: -69.6020, 0.2: -69.2079, 0.3: -68.8178, 0.4: -68.4316, 0.5: -68.0492,
           4.3: -56.0204, 4.4: -55.7615, 4.5: -55.5051, 4.6: -55.2513, 4.7: -55.0001,
           4.8: -70.0000, 4.9: -70.0000, 5.0: -70.0000}
    sim = oracle.OracleSim(0.1, "iaf_psc_alpha")
    sim.add_pop(1, _params(ALPHA_ORDER, NEST_ALPHA_DEFAULTS, I_e=1000.0))
    first = None
    for k in range(80):
        sp = sim.step_neuron(0)
        v = sim.get_state(0, "V_m", 1)[0]
        t = round((k + 1) * 0.1, 1)
        if t in ref:
            assert abs(v - ref[t]) <= 8e-4, (t, v)
        if sp and first is None:
            first = (k + 1) * 0.1  # last_spike_time = t + dt
    assert abs(first - 4.8) <= 1e-12


def _alpha_reference_step(state, p, x_next, w_step, dt):
    # restatement of _nest_neuron/iaf_psc_alpha_test.py:57-127
    y0, dI_ex, I_ex, dI_in, I_in, y3, r = (state[k] for k in
                                           ("y0", "dI_ex", "I_ex", "dI_in", "I_in", "y3", "r"))
    tau_m, c_m, tex, tin = p["tau_m"], p["C_m"], p["tau_syn_ex"], p["tau_syn_in"]
    theta = p["V_th"] - p["E_L"]
    v_reset = p["V_reset"] - p["E_L"]
    lower = -math.inf if p["V_min"] == -math.inf else p["V_min"] - p["E_L"]
    p11e = math.exp(-dt / tex); p21e = dt * p11e
    p11i = math.exp(-dt / tin); p21i = dt * p11i
    em1 = math.expm1(-dt / tau_m)
    p30 = -tau_m / c_m * em1
    p31e, p32e = _alpha_reference_p31_p32(tex, tau_m, c_m, dt)
    p31i, p32i = _alpha_reference_p31_p32(tin, tau_m, c_m, dt)
    if r == 0:
        y3 = (p30 * (y0 + p["I_e"]) + p31e * dI_ex + p32e * I_ex + p31i * dI_in + p32i * I_in
              + em1 * y3 + y3)
        y3 = max(y3, lower)
    else:
        r -= 1
    I_ex = p21e * dI_ex + p11e * I_ex
    dI_ex *= p11e
    dI_ex += math.e / tex * max(w_step, 0.0)
    I_in = p21i * dI_in + p11i * I_in
    dI_in *= p11i
    dI_in += math.e / tin * min(w_step, 0.0)
    spike = y3 >= theta
    if spike:
        r = int(math.ceil(p["t_ref"] / dt))
        y3 = v_reset
    state.update(y0=x_next, dI_ex=dI_ex, I_ex=I_ex, dI_in=dI_in, I_in=I_in, y3=y3, r=r)
    return spike


@pytest.mark.parametrize("E_L,V_min", [(-70.0, -math.inf), (0.0, -math.inf), (-65.0, -72.0)])
def test_iaf_psc_alpha_equations_with_spikes(oracle, E_L, V_min):
    # equation check of _nest_neuron/iaf_psc_alpha_test.py:247-407 (1e-11 with spikes)
    p = dict(NEST_ALPHA_DEFAULTS, E_L=E_L, V_th=E_L + 15.0, V_reset=E_L, V_min=V_min,
             tau_syn_ex=0.5, tau_syn_in=3.0, I_e=450.0, t_ref=0.5)
    rng = np.random.default_rng(3)
    w_seq = rng.normal(10.0, 20.0, 400) * (rng.random(400) < 0.3)
    sim = oracle.OracleSim(0.1, "iaf_psc_alpha")
    sim.add_pop(1, [p[k] for k in ALPHA_ORDER])
    sim.set_state(0, "V_m", [E_L])
    ref = dict(y0=0.0, dI_ex=0.0, I_ex=0.0, dI_in=0.0, I_in=0.0, y3=0.0, r=0)
    nspk = 0
    for k in range(400):
        sp = sim.step_neuron(0, w0=w_seq[k])
        rs = _alpha_reference_step(ref, p, 0.0, w_seq[k], 0.1)
        assert bool(sp) == rs
        nspk += rs
        assert sim.get_state(0, "V_m", 1)[0] == pytest.approx(ref["y3"] + E_L, abs=1e-11)
        assert sim.get_state(0, "dI_syn_ex", 1)[0] == pytest.approx(ref["dI_ex"], abs=1e-11)
        assert sim.get_state(0, "I_syn_in", 1)[0] == pytest.approx(ref["I_in"], abs=1e-11)
        assert sim.get_state(0, "r", 1)[0] == ref["r"]
    assert nspk > 0


# -------------------------------------------------------------- iaf_psc_exp

def test_iaf_psc_exp_dc_first_spike(oracle):
    # _nest_neuron/iaf_psc_exp_test.py:84-103: NEST DC test, first spike 4.8 ms
    sim = oracle.OracleSim(0.1, "iaf_psc_exp")
    sim.add_pop(1, _params(EXP_ORDER, NEST_ALPHA_DEFAULTS, I_e=1000.0))
    last = None
    for k in range(80):
        if sim.step_neuron(0):
            last = (k + 1) * 0.1
            break
    assert abs(last - 4.8) <= 1e-12


def test_iaf_psc_exp_equations(oracle):
    # restatement of the propagator/update equations of iaf_psc_exp.py:492-682
    p = dict(NEST_ALPHA_DEFAULTS, tau_syn_ex=2.0, tau_syn_in=5.0, I_e=200.0)
    dt = 0.1
    sim = oracle.OracleSim(dt, "iaf_psc_exp")
    sim.add_pop(1, [p[k] for k in EXP_ORDER])
    P11e, P11i, P22 = math.exp(-dt / 2.0), math.exp(-dt / 5.0), math.exp(-dt / 10.0)
    P21e = oracle.propagator_exp(2.0, 10.0, 250.0, dt)
    P21i = oracle.propagator_exp(5.0, 10.0, 250.0, dt)
    P20 = 10.0 / 250.0 * (1.0 - math.exp(-dt / 10.0))
    V, ie, ii, r = 0.0, 0.0, 0.0, 0
    rng = np.random.default_rng(1)
    for k in range(300):
        w = rng.normal(0, 80.0)
        sp = sim.step_neuron(0, w0=w)
        if r == 0:
            V = V * P22 + ie * P21e + ii * P21i + (200.0 + 0.0) * P20
        else:
            r -= 1
        ie *= P11e; ii *= P11i
        ie += max(w, 0.0); ii += min(w, 0.0)
        s = V >= 15.0
        if s:
            r = 20; V = 0.0
        assert bool(sp) == s
        assert sim.get_state(0, "V_m", 1)[0] == pytest.approx(V - 70.0, abs=1e-11)


# ---------------------------------------------------------- aeif_cond_alpha

def test_aeif_current_one_step_delay(oracle):
    # _nest_neuron/aeif_cond_alpha_test.py:259-279
    p = _params(AEIF_ORDER, AEIF_DEFAULTS, V_th=1e6, V_peak=1e6, Delta_T=0.0, g_L=0.0, a=0.0,
                b=0.0, I_e=0.0, V_reset=0.0)
    sim = oracle.OracleSim(0.1, "aeif_cond_alpha")
    sim.add_pop(1, p)
    sim.set_state(0, "V_m", [0.0])
    sim.step_neuron(0, x_next=100.0)
    assert abs(sim.get_state(0, "V_m", 1)[0]) < 1e-12
    sim.step_neuron(0, x_next=0.0)
    assert abs(sim.get_state(0, "V_m", 1)[0] - 0.03558718861209964) <= 1e-12


def _aeif_test_rhs(y, refr, i_stim, p):
    v, dg_ex, g_ex, dg_in, g_in, w = y
    v_eff = p["V_reset"] if refr else min(v, p["V_peak"])
    i_ex = g_ex * (v_eff - p["E_ex"])
    i_in = g_in * (v_eff - p["E_in"])
    dts = 1.0 if p["Delta_T"] == 0.0 else p["Delta_T"]
    i_sp = 0.0 if p["Delta_T"] == 0.0 else p["g_L"] * p["Delta_T"] * math.exp((v_eff - p["V_th"]) / dts)
    dv = 0.0 if refr else (-p["g_L"] * (v_eff - p["E_L"]) + i_sp - i_ex - i_in - w + p["I_e"] + i_stim) / p["C_m"]
    return np.array([dv, -dg_ex / p["tau_syn_ex"], dg_ex - g_ex / p["tau_syn_ex"],
                     -dg_in / p["tau_syn_in"], dg_in - g_in / p["tau_syn_in"],
                     (p["a"] * (v_eff - p["E_L"]) - w) / p["tau_w"]])


def _aeif_test_step(y, r, h, i_stim, p, x_next, w_step, dt):
    # restatement of _reference_step_jax, _nest_neuron/aeif_cond_alpha_test.py:72-188
    min_h, atol, rc = 1e-8, p["gsl_error_tol"], p["refr_counts"]
    t, h, it, spk = 0.0, max(h, min_h), 0, 0
    while t < dt and it < 100000:
        h = max(min_h, min(h, dt - t))
        refr = r > 0
        f = lambda yy: _aeif_test_rhs(yy, refr, i_stim, p)
        k1 = f(y)
        k2 = f(y + h * (1.0 / 4.0) * k1)
        k3 = f(y + h * (3.0 * k1 / 32.0 + 9.0 * k2 / 32.0))
        k4 = f(y + h * (1932.0 * k1 / 2197.0 - 7200.0 * k2 / 2197.0 + 7296.0 * k3 / 2197.0))
        k5 = f(y + h * (439.0 * k1 / 216.0 - 8.0 * k2 + 3680.0 * k3 / 513.0 - 845.0 * k4 / 4104.0))
        k6 = f(y + h * (-8.0 * k1 / 27.0 + 2.0 * k2 - 3544.0 * k3 / 2565.0
                        + 1859.0 * k4 / 4104.0 - 11.0 * k5 / 40.0))
        y4 = y + h * (25.0 * k1 / 216.0 + 1408.0 * k3 / 2565.0 + 2197.0 * k4 / 4104.0 - k5 / 5.0)
        y5 = y + h * (16.0 * k1 / 135.0 + 6656.0 * k3 / 12825.0 + 28561.0 * k4 / 56430.0
                      - 9.0 * k5 / 50.0 + 2.0 * k6 / 55.0)
        err = float(np.max(np.abs(y5 - y4)))
        accept = (err <= atol) or (h <= min_h)
        es = max(err, 1e-30)
        if accept:
            y = y5.copy()
            if r > 0:
                y[0] = p["V_reset"]
            if r <= 0 and y[0] >= p["V_peak"]:
                y[0] = p["V_reset"]; y[5] += p["b"]; spk += 1
                if rc > 0:
                    r = rc + 1
            t = t + h
            fac = 5.0 if err == 0.0 else min(5.0, max(0.2, 0.9 * (atol / es) ** 0.2))
        else:
            fac = min(1.0, max(0.2, 0.9 * (atol / es) ** 0.25))
        h = max(min_h, h * fac)
        it += 1
    if r > 0:
        r -= 1
    if w_step >= 0.0:
        y[1] += math.e / p["tau_syn_ex"] * w_step
    if w_step < 0.0:
        y[3] += math.e / p["tau_syn_in"] * (-w_step)
    return y, r, h, x_next, spk


def test_aeif_rkf45_matches_reference_loop(oracle):
    # _nest_neuron/aeif_cond_alpha_test.py:281-392 (atol 2e-6 on all states and h)
    p = dict(V_peak=0.0, V_reset=-58.0, t_ref=0.25, g_L=11.0, C_m=200.0, E_ex=0.0, E_in=-85.0,
             E_L=-70.0, Delta_T=2.0, tau_w=300.0, a=3.0, b=40.0, V_th=-50.0, tau_syn_ex=0.2,
             tau_syn_in=2.0, I_e=1200.0, gsl_error_tol=1e-6)
    sim = oracle.OracleSim(0.1, "aeif_cond_alpha")
    sim.add_pop(1, [p[k] for k in AEIF_ORDER])
    sim.set_state(0, "V_m", [-68.0])
    sim.set_state(0, "w", [5.0])
    x_seq = [0.0, 20.0, 0.0, -30.0, 0.0, 40.0, 0.0, 0.0, -10.0, 0.0, 0.0, 0.0] + [0.0] * 48
    w_seq = [0.0, 5.0, -2.0, 0.0, 4.0, -3.0, 0.0, 0.0, 1.0, 0.0, 0.0, -2.5] + [0.0] * 48
    pr = dict(p, refr_counts=int(math.ceil(0.25 / 0.1)))
    y = np.array([-68.0, 0.0, 0.0, 0.0, 0.0, 5.0])
    r, h, i_stim = 0, 0.1, 0.0
    names = ["V_m", "dg_ex", "g_ex", "dg_in", "g_in", "w"]
    any_spike = False
    for k in range(60):
        w = w_seq[k]
        sp = sim.step_neuron(0, w0=max(w, 0.0), w1=(-w if w < 0 else 0.0), x_next=x_seq[k])
        y, r, h, i_stim, cnt = _aeif_test_step(y, r, h, i_stim, pr, x_seq[k], w, 0.1)
        for i, nm in enumerate(names):
            assert sim.get_state(0, nm, 1)[0] == pytest.approx(y[i], abs=2e-6, rel=0), (k, nm)
        assert sim.get_state(0, "r", 1)[0] == r
        assert sim.get_state(0, "h", 1)[0] == pytest.approx(h, abs=2e-6, rel=0)
        assert bool(sp) == (cnt > 0)
        any_spike |= bool(sp)
    assert any_spike


# --------------------------------------------------------------------- STDP

def _host_facilitate(w, kplus, Wmax=100., lam=0.01, mu_plus=1.):
    nw = w / Wmax + lam * (1.0 - w / Wmax) ** mu_plus * kplus
    return nw * Wmax if nw < 1.0 else Wmax


def _host_depress(w, kminus, Wmax=100., alpha=1., lam=0.01, mu_minus=1.):
    nw = w / Wmax - alpha * lam * (w / Wmax) ** mu_minus * kminus
    return nw * Wmax if nw > 0.0 else 0.0


def _stdp_pair_net(oracle, lam=0.1, w0=10.0, mu=1.0, wmax=100.0):
    """Two iaf neurons, pre -> post one plastic edge with D=0 (lag 1 step)."""
    sim = oracle.OracleSim(1.0, "iaf_psc_alpha")
    pa = _params(ALPHA_ORDER, NEST_ALPHA_DEFAULTS, t_ref=0.0)
    sim.add_pop(1, pa)  # pre
    sim.add_pop(1, pa)  # post
    pj = sim.add_proj(0, 1, [0, 1], [0], [w0], [0])
    sim.set_stdp(pj, 20.0, 20.0, lam, 1.0, mu, mu, wmax)
    return sim, pj


def test_stdp_potentiation_then_depression_in_network(oracle):
    # stdp_synapse_rule_test.py potentiation/depression cases, driven through
    # the eager substrate of event_plastic.py:454-518: a forced pre spike then
    # a forced post spike potentiates by lambda*(1-w/Wmax)*K+.
    sim, pj = _stdp_pair_net(oracle)
    # force spikes by setting V above threshold before the step
    sim.set_state(0, "V_m", [100.0])          # pre fires at step 0
    sim.run(1)
    sim.run(1)                                # step 1: pre spike reaches synapse (lag 1)
    w_after_pre = sim.weights(pj, 1)[0]
    assert w_after_pre == pytest.approx(10.0)  # no post trace yet -> no depression
    sim.set_state(1, "V_m", [100.0])          # post fires at step 2
    sim.run(1)
    sim.run(1)                                # step 3: post spike seen by the synapse
    dec = math.exp(-1.0 / 20.0)
    kplus = 1.0 * dec * dec                   # pre trace after two decays
    expect = _host_facilitate(10.0, kplus, lam=0.1)
    assert sim.weights(pj, 1)[0] == pytest.approx(expect, rel=1e-14)
    assert expect > 10.0
    sim.set_state(0, "V_m", [100.0])          # pre fires at step 4 -> seen at step 5
    sim.run(2)
    kminus = dec * dec                        # post trace (spike seen at step 3)
    assert sim.weights(pj, 1)[0] == pytest.approx(_host_depress(expect, kminus, lam=0.1),
                                                  rel=1e-14)


def test_stdp_clamps(oracle):
    # stdp_synapse_rule_test.py wmax/zero clamps
    sim, pj = _stdp_pair_net(oracle, lam=5.0, w0=99.0)
    sim.set_state(0, "V_m", [100.0]); sim.run(2)
    sim.set_state(1, "V_m", [100.0]); sim.run(2)
    assert sim.weights(pj, 1)[0] == 100.0
    sim2, pj2 = _stdp_pair_net(oracle, lam=5.0, w0=1.0)
    sim2.set_state(1, "V_m", [100.0]); sim2.run(2)
    sim2.set_state(0, "V_m", [100.0]); sim2.run(2)
    assert sim2.weights(pj2, 1)[0] == 0.0


# ------------------------------------------------------------- delay timing

def _impulse_net(oracle, semantics, delay):
    sim = oracle.OracleSim(1.0, "iaf_psc_alpha", semantics=semantics)
    pa = _params(ALPHA_ORDER, NEST_ALPHA_DEFAULTS, t_ref=0.0)
    sim.add_pop(1, pa)
    sim.add_pop(1, pa)
    sim.add_proj(0, 1, [0, 1], [0], [50.0], [delay])
    sim.record_v([1])
    return sim


def test_legacy_delay_adds_holder_lag(oracle):
    # _nest_network/delay_test.py:39-50 (InputDelay out[t] = in[t-D]) plus the
    # holder lag of simulator.py:1773-1779: a spike of step m reaches step m+D+1.
    for D in (0, 2, 5):
        sim = _impulse_net(oracle, oracle.LEGACY, D)
        sim.set_state(0, "V_m", [100.0])
        _, _, v = sim.run(12)
        dI = [sim.get_state(1, "dI_syn_ex", 1)[0]]
        first = int(np.argmax(np.abs(v[:, 0] - v[0, 0]) > 0))
        # the jump enters dI at step D+1, V responds one step later
        assert first == D + 2, (D, first)


def test_ring_delay_exact_arrival(oracle):
    # _kernel/delay_scatter.py:7-9 and delay_scatter_network_test.py:250: an
    # event of step n over delay d arrives in step n + d (no extra lag).
    for d in (1, 2, 5):
        sim = _impulse_net(oracle, oracle.RING, d)
        sim.set_state(0, "V_m", [100.0])
        _, _, v = sim.run(12)
        first = int(np.argmax(np.abs(v[:, 0] - v[0, 0]) > 0))
        assert first == d + 1, (d, first)


def test_ring_docstring_example(oracle):
    # _kernel/delay_scatter.py:144-153: edges (0->0 d=1 w=.5), (0->1 d=3 w=2),
    # (1->1 d=2 w=4), payload [1, 1] at step 0, ring L=3 ->
    # slots [[0,2],[0.5,0],[0,4]]; i.e. post 0 receives .5 at step 1, post 1
    # receives 4 at step 2 and 2 at step 3.
    sim = oracle.OracleSim(1.0, "iaf_psc_alpha", semantics=oracle.RING)
    pa = _params(ALPHA_ORDER, NEST_ALPHA_DEFAULTS, t_ref=0.0, tau_syn_ex=1e6)
    sim.add_pop(2, pa)
    sim.add_pop(2, pa)
    sim.add_proj(0, 1, [0, 2, 3], [0, 1, 1], [0.5, 2.0, 4.0], [1, 3, 2])
    sim.set_state(0, "V_m", [100.0, 100.0])
    e = math.e / 1e6
    got = []
    for _ in range(4):
        before = sim.get_state(1, "dI_syn_ex", 2)
        sim.run(1)
        after = sim.get_state(1, "dI_syn_ex", 2)
        got.append(np.round((after - before * math.exp(-1.0 / 1e6)) / e, 9))
    np.testing.assert_allclose(got[1], [0.5, 0.0], atol=1e-6)
    np.testing.assert_allclose(got[2], [0.0, 4.0], atol=1e-6)
    np.testing.assert_allclose(got[3], [0.0, 2.0], atol=1e-6)


# ------------------------------------------------------------------ Poisson

def test_poisson_stream_statistics(oracle):
    lam = 1.7789
    us = [oracle.uniform01(11, 0, s, t) for s in range(200) for t in range(100)]
    ks = np.array([oracle.poisson(lam, u) for u in us])
    assert abs(ks.mean() - lam) < 0.05
    assert abs(ks.var() - lam) < 0.1
    assert all(0.0 <= u < 1.0 for u in us)
