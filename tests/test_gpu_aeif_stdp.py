"""GPU parity of the per-step engine (aeif_cond_alpha RKF45, plastic
stdp_synapse projections) against the float64 oracle.

Tolerances: FP64 RKF45 states within 2e-6 (the reference test's own band,
_nest_neuron/aeif_cond_alpha_test.py:281-392; CUDA's exp differs from the
host's by an ulp, and the adaptive controller amplifies nothing below that);
plastic weights within 1e-12 relative over a horizon where the rasters agree.
"""
import math

import numpy as np
import pytest

from brainpy.state_b200 import _lib
from tests.netbuild import random_csr

pytestmark = pytest.mark.gpu

AEIF = dict(V_peak=0.0, V_reset=-60.0, t_ref=0.0, g_L=30.0, C_m=281.0, E_ex=0.0, E_in=-85.0,
            E_L=-70.6, Delta_T=2.0, tau_w=144.0, a=4.0, b=80.5, V_th=-50.4, tau_syn_ex=0.2,
            tau_syn_in=2.0, I_e=0.0, gsl_error_tol=1e-6)
AEIF_ORDER = ["V_peak", "V_reset", "t_ref", "g_L", "C_m", "E_ex", "E_in", "E_L", "Delta_T",
              "tau_w", "a", "b", "V_th", "tau_syn_ex", "tau_syn_in", "I_e", "gsl_error_tol"]


def _aeif_net(sim_or_plan, is_plan, NE=160, NI=40, seed=4, t_ref=2.0):
    rng = np.random.default_rng(seed)
    p = [dict(AEIF, t_ref=t_ref)[k] for k in AEIF_ORDER]
    add_pop = sim_or_plan.add_pop
    add_proj = sim_or_plan.add_csr if is_plan else sim_or_plan.add_proj
    add_drive = sim_or_plan.add_poisson if is_plan else sim_or_plan.add_drive
    add_pop(NE, p)
    add_pop(NI, p)
    add_drive(0, 9000.0, 3.0, 5, 31, receptor=0)
    add_drive(1, 9000.0, 3.0, 5, 32, receptor=0)
    for pre, K, w, rec in ((0, 16, 0.8, 0), (1, 4, 2.5, 1)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            indptr, idx, ww, d = random_csr(rng, n_pre, n_post, K, w,
                                            rng.integers(5, 20, n_post * K))
            add_proj(pre, post, indptr, idx, ww, d, rec)
    return rng.uniform(-70.0, -55.0, NE + NI)


def test_aeif_network_fp64_matches_oracle(oracle):
    rec = np.arange(0, 200, 3)
    pl = _lib.Plan(0.1, "aeif_cond_alpha", precision=64)
    v0 = _aeif_net(pl, True)
    pl.record_v(rec)
    pl.upload()
    pl.set_state(0, "V_m", v0[:160])
    pl.set_state(1, "V_m", v0[160:])
    sim = oracle.OracleSim(0.1, "aeif_cond_alpha")
    _aeif_net(sim, False)
    sim.record_v(rec)
    sim.set_state(0, "V_m", v0[:160])
    sim.set_state(1, "V_m", v0[160:])
    pl.run(150)
    st, g = pl.spikes()
    ost, og, ov = sim.run(150)
    assert len(ost) > 0
    assert set(zip(st.tolist(), g.tolist())) == set(zip(ost.tolist(), og.tolist()))
    np.testing.assert_allclose(pl.v_trace(), ov, rtol=0, atol=2e-6)
    for name in ("w", "g_ex", "g_in"):
        np.testing.assert_allclose(pl.get_state(0, name), sim.get_state(0, name, 160),
                                   rtol=0, atol=2e-6)
    # the integrator did the same work: substep counts (accepted + rejected)
    # agree to 0.1 % (the GPU's reciprocals and err^(-1/5) round differently
    # from the oracle's divisions, which can move an acceptance at the margin)
    n_gpu, n_ref = pl.rk_substeps(), sim.rk_substeps
    assert n_ref >= 200 * 150
    assert abs(n_gpu - n_ref) <= 1e-3 * n_ref, (n_gpu, n_ref)


def test_aeif_fp32_rate_close_to_oracle(oracle):
    pl = _lib.Plan(0.1, "aeif_cond_alpha", precision=32)
    v0 = _aeif_net(pl, True)
    pl.upload()
    pl.set_state(0, "V_m", v0[:160])
    pl.set_state(1, "V_m", v0[160:])
    sim = oracle.OracleSim(0.1, "aeif_cond_alpha")
    _aeif_net(sim, False)
    sim.set_state(0, "V_m", v0[:160])
    sim.set_state(1, "V_m", v0[160:])
    pl.run(3000)
    st, _ = pl.spikes()
    ost, _, _ = sim.run(3000)
    assert len(ost) > 50
    assert abs(len(st) - len(ost)) / len(ost) < 0.1


def test_stdp_network_fp64_matches_oracle(oracle):
    _stdp_parity(oracle, 200, 50, 20, 5, 20.68, seed=9)


def test_stdp_rows_wider_than_one_work_item_match_oracle(oracle):
    """In- and out-degrees of about 300 plastic edges: every STDP row spans
    two 256-edge work items of the facilitation and depression kernels."""
    _stdp_parity(oracle, 320, 80, 300, 75, 20.68 * 20 / 300, seed=12, min_rows=257)


def _stdp_parity(oracle, NE, NI, KE, KI, J, seed, min_rows=0):
    rng = np.random.default_rng(seed)
    params = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]
    rec = np.arange(0, NE + NI, 5)
    pieces = []
    for pre, K, w in ((0, KE, J), (1, KI, -5.0 * J)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            pieces.append((pre, post) + random_csr(rng, n_pre, n_post, K, w, 15))
    v0 = rng.uniform(0.0, 20.0, NE + NI)

    def build(s, is_plan):
        s.add_pop(NE, params)
        s.add_pop(NI, params)
        (s.add_poisson if is_plan else s.add_drive)(0, 17789.0, 20.68, 15, 5)
        (s.add_poisson if is_plan else s.add_drive)(1, 17789.0, 20.68, 15, 6)
        ids = []
        for pre, post, indptr, idx, w, d in pieces:
            ids.append((s.add_csr if is_plan else s.add_proj)(pre, post, indptr, idx, w, d))
        # E -> E plastic (tau 20 ms, lambda 0.05, Wmax 3 x initial)
        if is_plan:
            s.attach_stdp(ids[0], 20.0, 20.0, 0.05, 1.0, 1.0, 1.0, 3 * J)
        else:
            s.set_stdp(ids[0], 20.0, 20.0, 0.05, 1.0, 1.0, 1.0, 3 * J)
        return ids

    pl = _lib.Plan(0.1, precision=64)
    ids = build(pl, True)
    pl.record_v(rec)
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    sim = oracle.OracleSim(0.1)
    build(sim, False)
    sim.record_v(rec)
    sim.set_state(0, "V_m", v0[:NE])
    sim.set_state(1, "V_m", v0[NE:])
    pl.run(250)
    st, g = pl.spikes()
    ost, og, ov = sim.run(250)
    assert len(ost) > 0
    assert set(zip(st.tolist(), g.tolist())) == set(zip(ost.tolist(), og.tolist()))
    np.testing.assert_allclose(pl.v_trace(), ov, rtol=0, atol=1e-9)
    indptr_ee = pieces[0][2]
    E = pieces[0][3].size
    if min_rows:
        # widest out-row and in-column of the plastic projection
        assert np.diff(indptr_ee).max() >= min_rows
        assert np.bincount(pieces[0][3], minlength=NE).max() >= min_rows
    w_gpu = pl.weights(ids[0])
    w_cpu = sim.weights(0 + 2, E)  # oracle ids count drives too
    assert np.any(w_cpu != J)
    np.testing.assert_allclose(w_gpu, w_cpu, rtol=1e-12, atol=0)


def test_stdp_triplet_network_fp64_matches_oracle(oracle):
    """stdp_triplet_synapse on E -> E (fast and slow traces per side):
    rasters identical and FP64 weights within 1e-12 of the oracle."""
    rng = np.random.default_rng(19)
    params = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]
    NE, NI = 200, 50
    pieces = []
    for pre, K, w in ((0, 20, 20.68), (1, 5, -103.4)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            pieces.append((pre, post) + random_csr(rng, n_pre, n_post, K, w, 15))
    v0 = rng.uniform(0.0, 20.0, NE + NI)
    trip = dict(tau_plus=16.8, tau_plus_triplet=101.0, tau_minus=20.0, tau_minus_triplet=110.0,
                Aplus=0.5, Aplus_triplet=0.2, Aminus=0.6, Aminus_triplet=0.1, Wmax=3 * 20.68)

    def build(s, is_plan):
        s.add_pop(NE, params)
        s.add_pop(NI, params)
        (s.add_poisson if is_plan else s.add_drive)(0, 17789.0, 20.68, 15, 5)
        (s.add_poisson if is_plan else s.add_drive)(1, 17789.0, 20.68, 15, 6)
        ids = [(s.add_csr if is_plan else s.add_proj)(pre, post, indptr, idx, w, d)
               for pre, post, indptr, idx, w, d in pieces]
        (s.attach_stdp_triplet if is_plan else s.set_stdp_triplet)(ids[0], **trip)
        return ids

    pl = _lib.Plan(0.1, precision=64)
    ids = build(pl, True)
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    sim = oracle.OracleSim(0.1)
    build(sim, False)
    sim.set_state(0, "V_m", v0[:NE])
    sim.set_state(1, "V_m", v0[NE:])
    pl.run(300)
    st, g = pl.spikes()
    ost, og, _ = sim.run(300)
    assert len(ost) > 0
    assert set(zip(st.tolist(), g.tolist())) == set(zip(ost.tolist(), og.tolist()))
    E = pieces[0][3].size
    w_cpu = sim.weights(0 + 2, E)  # oracle ids count drives too
    assert np.any(w_cpu > 20.68) and np.any(w_cpu < 20.68)
    np.testing.assert_allclose(pl.weights(ids[0]), w_cpu, rtol=1e-12, atol=0)


def test_stdp_synapse_hom_is_the_pair_rule():
    """Simulator facade: stdp_synapse_hom gives the weights stdp_synapse gives."""
    import brainpy.state_b200 as bs
    from brainpy.state_b200.units import Hz, mV, ms, pA
    out = []
    for syn_cls in (bs.stdp_synapse, bs.stdp_synapse_hom):
        sim = bs.Simulator(dt=0.1 * ms, precision=64)
        npar = dict(C_m=250.0, tau_m=20.0, tau_syn_ex=0.5, tau_syn_in=0.5, t_ref=2.0,
                    E_L=0.0, V_reset=10.0, V_th=20.0)
        ne = sim.create(bs.iaf_psc_alpha, 100, params=npar)
        noise = sim.create(bs.poisson_generator, rate=20000.0 * Hz)
        sim.connect(noise, ne, weight=20.68 * pA, delay=1.5 * ms, rule=bs.all_to_all)
        syn = syn_cls(weight=20.68, delay=1.5, lambda_=0.05, Wmax=3 * 20.68)
        proj = sim.connect(ne, ne, rule=bs.fixed_indegree(10), synapse=syn, seed=3)
        sim.simulate(50.0 * ms)
        out.append(sim._plan.weights(proj.proj_id))
    assert np.any(out[0] != 20.68)
    np.testing.assert_array_equal(out[0], out[1])


def test_weight_trace_per_step_matches_oracle(oracle):
    """record_weight / weight_trace: the (n_steps, n_edges) FP64 trajectory of
    a plastic projection after every step (_nest_network/simulator.py:382-396,
    :1868-1880), CSR order, against the oracle stepped one step at a time;
    two runs in a row (the second continues the first)."""
    rng = np.random.default_rng(23)
    NE, NI, J = 120, 30, 20.68
    params = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]
    pieces = []
    for pre, K, w in ((0, 15, J), (1, 4, -5.0 * J)):
        for post in (0, 1):
            n_pre, n_post = (NE if pre == 0 else NI), (NE if post == 0 else NI)
            pieces.append((pre, post) + random_csr(rng, n_pre, n_post, K, w, 15))
    v0 = rng.uniform(0.0, 20.0, NE + NI)

    def build(s, is_plan):
        s.add_pop(NE, params)
        s.add_pop(NI, params)
        (s.add_poisson if is_plan else s.add_drive)(0, 17789.0, 20.68, 15, 5)
        (s.add_poisson if is_plan else s.add_drive)(1, 17789.0, 20.68, 15, 6)
        ids = [(s.add_csr if is_plan else s.add_proj)(pre, post, indptr, idx, w, d)
               for pre, post, indptr, idx, w, d in pieces]
        (s.attach_stdp if is_plan else s.set_stdp)(ids[0], 20.0, 20.0, 0.05, 1.0, 1.0, 1.0,
                                                   3 * J)
        return ids

    pl = _lib.Plan(0.1, precision=64)
    ids = build(pl, True)
    pl.record_weights(ids[0])
    pl.upload()
    pl.set_state(0, "V_m", v0[:NE])
    pl.set_state(1, "V_m", v0[NE:])
    sim = oracle.OracleSim(0.1)
    build(sim, False)
    sim.set_state(0, "V_m", v0[:NE])
    sim.set_state(1, "V_m", v0[NE:])
    E = pieces[0][3].size
    for n in (70, 45):
        pl.run(n)
        tr = pl.weight_trace(ids[0])
        assert tr.shape == (n, E)
        ref = np.empty((n, E))
        for k in range(n):
            sim.run(1)
            ref[k] = sim.weights(0 + 2, E)   # oracle ids count the drives
        np.testing.assert_allclose(tr, ref, rtol=1e-12, atol=0)
    assert np.any(ref[-1] != J)


def test_aeif_fp32_spike_times_follow_fp64_oracle(oracle):
    """Uncoupled AdEx neurons on constant currents of 0.8-1.6 nA (adapting
    firing, 9 to 40 spikes), FP32 on the GPU against the float64 oracle over 500 ms:
    the FP32 exponential spike current (an FP32 exponent carried as hi + lo,
    within about 3 ulp of the rounded FP64 value) keeps the spike counts
    equal and every spike within two steps of the oracle's; the V_m traces
    agree to 0.5 mV away from the steps around a spike (the FP32 state rounds
    at each of the 5 000 steps, so the phase drifts slowly)."""
    currents = [800.0, 1000.0, 1300.0, 1600.0]
    n_steps = 5000
    pl = _lib.Plan(0.1, "aeif_cond_alpha", precision=32)
    sim = oracle.OracleSim(0.1, "aeif_cond_alpha")
    for I in currents:
        p = [dict(AEIF, I_e=I)[k] for k in AEIF_ORDER]
        pl.add_pop(1, p)
        sim.add_pop(1, p)
    rec = np.arange(len(currents))
    pl.record_v(rec)
    sim.record_v(rec)
    pl.upload()
    pl.run(n_steps)
    st, g = pl.spikes()
    ost, og, ov = sim.run(n_steps)
    v = pl.v_trace()
    near = np.zeros((n_steps, len(currents)), bool)
    for k in range(len(currents)):
        a, b = st[g == k], ost[og == k]
        assert a.size == b.size and a.size >= 5, (k, a.size, b.size)
        assert np.abs(a - b).max() <= 2, k
        for s in np.concatenate([a, b]):
            near[max(0, s - 5):s + 6, k] = True
    assert np.abs(v - ov)[~near].max() < 0.5
