"""The kernel-API front end on the GPU against the oracle built from the same
realised network (kernel timing, separate ex / in_ receptor ports with
different synaptic time constants, Poisson devices, keyed fixed_indegree).

Tolerances: FP64 spike counts per interval identical and V_m within 1e-9
(the tiled kernel with one ring per port; the Poisson units on the kernel's
block-key stream); FP32 rate within 5 %.
"""
import numpy as np
import pytest

from brainpy.state_b200 import _lib
from brainpy.state_b200 import kernel as K
from brainpy.state_b200.units import Hz, ms, pA

pytestmark = pytest.mark.gpu

PAR = dict(E_L=0.0, C_m=250.0, tau_m=20.0, t_ref=2.0, V_th=20.0, V_reset=10.0, tau_syn_ex=0.5,
           tau_syn_in=2.0)


def _network(model=K.iaf_psc_alpha, seed=11):
    # same charge per spike for the exponential kernel as for the alpha kernel
    J = 20.68 * (np.e if model is K.iaf_psc_exp else 1.0)
    rng = np.random.default_rng(seed)
    net = K.Network(dt=0.1 * ms, seed=seed)
    E = net.add(model, 200, params=PAR, init=dict(V_m=rng.uniform(0, 20, 200)), name="E")
    I = net.add(model, 50, params=PAR, init=dict(V_m=rng.uniform(0, 20, 50)), name="I")
    noise = net.add(K.poisson_generator, 250, params=dict(rate=17789.0 * Hz), name="noise")
    net.connect(noise, E + I, rule=K.one_to_one(), port="ex", weight=J * pA,
                delay=1.5 * ms)
    net.connect(E, E + I, rule=K.fixed_indegree(20), port="ex", weight=J * pA,
                delay=1.5 * ms, name="exc")
    net.connect(I, E + I, rule=K.fixed_indegree(5), port="in_", weight=-5.0 * J * pA,
                delay=0.8 * ms, name="inh")
    obs = net.observe(E[:40] + I[:10], "spike", "V_m", interval=0.5 * ms)
    return net, obs


def _oracle_twin(oracle, prog, model_name):
    sim = oracle.OracleSim(prog.dt, model_name, semantics=_lib.RING)
    sim.set_ports(True)
    for p in prog.net.populations:
        if not p.is_device:
            sim.add_pop(p.n, p.params)
    for post, rate, w, d, okey, unit0, t_min, t_max, port in prog.drives:
        sim.add_drive_keyed(post, rate, w, d, okey, unit0, t_min, t_max, receptor=port)
    for a, b, indptr, idx, w, d, port in prog.realised:
        sim.add_proj(a, b, indptr, idx, w, d, port)
    for p in prog.net.populations:
        if not p.is_device:
            sim.set_state(p.lib_pop, "V_m", np.broadcast_to(p.init["V_m"], (p.n,)))
    return sim


@pytest.mark.parametrize("model", [K.iaf_psc_alpha, K.iaf_psc_exp])
def test_kernel_frontend_fp64_matches_oracle(oracle, model):
    net, obs = _network(model)
    prog = net.compile("float64")
    run = prog.runner()
    r1 = run.simulate(20.0 * ms)
    r2 = run.cont(20.0 * ms)
    assert run.n == 400
    spk = np.concatenate([r1[obs]["spike"], r2[obs]["spike"]])
    vm = np.concatenate([r1[obs]["V_m"], r2[obs]["V_m"]])
    assert spk.shape == (80, 50) and vm.shape == (80, 50)
    np.testing.assert_allclose(r2[obs].times[:2], [20.5, 21.0])

    sim = _oracle_twin(oracle, prog, model.model_name)
    cols = np.array([prog._lib_gid(g) for g in obs.view.gids])
    sim.record_v(cols)
    st, g, v = sim.run(400)
    ref = np.zeros((80, 50))
    col = {int(c): i for i, c in enumerate(cols)}
    for s, gg in zip(st.tolist(), g.tolist()):
        if gg in col:
            ref[s // 5, col[gg]] += 1
    assert ref.sum() > 20
    np.testing.assert_array_equal(spk, ref)
    np.testing.assert_allclose(vm, v[4::5], rtol=0, atol=1e-9)
    # simulate() starts again from the initial state
    r3 = run.simulate(20.0 * ms)
    np.testing.assert_array_equal(r3[obs]["spike"], r1[obs]["spike"])


def test_kernel_frontend_fp32_rate_close_to_oracle(oracle):
    net, _ = _network()
    E, I = net.populations[0], net.populations[1]
    obs = net.observe(K.PopulationView(net, np.concatenate([E.gids, I.gids])), "spike",
                      name="all")
    prog = net.compile("float32")
    res = prog.runner().simulate(500.0 * ms)
    sim = _oracle_twin(oracle, prog, "iaf_psc_alpha")
    st, g, _ = sim.run(5000)
    # the plan records the observed neurons' spikes (here all of them)
    cols = np.array([prog._lib_gid(x) for x in obs.view.gids])
    ref = int(np.isin(g, cols).sum())
    n_gpu = int(res[obs]["spike"].sum())
    assert prog.plan.spikes()[0].size == n_gpu
    assert ref > 3000
    assert abs(n_gpu - ref) / ref < 0.05
