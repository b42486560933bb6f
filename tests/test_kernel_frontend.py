"""Kernel-API front end on the host: network structure (gids, views, names,
validation, after _kernel/network.py:316-716 and its doctests) and the keyed
fixed_indegree, checked bitwise against the oracle's restatement of the
kernel's key chain (_kernel/rng.py:106-300, _kernel/connectivity/rules.py:
226-265).  No GPU: connectivity is realised on the host."""
import numpy as np
import pytest

from brainpy.state_b200 import kernel as K
from brainpy.state_b200.units import ms, pA


def test_network_structure_and_names():
    net = K.Network(dt=0.1 * ms, seed=0)
    E = net.add(K.iaf_psc_alpha, 80, name="E")
    I = net.add(K.iaf_psc_alpha, 20, name="I")
    assert E.gids[:3].tolist() == [0, 1, 2] and I.gids[:3].tolist() == [80, 81, 82]
    anon = net.add(K.iaf_psc_alpha, 5)
    assert anon.name == "iaf_psc_alpha_0" and net.n_neurons == 105
    p = net.connect(E, E + I, rule=K.fixed_indegree(8), port="ex", weight=10.0 * pA,
                    delay=1.5 * ms)
    assert p.name == "FixedIndegree_0"
    rec = net.observe(E[:5], "spike", "V_m")
    assert rec.name == "Observer_0" and rec.size == 5
    assert len(net.populations) == 3 and len(net.projections) == 1 and len(net.observers) == 1
    v = (E[75:] + I[:3])
    parts = v.parts()
    assert [p.name for p, _ in parts] == ["E", "I"]
    assert parts[0][1].tolist() == [75, 76, 77, 78, 79] and parts[1][1].tolist() == [0, 1, 2]


def test_network_validation():
    with pytest.raises(ValueError):
        K.Network(dt=0.0 * ms)
    with pytest.raises(ValueError):
        K.Network(dt=0.1 * ms, seed=-1)
    net = K.Network(dt=0.1 * ms)
    E = net.add(K.iaf_psc_alpha, 10, name="E")
    with pytest.raises(ValueError, match="already used"):
        net.add(K.iaf_psc_alpha, 3, name="E")
    with pytest.raises(ValueError):
        net.add(K.iaf_psc_alpha, -1)
    with pytest.raises(NotImplementedError):
        net.add(K.iaf_psc_exp, 3)  # one neuron model per network
    with pytest.raises(ValueError, match="port"):
        net.connect(E, E)
    with pytest.raises(ValueError, match="one_to_one"):
        net.connect(E, E[:3], rule=K.one_to_one(), port="ex")
    with pytest.raises(NotImplementedError):
        K.fixed_indegree(3, allow_multapses=False)
    pg = net.add(K.poisson_generator, 10, params=dict(rate=100.0))
    with pytest.raises(NotImplementedError):
        net.connect(pg, E, rule=K.all_to_all(), port="ex")
    with pytest.raises(ValueError, match="interval"):
        net.observe(E, "spike", interval=0.15 * ms)


def test_keyed_fixed_indegree_matches_oracle_bitwise(oracle):
    net = K.Network(dt=0.1 * ms, seed=77)
    E = net.add(K.iaf_psc_alpha, 1500, name="E")   # more than one 1024-id block
    I = net.add(K.iaf_psc_alpha, 300, name="I")
    proj = net.connect(E + I, E[100:] + I, rule=K.fixed_indegree(7, allow_autapses=False),
                       port="ex", name="EI_rec")
    src, dst = K.realise_positions(net, proj)
    pre, post = proj.pre, proj.post
    where = {int(g): i for i, g in enumerate(pre.gids)}
    self_pos = np.array([where.get(int(g), -1) for g in post.gids])
    parts = [(p.name, local) for p, local in post.parts()]
    ref = oracle.kernel_fixed_indegree(77, "EI_rec", parts, pre.size, self_pos, 7)
    # realised in the rule's canonical order: post-major, pre ascending
    np.testing.assert_array_equal(src.reshape(-1, 7), np.sort(ref, axis=1))
    assert not np.any(pre.gids[src] == post.gids[dst])         # no autapses
    # a different projection name or seed gives other edges
    other = net.connect(E + I, E[100:] + I, rule=K.fixed_indegree(7), port="ex")
    assert not np.array_equal(K.realise_positions(net, other)[0], src)


def test_realised_edges_do_not_depend_on_unrelated_populations():
    """Keys come from the population's name and local ids, not global gids
    (_kernel/rng.py:274-303): an extra earlier population shifts the gids but
    not which (population, local id) pairs are connected."""
    def build(extra):
        net = K.Network(dt=0.1 * ms, seed=5)
        if extra:
            net.add(K.iaf_psc_alpha, 37, name="X")
        E = net.add(K.iaf_psc_alpha, 200, name="E")
        I = net.add(K.iaf_psc_alpha, 50, name="I")
        proj = net.connect(E, E + I, rule=K.fixed_indegree(9), port="ex", name="EE")
        src, dst = K.realise_positions(net, proj)
        def named(view, pos):
            out = []
            for g in view.gids[pos]:
                for p in net.populations:
                    if p.gid_start <= g < p.gid_start + p.n:
                        out.append((p.name, int(g - p.gid_start)))
            return out
        return named(proj.pre, src), named(proj.post, dst)
    assert build(False) == build(True)


def test_trial_indices():
    """The reference's doctest (_kernel/runner.py:100-106) and its checks."""
    assert K.trial_indices(3).tolist() == [0, 1, 2]
    assert K.trial_indices(2, "common").tolist() == [0, 0]
    assert int(K.trial_indices(None)) == 0
    assert K.trial_indices(4).dtype == np.uint32
    with pytest.raises(ValueError):
        K.trial_indices(2, "shared")
    for bad in (0, -1, 2.0, True):
        with pytest.raises(ValueError):
            K.trial_indices(bad)


def test_oracle_trial_folds_into_keyed_step_keys(oracle):
    """The oracle's keyed drive draws trial t's counts from
    fold(fold(fold(obj, b), n), t): its counts for trial 0 are the unbatched
    ones, another trial's differ."""
    from oracle import kernel_net as KN
    counts = []
    for trial in (0, 0, 3):
        sim = oracle.OracleSim(0.1, "iaf_psc_alpha", semantics=oracle.RING)
        sim.set_ports(True)
        a = sim.add_pop(200, [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -np.inf])
        sim.set_trial(trial)
        sim.add_drive_keyed(a, 30000.0, 25.0, 10, KN.object_key(7, "noise"), 0, 0, 2 ** 62, 0)
        sim.record_v(np.arange(0, 200, 9))
        _, _, v = sim.run(60, cap=1 << 16)
        counts.append(v)
    np.testing.assert_array_equal(counts[0], counts[1])
    assert np.abs(counts[2] - counts[0]).max() > 1e-6
