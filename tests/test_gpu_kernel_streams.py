"""GPU parity of networks on the reference kernel path's streams (C-ABI path).

The library realises the kernel path's Brunel network (brunel.
build_kernel_network: separate 'ex' / 'in_' ports, per-edge delays from the
DELAY stream, V_m from the INIT stream, noise counts from the device's block
keys); the oracle realises the same network independently
(oracle/kernel_net.py).  Tolerances as in test_gpu_parity: FP64 (atomic
delivery) identical spikes and |dV| <= 1e-9 mV over a horizon shorter than
the network's divergence; FP32 |dV| <= 2e-3 mV over 30 steps; population
rates within 1 % over 3 s at full size.
"""
import numpy as np
import pytest

from brainpy.state_b200 import brunel

pytestmark = pytest.mark.gpu


def _raster(steps, gids):
    return set(zip(steps.tolist(), gids.tolist()))


def _view(net, gids):
    from brainpy.state_b200.kernel import PopulationView
    return PopulationView(net, np.asarray(gids, np.int64))


@pytest.mark.parametrize("bits", [64, 32])
def test_tiled_ports_keyed_drive_matches_oracle(oracle, bits):
    """Order 100 (400 E + 100 I): the tiled kernel with one ring per port and
    the warp-shared keyed drive pass."""
    from oracle import kernel_net as KN
    order = 100
    rec = np.arange(0, 500, 7)
    net, p, _ = brunel.build_kernel_network(order=order)
    obs = net.observe(_view(net, rec), "V_m", name="taps")
    prog = net.compile("float64" if bits == 64 else "float32")
    assert prog.plan.engine == "tiled"
    sim, _ = KN.build(p, seed=1234, order=order, bits=bits)
    sim.record_v(rec)
    n = 300 if bits == 64 else 30
    res = prog.runner().simulate(n * 0.1)
    st, g = prog.plan.spikes()
    ost, og, ov = sim.run(n)
    v = res[obs]["V_m"]
    if bits == 64:
        assert len(st) > 0
        assert _raster(st, g) == _raster(ost, og)
        np.testing.assert_allclose(v, ov, rtol=0, atol=1e-9)
    else:
        np.testing.assert_allclose(v, ov, rtol=0, atol=2e-3)


def test_per_step_engine_keyed_drive_matches_oracle(oracle):
    """A drive onto the 'in_' port keeps a separate-port plan on the per-step
    engine; its keyed Poisson counts (two parts of one device population) must
    still be the oracle's."""
    from brainpy.state_b200.kernel import (Network, fixed_indegree, iaf_psc_alpha, one_to_one,
                                           poisson_generator)
    from brainpy.state_b200.units import Hz, ms, mV, pA, pF
    from oracle import kernel_net as KN
    net = Network(dt=0.1 * ms, seed=99)
    prm = dict(E_L=0.0 * mV, V_th=20.0 * mV, V_reset=10.0 * mV, tau_m=20.0 * ms,
               tau_syn_ex=0.5 * ms, tau_syn_in=0.5 * ms, C_m=250.0 * pF)
    A = net.add(iaf_psc_alpha, 300, params=prm, name="A")
    noise = net.add(poisson_generator, 600, params=dict(rate=30000.0 * Hz), name="noise")
    net.connect(noise[:300], A, one_to_one(), port="ex", weight=25.0 * pA, delay=1.0 * ms,
                name="n_ex")
    net.connect(noise[300:], A, one_to_one(), port="in_", weight=-10.0 * pA, delay=1.0 * ms,
                name="n_in")
    net.connect(A, A, fixed_indegree(20), port="ex", weight=15.0 * pA, delay=1.5 * ms, name="AA")
    obs = net.observe(A[::10], "V_m", name="v")
    prog = net.compile("float64")
    assert prog.plan.engine == "windowed"  # lags of 10 and 15 steps
    sim = oracle.OracleSim(0.1, "iaf_psc_alpha", semantics=oracle.RING)
    sim.set_ports(True)
    a = sim.add_pop(300, net.populations[0].params)
    okey = KN.object_key(99, "noise")
    sim.add_drive_keyed(a, 30000.0, 25.0, 10, okey, 0, 0, 2 ** 62, 0)
    sim.add_drive_keyed(a, 30000.0, -10.0, 10, okey, 300, 0, 2 ** 62, 1)
    for (pa, pb, indptr, idx, w, d, port) in prog.realised:
        sim.add_proj(pa, pb, indptr, idx, w, d, port)
    sim.set_state(a, "V_m", np.zeros(300))
    sim.record_v(np.arange(0, 300, 10))
    res = prog.runner().simulate(20.0)
    st, g = prog.plan.spikes()
    ost, og, ov = sim.run(200)
    assert len(st) > 0
    assert _raster(st, g) == _raster(ost, og)
    np.testing.assert_allclose(res[obs]["V_m"], ov, rtol=0, atol=1e-9)


def test_headline_kernel_network_rates_within_1pct_of_oracle(oracle):
    """The headline network at full size (Brunel order 2500, 12 500 neurons,
    15.6 M edges, per-edge delays Uniform(1.0, 3.0) ms on the kernel's
    streams), 3 s simulated: the FP32 and FP64 forms' population rates within
    1 % of the float64 oracle's on the same network (each precision draws its
    delays in its own float width, as the reference does with x64 off / on).
    The library's and the oracle's realisations must be identical."""
    import os
    from oracle import kernel_net as KN
    steps = 30000
    for bits in (32, 64):
        net, p, _ = brunel.build_kernel_network(order=2500)
        prog = net.compile("float64" if bits == 64 else "float32", spike_capacity=1 << 23)
        assert prog.plan.engine == "tiled"
        sim, st = KN.build(p, seed=1234, order=2500, bits=bits)
        for a, b in zip(prog.realised, st["csr"]):
            for x, y in zip(a, b):
                np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
        count = 0
        for _ in range(steps // 10000):
            prog.plan.run(10000)
            count += prog.plan.spikes()[0].size
        prog.plan.close()
        sim.set_threads(os.cpu_count() or 1)
        ref = 0
        for _ in range(steps // 10000):
            ref += sim.run(10000, cap=1 << 21)[0].size
        rate = ref / (p["NE"] + p["NI"]) / (steps * 1e-4)
        assert 20.0 < rate < 60.0   # Hz
        assert abs(count - ref) / ref < 0.01, (bits, count, ref)


def test_batched_trials_fold_the_trial_into_the_drive_keys(oracle):
    """Runner(batch=3): trial 0 is the unbatched run; trial 2's noise comes
    from the step keys with 2 folded in (the oracle run with that trial);
    trials differ; rng='common' repeats trial 0 (_kernel/runner.py:84-113,
    _kernel/rng.py:335-356)."""
    from brainpy.state_b200.kernel import Runner
    from oracle import kernel_net as KN
    order, n = 100, 300
    rec = np.arange(0, 500, 7)
    net, p, _ = brunel.build_kernel_network(order=order)
    obs = net.observe(_view(net, rec), "V_m", name="taps")
    prog = net.compile("float64")
    base = prog.runner().simulate(n * 0.1)[obs]["V_m"]
    run = Runner(prog, batch=3)
    assert run.trials.tolist() == [0, 1, 2]
    v = run.simulate(n * 0.1)[obs]["V_m"]
    assert v.shape == (3,) + base.shape
    np.testing.assert_array_equal(v[0], base)
    assert np.abs(v[1] - v[0]).max() > 1e-3
    sim, _ = KN.build(p, seed=1234, order=order, bits=64)
    sim.set_trial(2)
    sim.record_v(rec)
    _, _, ov = sim.run(n)
    np.testing.assert_allclose(v[2], ov, rtol=0, atol=1e-9)
    common = Runner(prog, batch=2, rng="common").simulate(n * 0.1)[obs]["V_m"]
    np.testing.assert_array_equal(common[0], base)
    np.testing.assert_array_equal(common[1], base)
