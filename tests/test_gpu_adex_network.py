"""The AdEx conductance network with plasticity at full size (16 000 E +
4 000 I aeif_cond_alpha, 2 000 lognormal conductance inputs each, 25.6 M
plastic E->E stdp_synapse edges, 5 kHz drive), built through the Simulator
API: size-independent properties of a 50 ms run (the float64 oracle cannot
run it in a test's time).  FP64 parity of the same engine on small networks
is in test_gpu_aeif_stdp.py."""
import numpy as np
import pytest

from brainpy.state_b200 import adex_net
from brainpy.state_b200.units import ms

pytestmark = pytest.mark.gpu


def test_full_size_adex_stdp_network_runs_and_keeps_weights_bounded():
    sim, h = adex_net.build(scale=1.0, precision=32, drive_nS=6.0)
    res = sim.simulate(50.0 * ms)
    n = h["NE"] + h["NI"]
    assert h["CE"] == 1600 and h["CI"] == 400        # 2 000 inputs per neuron
    ee = h["ee"]
    assert ee.n_edges == 16000 * 1600               # 25.6 M plastic edges
    spikes = res.spikes(h["rec"])
    assert spikes.shape == (500, n)
    assert spikes.sum() > 0
    w = sim._plan.weights(ee.proj_id)
    indptr, post, d, w0 = sim._plan.csr(ee.proj_id)
    assert np.all(np.isfinite(w)) and np.all(w >= 0.0)
    changed = w != w0
    assert changed.sum() > 1000                      # the rule acted
    # facilitation stops at Wmax, depression at 0: a changed weight never
    # leaves [0, max(w0, Wmax)]
    assert np.all(w[changed] <= np.maximum(w0[changed], h["Wmax"]) + 1e-12)


def test_scaled_adex_stdp_network_fp32_rate_close_to_oracle(oracle):
    """The same network at scale 0.05 (800 E + 200 I, in-degrees 80 + 20),
    FP32 stages with FP64 error control and FP64 plastic weights, against the
    float64 oracle on the identical realised network (oracle/mirror.py), 500 ms:
    population rates within 5 % (the network is chaotic: trajectories separate,
    the rate does not) and mean plastic weight within 2 %."""
    import os
    from oracle import mirror
    sim, h = adex_net.build(scale=0.05, precision=32)
    sim.simulate(0.0 * ms)
    osim, pids = mirror.from_simulator(sim, threads=os.cpu_count() or 1)
    res = sim.cont(500.0 * ms)
    count = float(res.spikes(h["rec"]).sum())
    ref = osim.run(5000, cap=1 << 22)[0].size
    assert ref > 100
    assert abs(count - ref) / ref < 0.05, (count, ref)
    w = sim._plan.weights(h["ee"].proj_id)
    w_ref = osim.weights(pids[0], w.size)
    assert abs(w.mean() - w_ref.mean()) / w_ref.mean() < 0.02
