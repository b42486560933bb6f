"""The kernel front end realises networks on the reference kernel path's
streams: the library's realisation (brainpy.state_b200.kernel, host only)
must equal the oracle's independent one (oracle/kernel_net.py) bit for bit --
connectivity in the rule's canonical order, per-edge delays drawn from the
projection's DELAY stream and rounded the NEST way, initial V_m from each
population's INIT stream, and the drive units of the noise device.
"""
import numpy as np
import pytest

from brainpy.state_b200 import brunel, streams
from brainpy.state_b200.units import ms


def test_delay_steps_reference_examples():
    # _kernel/delays.py:85-86: [0.0, 0.04, 0.05, 0.15, 1.5] ms at dt 0.1 ms
    d = np.array([0.0, 0.04, 0.05, 0.15, 1.5])
    assert streams.delay_steps(d, 0.1, 64).tolist() == [0, 0, 1, 2, 15]
    # the same decimals stored in float32 round half up as NEST does
    d32 = d.astype(np.float32).astype(np.float64)
    assert streams.delay_steps(d32, 0.1, 32).tolist() == [0, 0, 1, 2, 15]
    # 0.35 ms is 0.3499999940 in float32: still 4 steps (the docstring's case)
    assert streams.delay_steps(np.float32(0.35).astype(np.float64)[None], 0.1, 32).tolist() == [4]


def test_name_key_and_object_key_follow_the_key_chain(oracle):
    from oracle import kernel_net as KN
    for name in ("E", "I", "noise", "E_EI"):
        a = streams.object_key(1234, name)
        b = KN.object_key(1234, name)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(streams.name_key(a, "V_m"), KN.name_key(b, "V_m"))


@pytest.mark.parametrize("bits", [32, 64])
def test_kernel_brunel_realisation_equals_oracle(oracle, bits):
    from oracle import kernel_net as KN
    net, p, _ = brunel.build_kernel_network(order=500)
    prog = net.compile("float64" if bits == 64 else "float32", upload=False)
    _, st = KN.build(p, seed=1234, order=500, bits=bits)
    assert len(prog.realised) == len(st["csr"]) == 4
    for a, b in zip(prog.realised, st["csr"]):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
    neurons = [q for q in net.populations if not q.is_device]
    for q, pop in enumerate(neurons):
        np.testing.assert_array_equal(prog.initial_v(pop), st["v0"][q])
    assert [(d[0], d[5]) for d in prog.drives] == st["drives"]
    delays = np.concatenate([r[5] for r in prog.realised])
    assert delays.min() == 10 and delays.max() == 30


def test_distributed_weights_follow_the_weight_stream():
    from brainpy.state_b200.kernel import (Network, fixed_indegree, iaf_psc_alpha, Normal,
                                           Uniform)
    from brainpy.state_b200.units import pA
    net = Network(dt=0.1 * ms, seed=7)
    A = net.add(iaf_psc_alpha, 300, name="A")
    proj = net.connect(A, A, fixed_indegree(20), port="ex", weight=Uniform(1.0 * pA, 5.0 * pA),
                       delay=Uniform(1.0 * ms, 2.0 * ms), name="AA")
    net.connect(A, A, fixed_indegree(5), port="in_", weight=Normal(-3.0 * pA, 0.5 * pA, high=0.0 * pA),
                name="AA_in")
    prog = net.compile("float32", upload=False)
    okey = streams.object_key(7, "AA")
    w_ref = np.clip(streams._lib.jax_uniform(streams.fold_in(okey, streams.WEIGHT_STREAM), 6000,
                                             32, 1.0, 5.0), 1.0, 5.0)
    # realised CSR holds the canonical-order draws permuted by the stable pre sort
    from brainpy.state_b200.kernel import realise_positions
    src, dst = realise_positions(net, proj)
    order = np.argsort(src, kind="stable")
    np.testing.assert_array_equal(prog.realised[0][4], w_ref[order])
    w_in = prog.realised[1][4]
    assert np.all(w_in <= 0.0) and abs(w_in.mean() + 3.0) < 0.1
