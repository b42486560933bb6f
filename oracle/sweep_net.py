"""One instance of the batched Brunel sweep built by the oracle alone --
TEST INFRASTRUCTURE ONLY (tests/, the CPU legs of bench.py).

An instance is Brunel model A with NE excitatory and NE / 4 inhibitory
iaf_psc_alpha neurons, in-degrees 10 %, its own g and eta, a homogeneous
delay, and seeds derived from the instance seed with the reference
Simulator's formula (seed * 1000003 + ordinal + 1) & 0x7fffffff
(_nest_network/simulator.py:926-935): ordinals 0 and 1 for the E and I
drives, 2..5 for E->E, E->I, I->E, I->I (the library's batch and stand-alone
plans use the same).  Connectivity is the legacy fixed_indegree sampler with
32-bit draws (_nest_network/connectivity.py:101-135) and the CSR by stable
pre sort (:39-53); the drives are the library's counter stream; V_m ~
U[0, 20) mV from numpy's generator seeded instance seed + 7 (the library's
choice for the sweep, which the configuration leaves open).
"""
from __future__ import annotations

import numpy as np

from . import kernel_net as KN
from . import oracle as O


def derive_seed(base, ordinal):
    return (int(base) * 1_000_003 + ordinal + 1) & 0x7FFFFFFF


def build(spec, noise_delay=15, threads=1):
    """OracleSim of sweep instance ``spec`` (NE, NI, g, eta, seed,
    delay_steps) with RING timing; returns (sim, params)."""
    p = KN.brunel_params(2500, g=spec["g"], eta=spec["eta"])
    NE, NI = spec["NE"], spec["NI"]
    p.update(NE=NE, NI=NI, CE=int(0.1 * NE), CI=int(0.1 * NI))
    sim = O.OracleSim(0.1, "iaf_psc_alpha", semantics=O.RING)
    sim.set_threads(threads)
    e = sim.add_pop(NE, p["neuron"])
    i = sim.add_pop(NI, p["neuron"])
    sim.add_drive(e, p["rate"], p["J_ex"], noise_delay, derive_seed(spec["seed"], 0))
    sim.add_drive(i, p["rate"], p["J_ex"], noise_delay, derive_seed(spec["seed"], 1))
    ordinal = 2
    for pre, K, w in ((e, p["CE"], p["J_ex"]), (i, p["CI"], p["J_in"])):
        for post in (e, i):
            n_pre, n_post = (NE if pre == e else NI), (NE if post == e else NI)
            src, dst = O.fixed_indegree(derive_seed(spec["seed"], ordinal), n_pre, n_post, K,
                                        pre_is_post=pre == post, allow_autapses=True, nbits=32)
            _, idx, indptr = O.csr_structure(src, dst, n_pre)
            sim.add_proj(pre, post, indptr, idx, np.full(idx.size, float(w)),
                         np.full(idx.size, int(spec["delay_steps"]), np.int32))
            ordinal += 1
    vr = np.random.default_rng(spec["seed"] + 7)
    sim.set_state(e, "V_m", vr.uniform(0.0, 20.0, NE))
    sim.set_state(i, "V_m", vr.uniform(0.0, 20.0, NI))
    return sim, p
