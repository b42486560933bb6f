"""The AdEx conductance network with plasticity, built through the Simulator
API: 16 000 E + 4 000 I ``aeif_cond_alpha`` (NEST defaults), fixed in-degree
of 10 % of each population (1 600 E + 400 I = 2 000 inputs), lognormal
conductance weights (mu = ln 1 nS, sigma = 0.5), E->E as ``stdp_synapse``
(tau_plus 20 ms, lambda 0.01, alpha 1, mu_plus = mu_minus = 1, Wmax = 3 x the
mean initial weight), an independent 5 kHz Poisson drive per neuron, adaptive
RKF45 with tolerance 1e-6.  Excitatory inputs go to g_ex, inhibitory ones to
g_in.  ``scale`` shrinks both populations (and so the in-degrees) for tests.
"""
from __future__ import annotations

import math

from .simulator import (LogNormal, Simulator, Uniform, aeif_cond_alpha, fixed_indegree,
                        poisson_generator, spike_recorder, stdp_synapse)
from .units import Hz, mV, ms, nS

WEIGHT_MU, WEIGHT_SIGMA = 0.0, 0.5          # ln nS
MEAN_WEIGHT = math.exp(WEIGHT_MU + 0.5 * WEIGHT_SIGMA ** 2)


def build(scale=1.0, precision=32, drive_nS=6.0, delay_ms=1.5, drive_hz=5000.0, plastic=True,
          n_record=None):
    """(Simulator, handles) with E, I, the E->E projection handle and a spike
    recorder on every neuron (or on the first n_record E neurons).

    The drive weight is not part of the configuration; 6 nS is the smallest
    of those tried (1, 2, 4, 6, 8, 10 nS) that makes the network fire.  From
    V_m ~ U[-70.6, -60) mV it then bursts at ~300 Hz for its first
    milliseconds, the E->E rule depresses those weights, and the rate falls."""
    sim = Simulator(dt=0.1 * ms, precision=precision)
    NE, NI = int(round(16000 * scale)), int(round(4000 * scale))
    vinit = Uniform(-70.6 * mV, -60.0 * mV)
    E = sim.create(aeif_cond_alpha, NE, params=dict(V_initializer=vinit))
    I = sim.create(aeif_cond_alpha, NI, params=dict(V_initializer=vinit))
    noise = sim.create(poisson_generator, rate=drive_hz * Hz)
    for pop in (E, I):
        sim.connect(noise, pop, weight=drive_nS * nS, delay=delay_ms * ms, receptor_type=1)
    CE, CI = max(1, NE // 10), max(1, NI // 10)
    w = LogNormal(WEIGHT_MU, WEIGHT_SIGMA)
    syn = stdp_synapse(weight=1.0, delay=delay_ms, tau_plus=20.0, tau_minus=20.0, lambda_=0.01,
                       alpha=1.0, mu_plus=1.0, mu_minus=1.0, Wmax=3.0 * MEAN_WEIGHT)
    ee = sim.connect(E, E, rule=fixed_indegree(CE), weight=w, delay=delay_ms * ms,
                     receptor_type=1, synapse=syn if plastic else None, seed=1)
    sim.connect(E, I, rule=fixed_indegree(CE), weight=w, delay=delay_ms * ms, receptor_type=1,
                seed=2)
    for post, s in ((E, 3), (I, 4)):
        sim.connect(I, post, rule=fixed_indegree(CI), weight=w, delay=delay_ms * ms,
                    receptor_type=2, seed=s)
    rec = sim.create(spike_recorder)
    sim.connect(E + I if n_record is None else E[:n_record], rec)
    return sim, dict(E=E, I=I, ee=ee, rec=rec, NE=NE, NI=NI, CE=CE, CI=CI,
                     Wmax=3.0 * MEAN_WEIGHT)
