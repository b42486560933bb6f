"""Mirror a facade Simulator's realised network into the float64 oracle --
TEST INFRASTRUCTURE ONLY (tests/ and the parity sections of bench.py).

The Simulator's deferred operations are replayed in creation order: drives
with their seeds and windows, every projection with the CSR the library
realised (read back from the uploaded plan's host copy, so connectivity and
distributed weights are the library's; their own parity is tested
elsewhere), plasticity with the synapse spec's parameters, and the initial
V_m the plan was given.  Call it after ``sim.simulate(0 ms)`` (the network
built and initialised, no step taken).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def from_simulator(sim, threads=1):
    """(OracleSim, oracle input ids of the projections in plan order)."""
    pl = sim._plan
    sem = O.LEGACY if sim.delivery == "legacy" else O.RING
    osim = O.OracleSim(sim.dt, sim._model.model_name, semantics=sem)
    osim.set_threads(threads)
    for p in sim._pops:
        osim.add_pop(p.n, p.params)
    proj_ids = []
    j = 0
    for op in sim._ops:
        if op[0] == "drive":
            _, pop, rate, w, d, seed, t_min, t_max, rec = op
            osim.add_drive(pop, rate, w, d, seed, t_min, t_max, rec)
            continue
        syn, rec = op[-1], op[-2]
        a, b = op[1], op[2]
        indptr, post, d, w0 = pl.csr(j)
        oid = osim.add_proj(a, b, indptr, post, w0, d, rec)
        proj_ids.append(oid)
        if syn is not None:
            if hasattr(syn, "taus"):
                t = syn.taus
                osim.set_stdp_triplet(oid, t["tau_plus"], t["tau_plus_triplet"], t["tau_minus"],
                                      t["tau_minus_triplet"], syn.Aplus, syn.Aplus_triplet,
                                      syn.Aminus, syn.Aminus_triplet, syn.Wmax)
            else:
                osim.set_stdp(oid, syn.tau_plus, syn.tau_minus, syn.lambda_, syn.alpha,
                              syn.mu_plus, syn.mu_minus, syn.Wmax)
        j += 1
    for p in sim._pops:
        osim.set_state(p.pop_id, "V_m", np.asarray(pl.get_state(p.pop_id, "V_m"), np.float64))
    return osim, proj_ids
