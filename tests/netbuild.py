"""Build the same network into the CUDA plan and the CPU oracle (tests only)."""
from __future__ import annotations

import math

import numpy as np

from brainpy.state_b200 import _lib

ALPHA_ORDER = ["E_L", "C_m", "tau_m", "t_ref", "V_th", "V_reset", "tau_syn_ex", "tau_syn_in",
               "I_e", "V_min"]


def brunel_alpha_params(V_reset=10.0):
    return dict(E_L=0.0, C_m=250.0, tau_m=20.0, t_ref=2.0, V_th=20.0, V_reset=V_reset,
                tau_syn_ex=0.5, tau_syn_in=0.5, I_e=0.0, V_min=-math.inf)


def random_csr(rng, n_pre, n_post, K, w, delays, self_ok=True):
    """fixed in-degree K with multapses, CSR by stable pre sort."""
    pre = rng.integers(0, n_pre, size=(n_post, K)).reshape(-1)
    post = np.repeat(np.arange(n_post), K)
    order = np.argsort(pre, kind="stable")
    indptr = np.concatenate([[0], np.cumsum(np.bincount(pre, minlength=n_pre))]).astype(np.int64)
    d = np.broadcast_to(np.asarray(delays), pre.shape)[order] if np.ndim(delays) else \
        np.full(pre.size, int(delays))
    return indptr, post[order].astype(np.int32), np.full(pre.size, float(w)), d.astype(np.int32)


class Net:
    """Small Brunel-style network description (pops, projections, drives)."""

    def __init__(self, NE=200, NI=50, CE=20, CI=5, J=20.68, g=5.0, delay=15, rate=17789.0,
                 seed=5, per_edge_delay=None, dt=0.1, V_reset=10.0, model="iaf_psc_alpha"):
        rng = np.random.default_rng(seed)
        if model == "iaf_psc_exp":
            J = J * math.e  # same charge per spike as the alpha kernel
        self.dt = dt
        self.model = model
        p = brunel_alpha_params(V_reset)
        order = ALPHA_ORDER if model == "iaf_psc_alpha" else ALPHA_ORDER[:-1]
        self.params = [p[k] for k in order]
        self.NE, self.NI = NE, NI
        self.v0 = rng.uniform(0.0, 20.0, NE + NI)
        self.projs = []
        for pre, K, w in ((0, CE, J), (1, CI, -g * J)):
            for post in (0, 1):
                n_pre = NE if pre == 0 else NI
                n_post = NE if post == 0 else NI
                if per_edge_delay is not None:
                    lo, hi = per_edge_delay
                    dl = rng.integers(lo, hi + 1, size=n_post * K)
                else:
                    dl = delay
                self.projs.append((pre, post) + random_csr(rng, n_pre, n_post, K, w, dl))
        self.drives = [(0, rate, J, delay, 101), (1, rate, J, delay, 102)]

    def to_plan(self, precision=64, semantics=0, deterministic=False, rec=None):
        pl = _lib.Plan(self.dt, self.model, precision=precision, semantics=semantics,
                       deterministic=deterministic)
        e = pl.add_pop(self.NE, self.params)
        i = pl.add_pop(self.NI, self.params)
        # creation order: drives first (as in the reference Brunel script)
        for post, rate, w, d, seed in self.drives:
            pl.add_poisson(post, rate, w, d, seed)
        for pre, post, indptr, idx, w, d in self.projs:
            pl.add_csr(pre, post, indptr, idx, w, d)
        if rec is not None:
            pl.record_v(rec)
        pl.upload()
        pl.set_state(e, "V_m", self.v0[:self.NE])
        pl.set_state(i, "V_m", self.v0[self.NE:])
        return pl

    def to_oracle(self, oracle, semantics=0, rec=None):
        sim = oracle.OracleSim(self.dt, self.model, semantics=semantics)
        e = sim.add_pop(self.NE, self.params)
        i = sim.add_pop(self.NI, self.params)
        for post, rate, w, d, seed in self.drives:
            sim.add_drive(post, rate, w, d, seed)
        for pre, post, indptr, idx, w, d in self.projs:
            sim.add_proj(pre, post, indptr, idx, w, d)
        if rec is not None:
            sim.record_v(rec)
        sim.set_state(e, "V_m", self.v0[:self.NE])
        sim.set_state(i, "V_m", self.v0[self.NE:])
        return sim
