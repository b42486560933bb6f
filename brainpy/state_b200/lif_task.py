"""Gradient-training workload: a recurrent iaf_psc_exp network driven by
Poisson input channels, trained so that the exponentially filtered rates of
its first neurons follow target sinusoids.

All arrays are numpy (host); ``seed`` fixes everything.  Sizes default to
800 E + 200 I neurons, 10 % random recurrent connectivity (no self
connections) with weights N(0, (0.5 pA)^2) / fan-in, Dale-signed by the
pre neuron (E positive, I negative), 100 input channels at rates U[5, 50] Hz
into every neuron with half-normal weights of scale 900 pA / sqrt(100), batch
64, 1000 steps of dt = 1 ms, 10 readout neurons filtered with tau = 20 ms,
targets 10 * (1 + sin(2 pi f t + phi)) Hz with f ~ U[1, 5] Hz, phi ~ U[0, 2 pi).
The neuron parameters are NEST's iaf_psc_exp defaults.
"""
from __future__ import annotations

import math

import numpy as np

# E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in I_e
IAF_PSC_EXP_DEFAULTS = [-70.0, 250.0, 10.0, 2.0, -55.0, -70.0, 2.0, 2.0, 0.0]


def make_task(n_exc=800, n_inh=200, n_in=100, batch=64, n_steps=1000, dt=1.0, p_conn=0.1,
              w_std=0.5, w_in_scale=900.0, rate_range=(5.0, 50.0), n_readout=10,
              readout_tau=20.0, slope=25.0, seed=1234, params=None, relaxed=False,
              detach_reset=False):
    rng = np.random.default_rng(seed)
    n = n_exc + n_inh
    # recurrent structure, rows = post neurons, columns (pre) ascending
    mask = rng.random((n, n)) < p_conn
    np.fill_diagonal(mask, False)
    row_ptr = np.concatenate([[0], np.cumsum(mask.sum(1))]).astype(np.int64)
    col = np.nonzero(mask)[1].astype(np.int32)
    fan_in = np.maximum(np.diff(row_ptr), 1)
    post = np.repeat(np.arange(n), np.diff(row_ptr))
    mag = np.abs(rng.normal(0.0, w_std, col.size)) / np.sqrt(fan_in[post])
    w = np.where(col < n_exc, mag, -mag)
    w_in = np.abs(rng.normal(0.0, w_in_scale / math.sqrt(n_in), (n, n_in)))
    rates = rng.uniform(rate_range[0], rate_range[1], n_in)
    lam = rates * dt * 1e-3
    inputs = rng.poisson(lam[None, None, :], (n_steps, batch, n_in)).astype(np.uint8)
    f = rng.uniform(1.0, 5.0, (batch, n_readout))
    phi = rng.uniform(0.0, 2 * math.pi, (batch, n_readout))
    t = (np.arange(n_steps) * dt * 1e-3)[:, None, None]
    targets = 10.0 * (1.0 + np.sin(2 * math.pi * f[None] * t + phi[None]))
    cfg = dict(dt=dt, n=n, n_in=n_in, batch=batch, n_steps=n_steps, n_readout=n_readout,
               readout_tau=readout_tau, slope=slope, relaxed=int(relaxed),
               detach_reset=int(detach_reset),
               params=list(params if params is not None else IAF_PSC_EXP_DEFAULTS))
    return dict(cfg=cfg, row_ptr=row_ptr, col=col, w=w, w_in=w_in, inputs=inputs,
                targets=targets, n_exc=n_exc)
