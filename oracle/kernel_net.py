"""The reference kernel path's Brunel network built by the oracle alone --
TEST INFRASTRUCTURE ONLY (tests/, the CPU legs of bench.py).

Every structure is realised from the oracle's own restatements of the
reference's streams, with no call into the product library:

* populations 'E', 'I'; device 'noise' (one poisson_generator unit per
  neuron) one_to_one onto E + I, port 'ex'; 'E_EI' fixed_indegree(CE) from E
  onto E + I (port 'ex'), 'I_EI' fixed_indegree(CI) from I (port 'in_')
  (_kernel/validation/brunel.py:59-139);
* sources: the kernel's per-post key chain and randint
  (_kernel/connectivity/rules.py:226-265, _kernel/rng.py:237-300), edges in
  the rule's canonical order, post-major and pre ascending (rules.py:83-88);
* per-edge delays Uniform(lo ms, hi ms) from fold(object_key, DELAY_STREAM)
  (_kernel/compiler.py:95-97,841-850), rounded to steps the NEST way
  (_kernel/delays.py:50-98);
* initial V_m Uniform(v0, v1) mV from name_key(fold(object_key(E or I),
  INIT_STREAM), 'V_m') (_kernel/compiler.py:819, _kernel/params.py:348-354);
* the noise counts from the device population's block keys
  (_kernel/models/devices.py:46-145, _kernel/rng.py:338-420).
"""
from __future__ import annotations

import math
import zlib

import numpy as np

from . import oracle as O

INIT_STREAM = 0xFFFFFFFE
DELAY_STREAM = 0xFFFFFFFC


def psp_norm(tau_mem, c_mem, tau_syn):
    """PSC amplitude (pA) of a 1 mV alpha-PSP peak
    (_kernel/validation/brunel.py:25-36)."""
    from scipy.special import lambertw
    a = tau_mem / tau_syn
    b = 1.0 / tau_syn - 1.0 / tau_mem
    x = -math.exp(-1.0 / a) / a
    t_max = 1.0 / b * (-lambertw(x, k=-1 if x < 0 else 0).real - 1.0 / a)
    return (math.exp(1.0) / (tau_syn * c_mem * b)
            * ((math.exp(-t_max / tau_mem) - math.exp(-t_max / tau_syn)) / b
               - t_max * math.exp(-t_max / tau_syn)))


def brunel_params(order, g=5.0, eta=2.0, epsilon=0.1, V_reset=10.0):
    """Sizes, in-degrees, weights (pA) and Poisson rate (Hz) of Brunel model A
    (_kernel/validation/brunel.py:39-56); neuron parameters in the library's
    iaf_psc_alpha order (E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in
    I_e V_min) with the configuration's V_reset."""
    ne, ni = 4 * order, order
    ce, ci = int(epsilon * ne), int(epsilon * ni)
    tau_syn, tau_mem, c_mem, theta = 0.5, 20.0, 250.0, 20.0
    j_ex = 0.1 / psp_norm(tau_mem, c_mem, tau_syn)
    nu_th = (theta * c_mem) / (j_ex * ce * math.exp(1) * tau_mem * tau_syn)
    return dict(NE=ne, NI=ni, CE=ce, CI=ci, J_ex=j_ex, J_in=-g * j_ex,
                rate=1000.0 * eta * nu_th * ce,
                neuron=[0.0, c_mem, tau_mem, 2.0, theta, V_reset, tau_syn, tau_syn, 0.0, -math.inf])


def object_key(seed, name):
    hi, lo = O.name_id(name)
    return O.jax_fold_in(O.jax_fold_in(O.jax_key(seed), hi), lo)


def name_key(key, name):
    return O.jax_fold_in(key, zlib.crc32(name.encode()) & 0x7FFFFFFF)


def delay_steps(d_ms, dt_ms, bits):
    """_kernel/delays.py:50-98: floor(d * steps_per_ms + 0.5) in float64;
    float32 inputs within 8 eps32 * max(y, 1) of an integer y snap to it."""
    d = np.asarray(d_ms, np.float64)
    spm = 1.0 / dt_ms
    k = np.rint(spm)
    if k >= 1 and abs(spm - k) <= 1e-6 * k:
        spm = k
    y = d * spm + 0.5
    out = np.floor(y)
    if bits == 32:
        eps = float(np.finfo(np.float32).eps)
        out = np.where(np.abs(y - np.rint(y)) <= 8 * eps * np.maximum(y, 1.0), np.rint(y), out)
    return out.astype(np.int64)


def uniform_dist(key, n, bits, lo, hi):
    """The kernel's Uniform(lo, hi).sample: jax.random.uniform(key, (n,), dtype,
    lo, hi), then clip to [lo, hi] (_kernel/params.py:251-285)."""
    t = np.float32 if bits == 32 else np.float64
    u = O.jax_uniform(key, n, bits, lo, hi).astype(t)
    return np.clip(u, t(lo), t(hi)).astype(np.float64)


def build(params, seed=1234, order=2500, delay=(1.0, 3.0), noise_delay_steps=15, bits=32,
          v_init=(0.0, 20.0), dt=0.1):
    """Returns (OracleSim, structure): ``params`` as brunel_params gives them
    (NE, NI, CE, CI, J_ex, J_in, rate, neuron); structure holds the CSR of
    every (pre, post) pair in creation order, the initial V_m, the drives."""
    NE, NI, CE, CI = params["NE"], params["NI"], params["CE"], params["CI"]
    N = NE + NI
    sim = O.OracleSim(dt, "iaf_psc_alpha", semantics=O.RING)
    sim.set_ports(True)
    e = sim.add_pop(NE, params["neuron"])
    i = sim.add_pop(NI, params["neuron"])
    st = {"csr": [], "v0": [], "drives": []}
    # creation order of the kernel network: noise_EI, E_EI, I_EI
    okey = object_key(seed, "noise")
    for pop, u0 in ((e, 0), (i, NE)):
        sim.add_drive_keyed(pop, params["rate"], params["J_ex"], noise_delay_steps, okey, u0,
                            0, 2 ** 62, 0)
        st["drives"].append((pop, u0))
    parts = [("E", np.arange(NE)), ("I", np.arange(NI))]
    for name, pre_pop, n_pre, K, w, port in (("E_EI", e, NE, CE, params["J_ex"], 0),
                                             ("I_EI", i, NI, CI, params["J_in"], 1)):
        src = O.kernel_fixed_indegree(seed, name, parts, n_pre, None, K).reshape(-1)
        dst = np.repeat(np.arange(N, dtype=np.int64), K)
        order = np.lexsort((src, dst))
        src, dst = src[order], dst[order]
        E = src.size
        if isinstance(delay, tuple):
            dk = O.jax_fold_in(object_key(seed, name), DELAY_STREAM)
            ds = delay_steps(uniform_dist(dk, E, bits, delay[0], delay[1]), dt, bits)
        else:
            ds = np.full(E, int(delay), np.int64)
        for post_pop, lo, hi in ((e, 0, NE), (i, NE, N)):
            m = (dst >= lo) & (dst < hi)
            p_, q_, d_ = src[m], dst[m] - lo, ds[m]
            ordr = np.argsort(p_, kind="stable")
            indptr = np.concatenate([[0], np.cumsum(np.bincount(p_, minlength=n_pre))])
            idx, dd = q_[ordr].astype(np.int32), d_[ordr].astype(np.int32)
            ww = np.full(idx.size, float(w))
            sim.add_proj(pre_pop, post_pop, indptr.astype(np.int64), idx, ww, dd, port)
            st["csr"].append((pre_pop, post_pop, indptr.astype(np.int64), idx, ww, dd, port))
    for pop, name, n in ((e, "E", NE), (i, "I", NI)):
        k = name_key(O.jax_fold_in(object_key(seed, name), INIT_STREAM), "V_m")
        v = uniform_dist(k, n, bits, v_init[0], v_init[1])
        sim.set_state(pop, "V_m", v)
        st["v0"].append(v)
    return sim, st
