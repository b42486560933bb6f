"""Brunel (2000) balanced-network builders used by the benchmark and examples.

Parameters follow the reference's Brunel script (``examples/nest_like/
brunel_alpha.py:32-69`` and ``benchmarks/brunel_simulator_baseline.py:63-131``):
tau_syn 0.5 ms, tau_m 20 ms, C_m 250 pF, theta 20 mV, t_ref 2 ms, g = 5,
eta = 2, epsilon = 0.1, J = 0.1 mV PSP amplitude.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib


def psp_norm(tau_mem, c_mem, tau_syn):
    """Peak PSP of a 1 pA alpha current (brunel_alpha.py:32-38)."""
    from scipy.special import lambertw
    a = tau_mem / tau_syn
    b = 1.0 / tau_syn - 1.0 / tau_mem
    x = -math.exp(-1.0 / a) / a
    lw = lambertw(x, k=-1 if x < 0 else 0).real
    t_max = 1.0 / b * (-lw - 1.0 / a)
    return (math.exp(1.0) / (tau_syn * c_mem * b)
            * ((math.exp(-t_max / tau_mem) - math.exp(-t_max / tau_syn)) / b
               - t_max * math.exp(-t_max / tau_syn)))


def brunel_params(order, g=5.0, eta=2.0, epsilon=0.1, J=0.1, V_reset=10.0):
    tau_syn, tau_mem, c_mem, theta, t_ref = 0.5, 20.0, 250.0, 20.0, 2.0
    NE, NI = 4 * order, order
    CE, CI = int(epsilon * NE), int(epsilon * NI)
    j_ex = J / psp_norm(tau_mem, c_mem, tau_syn)
    nu_th = (theta * c_mem) / (j_ex * CE * math.e * tau_mem * tau_syn)
    rate = 1000.0 * (eta * nu_th) * CE
    neuron = [0.0, c_mem, tau_mem, t_ref, theta, V_reset, tau_syn, tau_syn, 0.0, -math.inf]
    return dict(NE=NE, NI=NI, CE=CE, CI=CI, J_ex=j_ex, J_in=-g * j_ex, rate=rate,
                neuron=neuron, g=g, eta=eta)


def derive_seed(base, ordinal):
    return ((0 if base is None else int(base)) * 1_000_003 + ordinal + 1) & 0x7FFFFFFF


def initial_v(seed, NE, NI, v_init=(0.0, 20.0)):
    """Initial V_m of build_plan's E and I populations (uniform, seeded)."""
    vr = np.random.default_rng(seed + 7)
    return vr.uniform(v_init[0], v_init[1], NE), vr.uniform(v_init[0], v_init[1], NI)


def build_plan(order=2500, precision=32, delay_steps=(10, 30), noise_delay=15, seed=1234,
               semantics=_lib.RING, deterministic=False, rec_v=100, spike_capacity=1 << 23,
               v_init=(0.0, 20.0), g=5.0, eta=2.0, upload=True):
    """Brunel network in one plan.  ``delay_steps``: an int (homogeneous) or a
    (lo, hi) pair of per-edge delays drawn uniformly on the step grid.
    ``upload=False`` stops before the device (the host copy of the structure
    stays readable through ``csr``)."""
    p = brunel_params(order, g=g, eta=eta)
    pl = _lib.Plan(0.1, "iaf_psc_alpha", precision=precision, semantics=semantics,
                   deterministic=deterministic, spike_capacity=spike_capacity)
    e = pl.add_pop(p["NE"], p["neuron"])
    i = pl.add_pop(p["NI"], p["neuron"])
    # creation order as in the reference script: noise -> E, noise -> I,
    # E -> E+I (seed 1), I -> E+I (seed 2)
    pl.add_poisson(e, p["rate"], p["J_ex"], noise_delay, derive_seed(seed, 0))
    pl.add_poisson(i, p["rate"], p["J_ex"], noise_delay, derive_seed(seed, 1))
    rng = np.random.default_rng(seed)
    nbits = 64 if precision == 64 else 32
    ordinal = 2
    for pre, K, w, s in ((e, p["CE"], p["J_ex"], 1), (i, p["CI"], p["J_in"], 2)):
        for post in (e, i):
            n_post = p["NE"] if post == e else p["NI"]
            if isinstance(delay_steps, tuple):
                d = rng.integers(delay_steps[0], delay_steps[1] + 1, size=K * n_post)
                pl.add_fixed_indegree(pre, post, K, derive_seed(s, ordinal), w,
                                      delay_steps=d.astype(np.int32), nbits=nbits)
            else:
                pl.add_fixed_indegree(pre, post, K, derive_seed(s, ordinal), w,
                                      delay_const=int(delay_steps), nbits=nbits)
            ordinal += 1
    N = p["NE"] + p["NI"]
    if rec_v:
        pl.record_v(np.linspace(0, N - 1, rec_v).astype(np.int32))
    if not upload:
        return pl, p
    pl.upload()
    ve, vi = initial_v(seed, p["NE"], p["NI"], v_init)
    pl.set_state(e, "V_m", ve)
    pl.set_state(i, "V_m", vi)
    return pl, p


# ------------------------------------------------- kernel-path network

KERNEL_NAMES = dict(E="E", I="I", noise="noise", noise_proj="noise_EI", e_proj="E_EI",
                    i_proj="I_EI")


def build_kernel_network(order=2500, seed=1234, delay=(1.0, 3.0), noise_delay=1.5, V_reset=10.0,
                         v_init=(0.0, 20.0), g=5.0, eta=2.0, n_rec=0, record_v=False):
    """The Brunel network as the reference's kernel path builds it
    (``_kernel/validation/brunel.py:59-139``, used by
    ``benchmarks/k1a4_delays.py --net brunel``): populations 'E', 'I' and a
    'noise' poisson_generator of one unit per neuron connected one_to_one onto
    E + I (port 'ex', 1.5 ms); 'E_EI' = fixed_indegree(CE) from E onto E + I
    (port 'ex') and 'I_EI' = fixed_indegree(CI) from I (port 'in_') with
    per-edge delays ``Uniform(delay[0] ms, delay[1] ms)`` rounded to the step
    grid (NEST rounding), or a fixed delay when ``delay`` is a number.  The
    neuron parameters are the configuration's (V_reset 10 mV, V_m initialised
    ``Uniform(0, 20) mV``); every random draw comes from the kernel's streams
    for ``seed``.  Returns (Network, params, observers)."""
    from .kernel import Network, fixed_indegree, iaf_psc_alpha, one_to_one, poisson_generator
    from .streams import Uniform
    from .units import Hz, mV, ms, pA, pF
    p = brunel_params(order, g=g, eta=eta, V_reset=V_reset)
    npar = dict(C_m=250.0 * pF, tau_m=20.0 * ms, tau_syn_ex=0.5 * ms, tau_syn_in=0.5 * ms,
                t_ref=2.0 * ms, E_L=0.0 * mV, V_reset=V_reset * mV, V_th=20.0 * mV)
    init = dict(V_m=Uniform(v_init[0] * mV, v_init[1] * mV)) if v_init is not None else None
    net = Network(dt=0.1 * ms, seed=seed)
    E = net.add(iaf_psc_alpha, p["NE"], params=npar, init=init, name=KERNEL_NAMES["E"])
    I = net.add(iaf_psc_alpha, p["NI"], params=npar, init=init, name=KERNEL_NAMES["I"])
    noise = net.add(poisson_generator, p["NE"] + p["NI"], params=dict(rate=p["rate"] * Hz),
                    name=KERNEL_NAMES["noise"])
    net.connect(noise, E + I, one_to_one(), port="ex", weight=p["J_ex"] * pA,
                delay=noise_delay * ms, name=KERNEL_NAMES["noise_proj"])
    d = Uniform(delay[0] * ms, delay[1] * ms) if isinstance(delay, tuple) else delay * ms
    net.connect(E, E + I, fixed_indegree(p["CE"]), port="ex", weight=p["J_ex"] * pA, delay=d,
                name=KERNEL_NAMES["e_proj"])
    net.connect(I, E + I, fixed_indegree(p["CI"]), port="in_", weight=p["J_in"] * pA, delay=d,
                name=KERNEL_NAMES["i_proj"])
    obs = {}
    if n_rec:
        obs["spikes"] = net.observe(E + I, "spike", name="rec_spikes")
    if record_v:
        step = max(1, p["NE"] // 100)
        obs["V_m"] = net.observe(E[::step][:100], "V_m", name="rec_V")
    return net, p, obs


def kernel_out_degree(prog):
    """Out-degree of every library neuron of a compiled kernel network."""
    deg = np.zeros(prog.n_lib, np.int64)
    offs = {}
    g0 = 0
    for q, n in enumerate(prog.plan.pop_sizes):
        offs[q] = g0
        g0 += n
    for a, _, indptr, _, _, _, _ in prog.realised:
        deg[offs[a]:offs[a] + indptr.size - 1] += np.diff(indptr)
    return deg


# ------------------------------------------------------------ sweep batches

def sweep_instances(n=256, seed=1234, ne_range=(500, 8000), g_range=(3.0, 8.0),
                    eta_range=(0.9, 4.0), delay_steps=15):
    """Parameter sweep of Brunel networks: NE ~ U[ne_range] (NI = NE / 4,
    epsilon = 0.1), g ~ U[g_range], eta ~ U[eta_range], instance k seeded k."""
    rng = np.random.default_rng(seed)
    ne = rng.integers(ne_range[0], ne_range[1] + 1, size=n)
    g = rng.uniform(*g_range, size=n)
    eta = rng.uniform(*eta_range, size=n)
    return [dict(NE=int(ne[k]), NI=int(ne[k]) // 4, g=float(g[k]), eta=float(eta[k]), seed=k,
                 delay_steps=delay_steps) for k in range(n)]


def _instance_params(spec):
    p = brunel_params(2500, g=spec["g"], eta=spec["eta"])
    NE, NI = spec["NE"], spec["NI"]
    p.update(NE=NE, NI=NI, CE=int(0.1 * NE), CI=int(0.1 * NI))
    # the drive rate eta * nu_th * CE does not depend on CE (nu_th ~ 1 / CE)
    return p


def _instance_v0(spec, v_init=(0.0, 20.0)):
    vr = np.random.default_rng(spec["seed"] + 7)
    return (vr.uniform(v_init[0], v_init[1], spec["NE"]),
            vr.uniform(v_init[0], v_init[1], spec["NI"]))


def _instance_projs(spec, p):
    """(pre, post, K, seed, weight) in creation order: E->E, E->I, I->E, I->I."""
    out, ordinal = [], 2
    for pre, K, w in ((0, p["CE"], p["J_ex"]), (1, p["CI"], p["J_in"])):
        for post in (0, 1):
            out.append((pre, post, K, derive_seed(spec["seed"], ordinal), w))
            ordinal += 1
    return out


def build_batch(instances, precision=32, semantics=_lib.RING, tile=0, ctas_per_sm=0,
                record=(), noise_delay=15):
    """All sweep instances in one ``Batch`` (connectivity drawn on the GPU)."""
    b = _lib.Batch(0.1, "iaf_psc_alpha", precision=precision, semantics=semantics)
    params = []
    for spec in instances:
        p = _instance_params(spec)
        params.append(p)
        k = b.add_instance()
        e = b.add_pop(k, p["NE"], p["neuron"])
        i = b.add_pop(k, p["NI"], p["neuron"])
        b.add_poisson(k, e, p["rate"], p["J_ex"], noise_delay, derive_seed(spec["seed"], 0))
        b.add_poisson(k, i, p["rate"], p["J_ex"], noise_delay, derive_seed(spec["seed"], 1))
        for pre, post, K, s, w in _instance_projs(spec, p):
            b.add_fixed_indegree(k, pre, post, K, s, w, spec["delay_steps"], nbits=32)
        if k in record:
            b.record_spikes(k)
    b.upload(tile=tile, ctas_per_sm=ctas_per_sm)
    for k, spec in enumerate(instances):
        ve, vi = _instance_v0(spec)
        b.set_state(k, 0, "V_m", ve)
        b.set_state(k, 1, "V_m", vi)
    return b, params


def instance_plan(spec, precision=64, semantics=_lib.RING, deterministic=False,
                  noise_delay=15, spike_capacity=1 << 22):
    """One sweep instance as a stand-alone plan (host-drawn connectivity,
    the same seeds and 32-bit draws as ``build_batch``)."""
    p = _instance_params(spec)
    pl = _lib.Plan(0.1, "iaf_psc_alpha", precision=precision, semantics=semantics,
                   deterministic=deterministic, spike_capacity=spike_capacity)
    e = pl.add_pop(p["NE"], p["neuron"])
    i = pl.add_pop(p["NI"], p["neuron"])
    pl.add_poisson(e, p["rate"], p["J_ex"], noise_delay, derive_seed(spec["seed"], 0))
    pl.add_poisson(i, p["rate"], p["J_ex"], noise_delay, derive_seed(spec["seed"], 1))
    for pre, post, K, s, w in _instance_projs(spec, p):
        pl.add_fixed_indegree(pre, post, K, s, w, delay_const=spec["delay_steps"], nbits=32)
    pl.upload()
    ve, vi = _instance_v0(spec)
    pl.set_state(e, "V_m", ve)
    pl.set_state(i, "V_m", vi)
    return pl, p
