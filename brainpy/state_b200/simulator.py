"""NEST-style ``Simulator`` facade over libbspk (create / connect / simulate / cont).

Mirrors the reference's public API (``_nest_network/simulator.py:417-1883``):
populations are created with NEST parameter names, generators are realised
per target at ``connect`` (``simulator.py:1437-1463``), every realised
projection gets its own seed ``(seed * 1_000_003 + ordinal + 1) & 0x7FFFFFFF``
(``simulator.py:926-935``), recorders tap populations, and ``simulate`` /
``cont`` return a :class:`SimulationResult` with ``(T, n_rec)`` spike and
analog arrays.  The network step itself runs in libbspk's CUDA kernels; this
module only translates the description.

Differences from the reference, by design:

* one neuron model per Simulator (the kernels are specialised per model);
* ``delivery='legacy'`` (default) keeps the Simulator's timing (a spike of
  step m arrives at step m + D + 1); ``delivery='nest'`` uses the kernel /
  NEST ring timing (arrival at n + d) and accepts per-edge delay
  distributions;
* the Poisson drive uses the library's counter-based stream, not
  ``jax.random.poisson``.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

from . import _lib
from . import streams as _streams
from .units import Hz, Quantity, mV, ms, nS, pA, pF, mantissa

# ----------------------------------------------------------------- models


class _Model:
    kind = "neuron"
    model_name = ""
    order: tuple = ()
    units: dict = {}
    defaults: dict = {}
    conductance = False   # weights in nS into receptor ports, RKF45 per-step engine
    v_init_const = None   # default V_m when the model's V_initializer is a constant

    @classmethod
    def resolve(cls, params):
        vals = dict(cls.defaults)
        for k, v in (params or {}).items():
            if k in ("V_initializer", "w_initializer", "g_ex_initializer", "g_in_initializer"):
                continue
            if k not in cls.units:
                raise TypeError(f"{cls.__name__} got an unexpected parameter {k!r}")
            vals[k] = v
        out = []
        for k in cls.order:
            v = vals[k]
            if v is None:
                out.append(-math.inf)
                continue
            m = mantissa(v, cls.units[k])
            if np.ndim(m) != 0:
                raise NotImplementedError(f"per-neuron arrays for {k!r} are not supported")
            out.append(float(m))
        return out


class iaf_psc_alpha(_Model):
    """NEST iaf_psc_alpha (_nest_neuron/iaf_psc_alpha.py:349-365 defaults)."""
    model_name = "iaf_psc_alpha"
    order = ("E_L", "C_m", "tau_m", "t_ref", "V_th", "V_reset", "tau_syn_ex", "tau_syn_in",
             "I_e", "V_min")
    units = dict(E_L=mV, C_m=pF, tau_m=ms, t_ref=ms, V_th=mV, V_reset=mV, tau_syn_ex=ms,
                 tau_syn_in=ms, I_e=pA, V_min=mV)
    defaults = dict(E_L=-70.0, C_m=250.0, tau_m=10.0, t_ref=2.0, V_th=-55.0, V_reset=-70.0,
                    tau_syn_ex=2.0, tau_syn_in=2.0, I_e=0.0, V_min=None)
    v_default = "E_L"


class iaf_psc_exp(_Model):
    """NEST iaf_psc_exp, deterministic threshold (_nest_neuron/iaf_psc_exp.py:386-400)."""
    model_name = "iaf_psc_exp"
    order = ("E_L", "C_m", "tau_m", "t_ref", "V_th", "V_reset", "tau_syn_ex", "tau_syn_in",
             "I_e")
    units = dict(E_L=mV, C_m=pF, tau_m=ms, t_ref=ms, V_th=mV, V_reset=mV, tau_syn_ex=ms,
                 tau_syn_in=ms, I_e=pA)
    defaults = dict(E_L=-70.0, C_m=250.0, tau_m=10.0, t_ref=2.0, V_th=-55.0, V_reset=-70.0,
                    tau_syn_ex=2.0, tau_syn_in=2.0, I_e=0.0)
    v_default = "E_L"


class aeif_cond_alpha(_Model):
    """NEST aeif_cond_alpha with RKF45 (_nest_neuron/aeif_cond_alpha.py:379-404 defaults)."""
    model_name = "aeif_cond_alpha"
    order = ("V_peak", "V_reset", "t_ref", "g_L", "C_m", "E_ex", "E_in", "E_L", "Delta_T",
             "tau_w", "a", "b", "V_th", "tau_syn_ex", "tau_syn_in", "I_e", "gsl_error_tol")
    units = dict(V_peak=mV, V_reset=mV, t_ref=ms, g_L=nS, C_m=pF, E_ex=mV, E_in=mV, E_L=mV,
                 Delta_T=mV, tau_w=ms, a=nS, b=pA, V_th=mV, tau_syn_ex=ms, tau_syn_in=ms,
                 I_e=pA, gsl_error_tol=None)
    defaults = dict(V_peak=0.0, V_reset=-60.0, t_ref=0.0, g_L=30.0, C_m=281.0, E_ex=0.0,
                    E_in=-85.0, E_L=-70.6, Delta_T=2.0, tau_w=144.0, a=4.0, b=80.5, V_th=-50.4,
                    tau_syn_ex=0.2, tau_syn_in=2.0, I_e=0.0, gsl_error_tol=1e-6)
    v_default = "E_L"
    conductance = True


class iaf_cond_exp(_Model):
    """NEST iaf_cond_exp with RKF45 (_nest_neuron/iaf_cond_exp.py:295-318 defaults)."""
    model_name = "iaf_cond_exp"
    order = ("E_L", "C_m", "t_ref", "V_th", "V_reset", "E_ex", "E_in", "g_L", "tau_syn_ex",
             "tau_syn_in", "I_e", "gsl_error_tol")
    units = dict(E_L=mV, C_m=pF, t_ref=ms, V_th=mV, V_reset=mV, E_ex=mV, E_in=mV, g_L=nS,
                 tau_syn_ex=ms, tau_syn_in=ms, I_e=pA, gsl_error_tol=None)
    defaults = dict(E_L=-70.0, C_m=250.0, t_ref=2.0, V_th=-55.0, V_reset=-60.0, E_ex=0.0,
                    E_in=-85.0, g_L=16.6667, tau_syn_ex=0.2, tau_syn_in=2.0, I_e=0.0,
                    gsl_error_tol=1e-3)
    v_default = "E_L"
    v_init_const = -70.0
    conductance = True


class iaf_psc_exp_multisynapse(_Model):
    """NEST iaf_psc_exp_multisynapse: one exponential current per receptor, each
    with its own tau_syn (_nest_neuron/iaf_psc_exp_multisynapse.py:395-421
    defaults).  ``receptor_type`` k in 1..len(tau_syn) feeds receptor k; the
    library holds at most 4 receptors."""
    model_name = "iaf_psc_exp_multisynapse"
    order = ("E_L", "C_m", "tau_m", "t_ref", "V_th", "V_reset", "I_e")
    units = dict(E_L=mV, C_m=pF, tau_m=ms, t_ref=ms, V_th=mV, V_reset=mV, I_e=pA)
    defaults = dict(E_L=-70.0, C_m=250.0, tau_m=10.0, t_ref=2.0, V_th=-55.0, V_reset=-70.0,
                    I_e=0.0)
    v_default = "E_L"
    v_init_const = -70.0

    @classmethod
    def resolve(cls, params):
        params = dict(params or {})
        tau = np.atleast_1d(np.asarray(mantissa(params.pop("tau_syn", (2.0,)), ms),
                                       dtype=np.float64))
        if tau.ndim != 1 or not 1 <= tau.size <= 4:
            raise NotImplementedError("1 to 4 receptors (tau_syn entries) are supported")
        return super().resolve(params) + [float(tau.size)] + [float(t) for t in tau]


class iaf_cond_alpha(iaf_cond_exp):
    """NEST iaf_cond_alpha with RKF45 (_nest_neuron/iaf_cond_alpha.py:307-329 defaults)."""
    model_name = "iaf_cond_alpha"


class poisson_generator:
    """Poisson spike generator (_nest_device/poisson_generator.py), realised per target."""
    kind = "generator"

    def __init__(self, rate=0.0, start=0.0, stop=None, origin=0.0, rng_seed=None):
        self.rate = float(mantissa(rate, Hz))
        self.start = float(mantissa(start, ms))
        self.stop = None if stop is None else float(mantissa(stop, ms))
        self.origin = float(mantissa(origin, ms))
        self.rng_seed = rng_seed


class spike_recorder:
    kind = "spike_recorder"


class voltmeter:
    kind = "analog_recorder"
    record_from = ("V_m",)


class multimeter:
    kind = "analog_recorder"

    def __init__(self, record_from=("V_m",)):
        self.record_from = tuple(record_from)


# ------------------------------------------------------------------ rules


class _Rule:
    name = ""


class _AllToAll(_Rule):
    name = "all_to_all"


class _OneToOne(_Rule):
    name = "one_to_one"


class _FixedIndegree(_Rule):
    name = "fixed_indegree"

    def __init__(self, K):
        self.K = int(K)


all_to_all = _AllToAll()
one_to_one = _OneToOne()


def fixed_indegree(K):
    """Each post neuron gets exactly ``K`` edges (_nest_network/rules.py:93-100)."""
    if int(K) < 0:
        raise ValueError(f"K must be >= 0, got {K}")
    return _FixedIndegree(K)


class stdp_synapse:
    """Pair STDP spec (_nest_plasticity/stdp_synapse.py:118-155)."""

    def __init__(self, weight=1.0, delay=1.0, tau_plus=20.0, tau_minus=20.0, lambda_=0.01,
                 alpha=1.0, mu_plus=1.0, mu_minus=1.0, Wmax=100.0, Kplus=0.0):
        self.weight = weight
        self.delay = delay
        self.tau_plus = float(mantissa(tau_plus, ms))
        self.tau_minus = float(mantissa(tau_minus, ms))
        self.lambda_ = float(lambda_)
        self.alpha = float(alpha)
        self.mu_plus = float(mu_plus)
        self.mu_minus = float(mu_minus)
        self.Wmax = float(Wmax)
        if self.tau_plus <= 0:
            raise ValueError("'tau_plus' must be > 0.")
        if self.tau_minus <= 0:
            raise ValueError("'tau_minus' must be > 0.")
        if Kplus < 0:
            raise ValueError("Kplus must be non-negative.")

    def attach(self, pl, proj):
        pl.attach_stdp(proj, self.tau_plus, self.tau_minus, self.lambda_, self.alpha,
                       self.mu_plus, self.mu_minus, self.Wmax)


class stdp_synapse_hom(stdp_synapse):
    """NEST stdp_synapse_hom: the pair rule with parameters shared by every
    edge of the projection, which is already how every rule here is held
    (_nest_plasticity/stdp_synapse_hom.py:24-69)."""


class stdp_triplet_synapse:
    """Pfister-Gerstner triplet STDP spec (_nest_plasticity/stdp_triplet_synapse.py:126-158,
    NEST defaults)."""

    def __init__(self, weight=1.0, delay=1.0, tau_plus=16.8, tau_plus_triplet=101.0,
                 tau_minus=20.0, tau_minus_triplet=110.0, Aplus=5e-10, Aplus_triplet=0.0062,
                 Aminus=0.007, Aminus_triplet=0.00023, Wmax=100.0, Kplus=0.0,
                 Kplus_triplet=0.0):
        self.weight = weight
        self.delay = delay
        self.taus = {}
        for name, q in (("tau_plus", tau_plus), ("tau_plus_triplet", tau_plus_triplet),
                        ("tau_minus", tau_minus), ("tau_minus_triplet", tau_minus_triplet)):
            v = float(mantissa(q, ms))
            if v <= 0.0:
                raise ValueError(f"'{name}' must be > 0.")
            self.taus[name] = v
        self.Aplus, self.Aplus_triplet = float(Aplus), float(Aplus_triplet)
        self.Aminus, self.Aminus_triplet = float(Aminus), float(Aminus_triplet)
        self.Wmax = float(Wmax)
        if Kplus != 0.0 or Kplus_triplet != 0.0:
            raise NotImplementedError("the substrate seeds the traces at 0")

    def attach(self, pl, proj):
        pl.attach_stdp_triplet(proj, self.taus["tau_plus"], self.taus["tau_plus_triplet"],
                               self.taus["tau_minus"], self.taus["tau_minus_triplet"],
                               self.Aplus, self.Aplus_triplet, self.Aminus,
                               self.Aminus_triplet, self.Wmax)


# ----------------------------------------------------------- distributions


# The legacy ``_dist.py`` forms (sampled once at connect on the reference's
# keys; brainpy.state_b200.streams holds the stream restatements).
_DELAY_STREAM = _streams.DELAY_STREAM
_INIT_STREAM = _streams.INIT_STREAM


class Uniform(_streams.Uniform):
    """``low + (high - low) * jax.random.uniform(key, shape)`` (_dist.py:66-77)."""

    def __init__(self, low, high):
        super().__init__(low, high, legacy=True)


class Normal(_streams.Normal):
    """``mean + std * jax.random.normal(key, shape)`` (_dist.py:37-52)."""

    def __init__(self, mean, std):
        super().__init__(mean, std, legacy=True)


class LogNormal(_streams.LogNormal):
    """``exp(mean + std * jax.random.normal(key, shape))`` (_dist.py:55-63)."""

    def __init__(self, mean, std):
        super().__init__(mean, std, legacy=True)


_DISTS = (_streams.Distribution,)


# ----------------------------------------------------------------- views


class _Population:
    def __init__(self, sim, spec, n, params, pop_id, v_init):
        self.sim, self.spec, self.n, self.params, self.pop_id = sim, spec, n, params, pop_id
        self.v_init = v_init


class _Device:
    def __init__(self, spec, n=1):
        self.spec = spec
        self.n = n


class _Segment:
    def __init__(self, population, indices):
        self.population = population
        self.indices = np.asarray(indices, np.int64)


class NodeView:
    """Slice / concatenation of populations (_nest_network/nodeview.py)."""

    def __init__(self, segments):
        self.segments = list(segments)

    def __add__(self, other):
        return NodeView(self.segments + other.segments)

    def __getitem__(self, key):
        if len(self.segments) != 1:
            raise NotImplementedError("slicing a concatenated view")
        seg = self.segments[0]
        return NodeView([_Segment(seg.population, seg.indices[key])])

    def __len__(self):
        return int(sum(s.indices.size for s in self.segments))


# ---------------------------------------------------------------- results


class SimulationResult:
    """Recorded spikes and analog traces (_nest_network/simulator.py:306-414)."""

    def __init__(self, spikes, traces, events, duration_ms, dt, times, weights):
        self._spk = spikes
        self._traces = traces
        self._events = events
        self._T = duration_ms
        self._dt = dt
        self.times = times
        self._weights = weights

    @staticmethod
    def _key(node):
        return id(node.segments[0].population) if isinstance(node, NodeView) else id(node)

    def spikes(self, node):
        """``(n_steps, n_recorded)`` spike matrix of a spike recorder."""
        return self._spk[self._key(node)]

    def events(self, node):
        """Compact ``(step, sender_index)`` arrays of a spike recorder."""
        return self._events[self._key(node)]

    def n_events(self, node):
        return int(self._events[self._key(node)][0].size)

    def rate(self, node):
        """Mean rate in spikes/s over the recorded neurons."""
        steps, _ = self._events[self._key(node)]
        n = self._spk[self._key(node)].shape[1]
        return float(steps.size) / n / (self._T / 1000.0)

    def trace(self, recorder, recordable="V_m"):
        key = (self._key(recorder), recordable)
        if key not in self._traces:
            raise KeyError(f"recordable {recordable!r} was not recorded by this recorder")
        return self._traces[key]

    def weight_trace(self, proj):
        """Weights of a recorded plastic projection at the end of the window
        (``(1, n_edges)``, CSR order)."""
        return self._weights[id(proj)]


class _ProjHandle:
    def __init__(self, proj_id, n_edges):
        self.proj_id = proj_id
        self.n_edges = n_edges


# -------------------------------------------------------------- simulator


class Simulator:
    """NEST-flavoured builder and runner over the CUDA step library.

    Parameters
    ----------
    dt : time quantity or float (ms)
    precision : 32 | 64
    delivery : 'legacy' | 'nest'
    deterministic : bool -- FP64 bit-reproducible delivery (legacy timing only)
    """

    def __init__(self, *, dt, precision=32, delivery="legacy", deterministic=False, device=0,
                 spike_capacity=1 << 24):
        self.dt = float(mantissa(dt, ms))
        if delivery not in ("legacy", "nest"):
            raise ValueError("delivery must be 'legacy' or 'nest'")
        self.precision = int(precision)
        self.delivery = delivery
        self.deterministic = bool(deterministic)
        self.device = device
        self.spike_capacity = int(spike_capacity)
        self._pops = []
        self._model = None
        self._proj_counter = itertools.count()
        self._ops = []            # deferred plan operations in creation order
        self._spike_taps = {}     # id(recorder) -> [(population, indices)], view order
        self._analog_taps = {}    # id(recorder) -> (population, indices, names)
        self._weight_taps = {}
        self._plan = None
        self._step = 0
        self._rng = np.random.default_rng(0)

    # -- create
    def create(self, model_cls, size=1, *, params=None, **kw):
        if isinstance(model_cls, type) and issubclass(model_cls, _Model):
            if self._model is None:
                self._model = model_cls
            elif self._model is not model_cls:
                raise NotImplementedError("one neuron model per Simulator")
            vals = model_cls.resolve(params)
            v_init = (params or {}).get("V_initializer")
            pop = _Population(self, model_cls, int(size), vals, len(self._pops), v_init)
            self._pops.append(pop)
            self._plan = None
            return NodeView([_Segment(pop, np.arange(int(size)))])
        if model_cls is poisson_generator:
            dev = _Device(poisson_generator(**(params or {}), **kw))
            return NodeView([_Segment(dev, np.arange(1))])
        if model_cls in (spike_recorder, voltmeter):
            return NodeView([_Segment(_Device(model_cls()), np.arange(0))])
        if model_cls is multimeter:
            return NodeView([_Segment(_Device(multimeter(**(params or {}), **kw)), np.arange(0))])
        raise TypeError(f"unsupported model {model_cls!r}")

    @staticmethod
    def _derive_seed(base, ordinal):
        b = 0 if base is None else int(base)
        return (b * 1_000_003 + ordinal + 1) & 0x7FFFFFFF

    def _steps(self, delay):
        """NEST delay rounding floor(d/dt + 0.5) (_kernel/delays.py:50-100)."""
        d = np.asarray(delay, np.float64)
        spm = 1.0 / self.dt
        k = np.rint(spm)
        if k >= 1 and abs(spm - k) <= 1e-6 * k:
            spm = k
        return np.floor(d * spm + 0.5).astype(np.int64)

    # -- connect
    def connect(self, pre, post, *, rule=all_to_all, weight=None, delay=None, comm="sparse",
                receptor_type=None, synapse=None, allow_autapses=True, allow_multapses=True,
                seed=None):
        del comm  # both comm paths of the reference become the same CSR here
        if len(pre.segments) == 1 and isinstance(pre.segments[0].population, _Device) and \
                pre.segments[0].population.spec.kind == "analog_recorder":
            rec = pre.segments[0].population
            seg = post.segments[0]
            self._analog_taps[id(rec)] = (seg.population, seg.indices,
                                          tuple(getattr(rec.spec, "record_from", ("V_m",))))
            self._plan = None
            return None
        if len(post.segments) == 1 and isinstance(post.segments[0].population, _Device) and \
                post.segments[0].population.spec.kind == "spike_recorder":
            self._spike_taps[id(post.segments[0].population)] = [(sg.population, sg.indices)
                                                                 for sg in pre.segments]
            self._plan = None
            return None
        if not allow_multapses:
            raise NotImplementedError("allow_multapses=False")
        handles = []
        for ps in pre.segments:
            for qs in post.segments:
                ordinal = next(self._proj_counter)
                h = self._connect_pair(ps, qs, rule, weight, delay, receptor_type, synapse,
                                       allow_autapses, seed, ordinal)
                if h is not None:
                    handles.append(h)
        self._plan = None
        if not handles:
            return None
        return handles[0] if len(handles) == 1 else handles

    def _receptor(self, receptor_type):
        if receptor_type is None:
            return 0
        k = int(receptor_type)
        if self._model is iaf_psc_exp_multisynapse:
            if k < 1:
                raise ValueError("receptor_type must be >= 1")
            return k - 1  # the library checks it against the population's receptors
        if k not in (1, 2):
            raise ValueError("receptor_type must be 1 (excitatory) or 2 (inhibitory)")
        return k - 1

    def _connect_pair(self, ps, qs, rule, weight, delay, receptor_type, synapse,
                      allow_autapses, seed, ordinal):
        src, dst = ps.population, qs.population
        if not isinstance(dst, _Population):
            raise TypeError("post must be a neuron population")
        full_post = qs.indices.size == dst.n and np.all(qs.indices == np.arange(dst.n))
        w_unit = nS if self._model.conductance else pA
        if synapse is not None:
            weight = synapse.weight if weight is None else weight
            delay = synapse.delay if delay is None else delay
        if isinstance(src, _Device):
            gen = src.spec
            if not isinstance(gen, poisson_generator):
                raise TypeError("only poisson_generator sources are supported")
            if not full_post:
                raise NotImplementedError("generator into a population slice")
            gseed = self._derive_seed(gen.rng_seed, ordinal)
            dsteps = int(self._steps(mantissa(delay if delay is not None else 0.0, ms)))
            t_min = int(round((gen.origin + gen.start) / self.dt))
            t_max = 2 ** 62 if gen.stop is None else int(round((gen.origin + gen.stop) / self.dt))
            wv = float(mantissa(weight if weight is not None else 1.0, w_unit))
            self._ops.append(("drive", dst.pop_id, gen.rate, wv, dsteps, gseed, t_min, t_max,
                              self._receptor(receptor_type)))
            return None
        full_pre = ps.indices.size == src.n and np.all(ps.indices == np.arange(src.n))
        pseed = self._derive_seed(seed, ordinal)
        # the projection's keys: k_conn, k_w, k_rec = split(key(seed), 3)
        # (_nest_network/event_proj.py:147-149); distributed weights draw from
        # k_w, one value per edge in the sampler's order, before the CSR sort
        pkey = _streams.root_key(pseed)
        k_w = _streams.fold_in(pkey, 1)
        receptor = self._receptor(receptor_type)
        if isinstance(rule, _FixedIndegree) and full_pre and full_post:
            E = rule.K * dst.n
            dl = self._delays(delay, E, pkey)
            if isinstance(weight, _DISTS):
                wv = np.asarray(weight.sample_in(k_w, E, w_unit, self._bits), dtype=np.float64)
            else:
                wv = float(mantissa(weight if weight is not None else 1.0, w_unit))
            op = ("fixed_indegree", src.pop_id, dst.pop_id, rule.K, pseed, allow_autapses, wv,
                  dl, receptor, synapse)
            self._ops.append(op)
            return _ProjHandle(len([o for o in self._ops if o[0] != "drive"]) - 1, E)
        # explicit edges
        if isinstance(rule, _AllToAll):
            pre_l = np.repeat(ps.indices, qs.indices.size)
            post_l = np.tile(qs.indices, ps.indices.size)
            if src is dst and not allow_autapses:
                keep = pre_l != post_l
                pre_l, post_l = pre_l[keep], post_l[keep]
        elif isinstance(rule, _OneToOne):
            if ps.indices.size != qs.indices.size:
                raise ValueError("one_to_one requires equal sizes")
            pre_l, post_l = ps.indices.copy(), qs.indices.copy()
        elif isinstance(rule, _FixedIndegree):
            raise NotImplementedError("fixed_indegree on population slices")
        else:
            raise TypeError(f"unsupported rule {rule!r}")
        E = pre_l.size
        if isinstance(weight, _DISTS):
            w = weight.sample_in(k_w, E, w_unit, self._bits)
        else:
            w = np.broadcast_to(mantissa(weight if weight is not None else 1.0, w_unit),
                                (E,)).astype(np.float64)
        dl = self._delays(delay, E, pkey)
        order = np.argsort(pre_l, kind="stable")
        indptr = np.concatenate([[0], np.cumsum(np.bincount(pre_l, minlength=src.n))])
        self._ops.append(("csr", src.pop_id, dst.pop_id, indptr.astype(np.int64),
                          post_l[order].astype(np.int32), np.asarray(w)[order],
                          dl[order].astype(np.int32), receptor, synapse))
        return _ProjHandle(len([o for o in self._ops if o[0] != "drive"]) - 1, E)

    @property
    def _bits(self):
        return 64 if self.precision == 64 else 32

    def _delays(self, delay, E, pkey):
        """Delay steps of E edges (sampler order).  Per-edge delay
        distributions have no counterpart in the legacy reference (its delays
        are one value per projection, _nest_network/delay.py:29-128); they
        draw from fold(key(seed), DELAY_STREAM) of the projection so a run is
        reproducible."""
        if delay is None:
            steps = np.zeros(E, np.int64)
        elif isinstance(delay, _DISTS):
            d = delay.sample_in(_streams.fold_in(pkey, _DELAY_STREAM), E, ms, self._bits)
            steps = self._steps(d)
        else:
            steps = np.broadcast_to(self._steps(mantissa(delay, ms)), (E,)).astype(np.int64)
        if self.delivery == "nest" and np.any(steps < 1):
            raise ValueError("delays must be >= dt with delivery='nest'")
        return steps

    def record_weight(self, proj):
        if not isinstance(proj, _ProjHandle) or not self._is_plastic(proj):
            raise TypeError("record_weight requires a plastic projection handle")
        self._weight_taps[id(proj)] = proj
        return proj

    def _is_plastic(self, h):
        ops = [o for o in self._ops if o[0] != "drive"]
        return ops[h.proj_id][-1] is not None

    # -- build
    def _build(self, upload=True):
        """The library plan of the network; ``upload=False`` stops before the
        device (the realised structure stays readable through ``Plan.csr``)."""
        if self._model is None:
            raise RuntimeError("no neuron population")
        sem = _lib.LEGACY if self.delivery == "legacy" else _lib.RING
        pl = _lib.Plan(self.dt, self._model.model_name, precision=self.precision, semantics=sem,
                       deterministic=self.deterministic, device=self.device,
                       spike_capacity=self.spike_capacity)
        for p in self._pops:
            pl.add_pop(p.n, p.params)
        for op in self._ops:
            if op[0] == "drive":
                _, pop, rate, w, d, seed, t_min, t_max, rec = op
                pl.add_poisson(pop, rate, w, d, seed, t_min, t_max, rec)
            elif op[0] == "fixed_indegree":
                _, a, b, K, seed, auto, w, dl, rec, syn = op
                nbits = 64 if self.precision == 64 else 32
                per_edge = isinstance(w, np.ndarray)
                j = pl.add_fixed_indegree(a, b, K, seed, 1.0 if per_edge else w, delay_steps=dl,
                                          allow_autapses=auto, nbits=nbits, receptor=rec,
                                          w_draw=w if per_edge else None)
                self._attach(pl, j, syn)
            else:
                _, a, b, indptr, post, w, dl, rec, syn = op
                j = pl.add_csr(a, b, indptr, post, w, dl, rec)
                self._attach(pl, j, syn)
        gids, self._v_slices = [], {}
        for rid, (pop, idx, names) in self._analog_taps.items():
            if names != ("V_m",):
                raise NotImplementedError("analog recording of V_m only")
            start = len(gids)
            off = sum(q.n for q in self._pops[:pop.pop_id])
            gids.extend((off + idx).tolist())
            self._v_slices[rid] = slice(start, len(gids))
        if gids:
            pl.record_v(np.asarray(gids, np.int32))
        offs = np.cumsum([0] + [q.n for q in self._pops])
        tapped = [offs[pop.pop_id] + idx for segs in self._spike_taps.values()
                  for pop, idx in segs]
        pl.record_spikes_of(np.unique(np.concatenate(tapped)).astype(np.int32) if tapped
                            else np.zeros(0, np.int32))
        for h in self._weight_taps.values():
            pl.record_weights(h.proj_id)
        if not upload:
            return pl
        pl.upload()
        self._plan = pl
        return pl

    @staticmethod
    def _attach(pl, j, syn):
        if syn is not None:
            syn.attach(pl, j)

    def initial_v(self, pop_id):
        """Initial V_m of population ``pop_id`` (mV) as ``simulate`` sets it."""
        p = self._pops[pop_id]
        init = p.v_init
        if init is None and p.spec.v_init_const is not None:
            return np.full(p.n, p.spec.v_init_const)
        if init is None:
            return np.full(p.n, p.params[p.spec.order.index(p.spec.v_default)])
        if isinstance(init, _DISTS):
            # the reference draws V_initializer from brainstate's global
            # random state, which no Simulator seed sets; the facade draws
            # it from fold(fold(key(0), INIT_STREAM), population ordinal)
            k = _streams.fold_in(_streams.fold_in(_streams.root_key(0), _INIT_STREAM), p.pop_id)
            return init.sample_in(k, p.n, mV, self._bits)
        if callable(init):
            return np.broadcast_to(np.asarray(init(p.n), np.float64), (p.n,))
        return np.broadcast_to(mantissa(init, mV), (p.n,))

    def _init_state(self):
        pl = self._plan
        for p in self._pops:
            v = self.initial_v(p.pop_id)
            pl.set_state(p.pop_id, "V_m", v)
            for name in pl_state_names(self._model):
                pl.set_state(p.pop_id, name, np.zeros(p.n))
            if self._model.conductance:
                pl.set_state(p.pop_id, "h", np.full(p.n, self.dt))

    # -- run
    def _n_steps(self, duration):
        d = float(mantissa(duration, ms))
        r = d / self.dt
        n = int(round(r)) if abs(r - round(r)) < 1e-9 * max(1.0, r) else int(math.ceil(r))
        return n

    def simulate(self, duration):
        """Run ``duration`` from a freshly initialised state."""
        if self._plan is None:
            self._build()
        else:
            # re-initialise in place: restore the post-upload checkpoint
            self._plan.restore(self._ck0)
        if not hasattr(self, "_ck0") or self._ck_plan is not self._plan:
            self._init_state()
            self._ck0 = self._plan.checkpoint()
            self._ck_plan = self._plan
        self._step = 0
        return self._run_window(duration)

    def cont(self, duration):
        """Continue without re-initialising (``simulator.py:1822-1839``)."""
        if self._plan is None:
            return self.simulate(duration)
        return self._run_window(duration)

    def _run_window(self, duration):
        pl = self._plan
        n = self._n_steps(duration)
        step0 = pl.step
        pl.run(n)
        st, gid = pl.spikes()
        spikes, events = {}, {}
        offs = np.cumsum([0] + [p.n for p in self._pops])
        for rid, segs in self._spike_taps.items():
            # columns in view order, across the view's populations
            cols = np.concatenate([offs[pop.pop_id] + idx for pop, idx in segs])
            mat = np.zeros((n, cols.size), np.float32 if self.precision == 32 else np.float64)
            pos = np.full(int(offs[-1]), -1, np.int64)
            pos[cols] = np.arange(cols.size)
            col = pos[gid] if gid.size else np.zeros(0, np.int64)
            ok = col >= 0
            rows = st[ok] - step0
            mat[rows, col[ok]] = 1.0
            spikes[rid] = mat
            events[rid] = (rows, col[ok])
        traces = {}
        if self._analog_taps:
            # traces in the run's precision, like the spike matrices
            v = pl.v_trace(np.float32 if self.precision == 32 else np.float64)
            for rid, sl in self._v_slices.items():
                traces[(rid, "V_m")] = v[:, sl]
        # (n_steps, n_edges) FP64 weights after every step, CSR order
        weights = {k: pl.weight_trace(h.proj_id) for k, h in self._weight_taps.items()}
        times = (step0 + np.arange(n)) * self.dt
        return SimulationResult(spikes, traces, events, n * self.dt, self.dt, times, weights)


def pl_state_names(model):
    if model is iaf_psc_alpha:
        return ("I_syn_ex", "dI_syn_ex", "I_syn_in", "dI_syn_in", "y0", "r")
    if model is iaf_psc_exp:
        return ("i_syn_ex", "i_syn_in", "i_0", "i_1", "r")
    if model is iaf_cond_exp:
        return ("g_ex", "g_in", "I_stim", "r")
    if model is iaf_psc_exp_multisynapse:
        return ("i_const", "i_syn_0", "i_syn_1", "i_syn_2", "i_syn_3", "r")
    if model is iaf_cond_alpha:
        return ("dg_ex", "g_ex", "dg_in", "g_in", "I_stim", "r")
    return ("dg_ex", "g_ex", "dg_in", "g_in", "w", "I_stim", "r")
