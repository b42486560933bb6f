"""Kernel-API front end over libbspk: ``Network`` / ``PopulationView`` /
``Projection`` / ``Observer`` (``_kernel/network.py``, ``_kernel/observers.py``)
and ``Program`` / ``Runner`` / ``Results`` (``_kernel/runner.py:782-960``).

A ``Network`` collects populations, projections and observers without state;
``compile`` turns it into one library plan and ``runner()`` advances it:

* timing is the kernel's: an event of step n over a delay of d steps reaches
  step n + d, with NEST's rounding of delays to steps, floor(d / dt + 0.5)
  (``_kernel/delays.py:50-100``);
* the iaf models' receptor ports ``ex`` and ``in_`` stay apart and keep their
  weights' signs (the kernel models' ``Ports``); such plans run on the
  library's tiled kernel (one shared-memory ring per port) when every drive
  feeds ``ex``, else on its per-step engine;
* recording follows the kernel's dense rules (``_kernel/observers.py:1-20``):
  per interval of k steps, spike counts are summed and states are sampled at
  the window's last step; runs are whole multiples of every interval;
* every random draw follows the kernel's streams for the network's seed
  (``_kernel/rng.py``, ``_kernel/compiler.py:819-850``, module ``streams``):
  ``fixed_indegree`` (with multapses) draws its sources from the key chain
  (projection name, post population name, local id; blake2b name ids) with
  the library's restatement of ``jax.random.randint``; distributed weights
  and delays (``Uniform`` / ``Normal`` / ``LogNormal``) draw one value per
  edge in the rule's canonical order (post-major, pre ascending) from the
  projection's WEIGHT / DELAY streams; distributed initial ``V_m`` from the
  population's INIT stream; and each ``poisson_generator`` unit draws its
  counts from its population's block keys by the kernel's float32 CDF
  inversion (``_kernel/models/devices.py:46-145``).  Delays are drawn in the
  plan's precision (float32 or float64, as the reference does with
  ``jax_enable_x64`` off or on).

Limits of this front end: the neuron models are ``iaf_psc_alpha`` and
``iaf_psc_exp`` (one per network; the kernel's conductance models integrate
with fixed-substep RK4, which the library does not run); the one device is
``poisson_generator`` with rate * dt below 10 per step (the reference's CDF
inversion range), connected ``one_to_one`` onto whole neuron populations;
``fixed_indegree`` needs ``allow_multapses=True``; no plasticity or learners.
Batched trials (``Runner(program, batch=B, rng=...)``) fold the trial index
into the drives' step keys as the reference's ``vmap`` runs do.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from . import streams as S
from .simulator import iaf_psc_alpha, iaf_psc_exp
from .streams import LogNormal, Normal, Uniform, name_id
from .units import Hz, mV, ms, pA, mantissa

__all__ = ["Network", "PopulationView", "Projection", "Observer", "Program", "Runner", "Results",
           "trial_indices",
           "Recording", "poisson_generator", "all_to_all", "one_to_one", "fixed_indegree",
           "iaf_psc_alpha", "iaf_psc_exp", "name_id", "Uniform", "Normal", "LogNormal"]

GID_BLOCK = 1024          # ids per connectivity key block (_kernel/rng.py:79)
_PORTS = {"ex": 0, "in_": 1}


# ------------------------------------------------------------------ devices

class poisson_generator:
    """Poisson spike source (``_kernel/models/devices.py``), one independent
    train per device neuron: ``rate`` (Hz), active for start < t <= stop (ms)."""
    defaults = dict(rate=0.0, start=0.0, stop=None)

    @classmethod
    def resolve(cls, params):
        vals = dict(cls.defaults)
        for k, v in (params or {}).items():
            if k not in vals:
                raise TypeError(f"poisson_generator got an unexpected parameter {k!r}")
            vals[k] = v
        rate = float(mantissa(vals["rate"], Hz))
        if rate < 0:
            raise ValueError("rate must be >= 0")
        stop = None if vals["stop"] is None else float(mantissa(vals["stop"], ms))
        return dict(rate=rate, start=float(mantissa(vals["start"], ms)), stop=stop)


_NEURON_MODELS = (iaf_psc_alpha, iaf_psc_exp)


# -------------------------------------------------------------------- rules

class all_to_all:
    """Every pre to every post (``_kernel/connectivity/rules.py`` AllToAll)."""
    random = False

    def __init__(self, allow_autapses=True):
        self.allow_autapses = bool(allow_autapses)


class one_to_one:
    """Pre i to post i (equal sizes)."""
    random = False


class fixed_indegree:
    """``indegree`` sources per post neuron, uniform over the pre view with
    multapses (``_kernel/connectivity/rules.py:192-265``)."""
    random = True

    def __init__(self, indegree, allow_autapses=True, allow_multapses=True):
        if isinstance(indegree, bool) or int(indegree) != indegree or indegree < 0:
            raise ValueError(f"indegree must be a non-negative int, got {indegree!r}")
        self.indegree = int(indegree)
        self.allow_autapses = bool(allow_autapses)
        if not allow_multapses:
            raise NotImplementedError("fixed_indegree without multapses (Floyd / top-k "
                                      "sampling) is not available")
        self.allow_multapses = True


_RULE_NAMES = {all_to_all: "AllToAll", one_to_one: "OneToOne", fixed_indegree: "FixedIndegree"}


# ---------------------------------------------------------- network objects

class Population:
    def __init__(self, index, name, model, n, gid_start, params, init):
        self.index, self.name, self.model, self.n = index, name, model, n
        self.gid_start, self.params, self.init = gid_start, params, init
        self.lib_pop = None  # library population id after compile (neurons)

    @property
    def is_device(self):
        return self.model is poisson_generator

    @property
    def gids(self):
        return np.arange(self.gid_start, self.gid_start + self.n, dtype=np.int64)


class PopulationView:
    """Ordered gids of one network (``_kernel/network.py:156-255``): slicing
    and integer indexing select, ``+`` concatenates."""

    def __init__(self, net, gids, name=None):
        self.net = net
        self.gids = np.asarray(gids, dtype=np.int64).reshape(-1)
        self.name = name

    @property
    def size(self):
        return int(self.gids.size)

    def __len__(self):
        return self.size

    def __getitem__(self, key):
        g = self.gids[key]
        return PopulationView(self.net, np.atleast_1d(g))

    def __add__(self, other):
        if not isinstance(other, PopulationView) or other.net is not self.net:
            raise ValueError("views of different networks cannot be joined")
        return PopulationView(self.net, np.concatenate([self.gids, other.gids]))

    def parts(self):
        """Contiguous runs of the view by population: [(population, local ids)]."""
        if self.size == 0:
            return []
        starts = np.array([p.gid_start for p in self.net.populations], np.int64)
        pop = np.searchsorted(starts, self.gids, side="right") - 1
        cut = np.nonzero(np.diff(pop) != 0)[0] + 1
        bounds = np.concatenate([[0], cut, [self.size]])
        return [(self.net.populations[int(pop[a])], self.gids[a:b] - starts[pop[a]])
                for a, b in zip(bounds[:-1], bounds[1:])]

    @property
    def populations(self):
        seen = []
        for p, _ in self.parts():
            if p not in seen:
                seen.append(p)
        return seen


class Projection:
    def __init__(self, index, name, pre, post, rule, port, weight, delay):
        self.index, self.name, self.pre, self.post = index, name, pre, post
        self.rule, self.port, self.weight, self.delay = rule, port, weight, delay


class Observer:
    def __init__(self, index, name, view, recordables, interval):
        self.index, self.name, self.view = index, name, view
        self.recordables, self.interval = recordables, interval

    @property
    def size(self):
        return self.view.size

    def n_samples(self, n_steps):
        if n_steps % self.interval:
            raise ValueError(f"run of {n_steps} steps is not a multiple of observer "
                             f"{self.name!r} interval ({self.interval} steps)")
        return n_steps // self.interval


def _steps(q, dt, what):
    r = float(mantissa(q, ms)) / dt
    k = int(round(r))
    if abs(r - k) > 1e-6 * max(1.0, r):
        raise ValueError(f"{what} must be a whole multiple of dt={dt} ms")
    return k


class Network:
    """Graph of populations, projections and observers (``_kernel/network.py:316-716``).

    Parameters: dt (Quantity or ms), seed (int in [0, 2**32), the root of every
    random stream).
    """

    def __init__(self, dt, seed=0):
        self.dt = float(mantissa(dt, ms))
        if not self.dt > 0:
            raise ValueError(f"dt must be positive, got {dt}")
        if isinstance(seed, bool) or not isinstance(seed, (int, np.integer)) or \
                not 0 <= seed < 2 ** 32:
            raise ValueError(f"seed must be an int in [0, 2**32), got {seed!r}")
        self.seed = int(seed)
        self.populations, self.projections, self.observers = [], [], []
        self._names, self._ids, self._auto = set(), {}, {}

    @property
    def n_neurons(self):
        if not self.populations:
            return 0
        last = self.populations[-1]
        return last.gid_start + last.n

    def _unique(self, name, cls):
        if name is None:
            k = self._auto.get(cls, 0)
            while f"{cls}_{k}" in self._names:
                k += 1
            self._auto[cls] = k + 1
            name = f"{cls}_{k}"
        if not isinstance(name, str) or not name:
            raise TypeError(f"name must be a non-empty str, got {name!r}")
        if name in self._names:
            raise ValueError(f"name {name!r} is already used in this network")
        nid = name_id(name)
        if nid in self._ids:  # 64-bit collision
            raise ValueError(f"names {name!r} and {self._ids[nid]!r} hash to the same stream id")
        self._names.add(name)
        self._ids[nid] = name
        return name

    def _view(self, v, what):
        if not isinstance(v, PopulationView):
            raise TypeError(f"{what} must be a PopulationView, got {type(v).__name__}")
        if v.net is not self:
            raise ValueError(f"{what} belongs to another network")
        return v

    def add(self, model, n, params=None, init=None, *, name=None):
        """Add ``n`` neurons (or devices) of ``model``; returns their view."""
        if model not in _NEURON_MODELS and model is not poisson_generator:
            raise TypeError(f"model must be iaf_psc_alpha, iaf_psc_exp or poisson_generator, "
                            f"got {model!r}")
        if isinstance(n, bool) or not isinstance(n, (int, np.integer)) or n < 0:
            raise ValueError(f"n must be a non-negative int, got {n!r}")
        for p in self.populations:
            if not p.is_device and model is not poisson_generator and p.model is not model:
                raise NotImplementedError("one neuron model per network")
        vals = model.resolve(params)
        init = dict(init or {})
        for k in init:
            if k != "V_m":
                raise NotImplementedError(f"initial value of {k!r}: only V_m can be set")
            if model is poisson_generator:
                raise ValueError("a device has no initial state")
        name = self._unique(name, model.__name__)
        pop = Population(len(self.populations), name, model, int(n), self.n_neurons, vals, init)
        self.populations.append(pop)
        return PopulationView(self, pop.gids, name)

    def connect(self, pre, post, rule=None, *, port=None, weight=None, delay=None, name=None):
        """Connect ``pre`` to ``post`` (validated now, realised at compile)."""
        pre, post = self._view(pre, "pre"), self._view(post, "post")
        rule = all_to_all() if rule is None else rule
        if type(rule) not in _RULE_NAMES:
            raise TypeError(f"rule must be all_to_all, one_to_one or fixed_indegree, got {rule!r}")
        if any(p.is_device for p in post.populations):
            raise ValueError("a device cannot be a target")
        if port not in _PORTS:
            raise ValueError(f"port must be 'ex' or 'in_' for {sorted({p.model.__name__ for p in post.populations})}, got {port!r}")
        src_dev = [p.is_device for p in pre.populations]
        if any(src_dev) and not all(src_dev):
            raise ValueError("a pre view mixes devices and neurons")
        if all(src_dev) and src_dev:
            if not isinstance(rule, one_to_one):
                raise NotImplementedError("a poisson_generator connects one_to_one (one train "
                                          "per target)")
        if isinstance(rule, one_to_one) and pre.size != post.size:
            raise ValueError(f"one_to_one needs equal sizes, got {pre.size} and {post.size}")
        w = 1.0 if weight is None else weight
        if not isinstance(w, S.Distribution):
            w = np.asarray(mantissa(w, pA), dtype=np.float64)
        d = self.dt if delay is None else delay
        if isinstance(d, S.Distribution):
            lo = -np.inf if d.low is None else d.low
            if lo < 0:
                raise ValueError("a delay distribution must be bounded below by 0")
        else:
            d = np.asarray(mantissa(d, ms), dtype=np.float64)
            if np.any(d <= 0):
                raise ValueError("delays must be > 0")
        name = self._unique(name, _RULE_NAMES[type(rule)])
        proj = Projection(len(self.projections), name, pre, post, rule, port, w, d)
        self.projections.append(proj)
        return proj

    def observe(self, view, *recordables, interval=None, name=None):
        """Record ``recordables`` ('spike': counts per interval; 'V_m': sampled
        at the interval's last step) of ``view``, columns in view order."""
        view = self._view(view, "view")
        if not recordables:
            raise ValueError("nothing to record")
        for r in recordables:
            if r not in ("spike", "V_m"):
                raise NotImplementedError(f"recordable {r!r}: only 'spike' and 'V_m'")
        if any(p.is_device for p in view.populations):
            raise NotImplementedError("recording a device")
        if np.unique(view.gids).size != view.size:
            raise ValueError("an observer's view lists a neuron twice")
        k = 1 if interval is None else _steps(interval, self.dt, "interval")
        if k < 1:
            raise ValueError("interval must be >= dt")
        obs = Observer(len(self.observers), self._unique(name, "Observer"), view,
                       tuple(recordables), k)
        self.observers.append(obs)
        return obs

    def compile(self, precision="float32", *, upload=True, spike_capacity=None):
        """Realise connectivity and build the library plan: a :class:`Program`.
        ``upload=False`` stops before the device (the realised structure stays
        readable on the host: ``Program.realised``, ``Program.initial_v``)."""
        if precision not in ("float32", "float64"):
            raise ValueError("precision must be 'float32' or 'float64'")
        return Program(self, 64 if precision == "float64" else 32, upload=upload,
                       spike_capacity=spike_capacity)


# ----------------------------------------------------------------- compiled

def _delay_steps(d, dt, bits=64):
    """NEST rounding of delays to steps (``streams.delay_steps``), at least 1."""
    s = S.delay_steps(d, dt, bits)
    if np.any(s < 1):
        raise ValueError(f"a delay rounds to 0 steps at dt={dt} ms")
    return s


def _grid_steps(t_ms, dt):
    """Steps of a device time, rounded up to the grid with values within
    1e-6 steps of a grid point snapped to it (NEST's Time conversion,
    ``_kernel/units.py:229-270``)."""
    r = float(t_ms) / dt
    k = round(r)
    return int(k) if abs(r - k) <= 1e-6 * max(1.0, abs(r)) else int(np.ceil(r))


def realise_positions(net, proj):
    """Edges of a neuron-to-neuron projection as (positions in the pre view,
    positions in the post view), on the host: one_to_one, all_to_all (post
    major) or the kernel's keyed fixed_indegree (post major, K per post)."""
    pre, post, rule = proj.pre, proj.post, proj.rule
    if isinstance(rule, one_to_one):
        return np.arange(pre.size, dtype=np.int64), np.arange(post.size, dtype=np.int64)
    if isinstance(rule, all_to_all):  # already canonical
        src = np.tile(np.arange(pre.size, dtype=np.int64), post.size)
        dst = np.repeat(np.arange(post.size, dtype=np.int64), pre.size)
        if not rule.allow_autapses:
            keep = pre.gids[src] != post.gids[dst]
            src, dst = src[keep], dst[keep]
        return src, dst
    K = rule.indegree
    self_pos = None
    if not rule.allow_autapses:
        where = {int(g): i for i, g in enumerate(pre.gids)}
        self_pos = np.array([where.get(int(g), -1) for g in post.gids], np.int64)
    parts = [(name_id(p.name), local) for p, local in post.parts()]
    pos = _lib.kernel_fixed_indegree(net.seed, name_id(proj.name), parts, pre.size, self_pos, K)
    src, dst = pos.reshape(-1), np.repeat(np.arange(post.size, dtype=np.int64), K)
    # the rule's canonical edge order: post-major, pre ascending, stable
    # (_kernel/connectivity/rules.py:83-88)
    order = np.lexsort((src, dst))
    return src[order], dst[order]


class Program:
    """A compiled network: the library plan plus the gid maps (``runner()``)."""

    def __init__(self, net, precision, upload=True, spike_capacity=None, trial=0):
        self.net, self.precision, self.dt = net, precision, net.dt
        self.spike_capacity, self.trial = spike_capacity, int(trial)
        neurons = [p for p in net.populations if not p.is_device]
        model = neurons[0].model if neurons else iaf_psc_alpha
        kw = {} if spike_capacity is None else {"spike_capacity": int(spike_capacity)}
        pl = _lib.Plan(net.dt, model.model_name, precision=precision, semantics=_lib.RING, **kw)
        pl.set_ports(True)
        if self.trial:
            pl.set_trial(self.trial)
        self.lib_gid0 = {}  # population index -> first library gid
        g0 = 0
        for p in neurons:
            p.lib_pop = pl.add_pop(p.n, p.params)
            self.lib_gid0[p.index] = g0
            g0 += p.n
        self.n_lib = g0
        self.realised = []  # (pre lib pop, post lib pop, indptr, post local, w, delay steps, port)
        self.edge_delays = {}  # projection name -> delay steps in canonical edge order
        self.drives = []    # (post lib pop, rate, w, delay steps, object key, first unit, t_min, t_max, port)
        for proj in net.projections:
            self._realise(pl, proj)
        rec_v = sorted({int(self._lib_gid(g)) for o in net.observers if "V_m" in o.recordables
                        for g in o.view.gids})
        self.rec_v = np.array(rec_v, np.int64)
        if rec_v:
            pl.record_v(self.rec_v)
        # spikes: of the observed neurons when any observer records them, of
        # every neuron otherwise (plan-level users read them all)
        rec_s = sorted({int(self._lib_gid(g)) for o in net.observers if "spike" in o.recordables
                        for g in o.view.gids})
        if rec_s:
            pl.record_spikes_of(np.array(rec_s, np.int32))
        self.plan = pl
        self._ck0 = None
        if not upload:
            return
        pl.upload()
        for p in neurons:
            pl.set_state(p.lib_pop, "V_m", self.initial_v(p))
        # the initial state in page-locked memory: simulate() restores it with
        # one host-to-device copy per buffer
        self._ck0 = pl.checkpoint(pinned=True)
        # library columns of every observer, in view order
        self.obs_cols = {o.name: np.array([self._lib_gid(x) for x in o.view.gids], np.int64)
                         for o in net.observers}
        # library gid -> observer column (-1: not observed), per spike observer
        self.obs_pos = {}
        for o in net.observers:
            pos = np.full(self.n_lib, -1, np.int64)
            pos[self.obs_cols[o.name]] = np.arange(self.obs_cols[o.name].size)
            self.obs_pos[o.name] = pos

    @property
    def bits(self):
        """Width of the plan's floating-point draws (32 or 64)."""
        return 64 if self.precision == 64 else 32

    def initial_v(self, p):
        """Initial V_m of population ``p``: E_L, a value, or a distribution
        drawn from name_key(fold(object_key, INIT_STREAM), 'V_m') in the
        plan's precision (``_kernel/params.py:652-693``)."""
        v0 = p.init.get("V_m")
        if v0 is None:
            return np.full(p.n, p.params[p.model.order.index("E_L")])
        if isinstance(v0, S.Distribution):
            key = S.name_key(S.fold_in(S.object_key(self.net.seed, p.name), S.INIT_STREAM), "V_m")
            return v0.sample_in(key, p.n, mV, self.bits)
        v = np.broadcast_to(np.asarray(mantissa(v0, mV), np.float64), (p.n,))
        return np.ascontiguousarray(v, np.float64)

    def _lib_gid(self, gid):
        for p in self.net.populations:
            if p.gid_start <= gid < p.gid_start + p.n:
                if p.is_device:
                    raise ValueError("a device has no library id")
                return self.lib_gid0[p.index] + (gid - p.gid_start)
        raise ValueError(f"gid {gid} out of range")

    def _realise(self, pl, proj):
        net, dt = self.net, self.dt
        port = _PORTS[proj.port]
        if proj.pre.size == 0 or proj.post.size == 0:
            return
        if proj.pre.populations[0].is_device:
            self._realise_drive(pl, proj, port)
            return
        src, dst = realise_positions(net, proj)
        pre, post = proj.pre, proj.post
        E = src.size
        okey = S.object_key(net.seed, proj.name)
        if isinstance(proj.weight, S.Distribution):
            w = proj.weight.sample_in(S.fold_in(okey, S.WEIGHT_STREAM), E, pA, self.bits)
        else:
            w = np.broadcast_to(proj.weight, (E,)).astype(np.float64)
        if isinstance(proj.delay, S.Distribution):
            # jax's default float: float32 unless the run enables x64
            dq = proj.delay.sample_in(S.fold_in(okey, S.DELAY_STREAM), E, ms, self.bits)
            ds = _delay_steps(dq, dt, self.bits)
        else:
            ds = _delay_steps(np.broadcast_to(proj.delay, (E,)).astype(np.float64), dt)
        self.edge_delays[proj.name] = ds
        pre_lib = np.array([self._lib_gid(g) for g in pre.gids], np.int64)[src]
        post_lib = np.array([self._lib_gid(g) for g in post.gids], np.int64)[dst]
        neurons = [p for p in net.populations if not p.is_device]
        bounds = [(p.lib_pop, self.lib_gid0[p.index], p.n) for p in neurons]
        for a, a0, an in bounds:
            ma = (pre_lib >= a0) & (pre_lib < a0 + an)
            for b, b0, bn in bounds:
                m = ma & (post_lib >= b0) & (post_lib < b0 + bn)
                if not m.any():
                    continue
                pl_, po = pre_lib[m] - a0, post_lib[m] - b0
                order = np.argsort(pl_, kind="stable")  # CSR rows = pre, stable
                indptr = np.zeros(an + 1, np.int64)
                np.add.at(indptr, pl_ + 1, 1)
                indptr = np.cumsum(indptr)
                idx = po[order].astype(np.int32)
                ww, dd = w[m][order], ds[m][order].astype(np.int32)
                pl.add_csr(a, b, indptr, idx, ww, dd, port)
                self.realised.append((a, b, indptr, idx, ww, dd, port))

    def _realise_drive(self, pl, proj, port):
        """A poisson_generator connected one_to_one: unit u of the device
        population (its position in the device's view) drives the neuron at
        the same position of the post view, on the kernel's block-key stream
        of the device population's name (``_kernel/models/devices.py``)."""
        dev = proj.pre.populations[0]
        prm = dev.params
        for p, local in proj.post.parts():
            if local.size != p.n or not np.array_equal(local, np.arange(p.n)):
                raise NotImplementedError("a poisson_generator drives whole neuron populations")
        if isinstance(proj.weight, S.Distribution) or isinstance(proj.delay, S.Distribution) or \
                proj.weight.size != 1 or proj.delay.size != 1:
            raise NotImplementedError("a poisson_generator takes one weight and one delay")
        w = float(proj.weight)
        ds = int(_delay_steps(np.array([float(proj.delay)]), self.dt)[0])
        t_min = _grid_steps(prm["start"], self.dt)
        t_max = 2 ** 62 if prm["stop"] is None else _grid_steps(prm["stop"], self.dt)
        units = proj.pre.gids - dev.gid_start  # device-local unit of each view position
        okey = S.object_key(self.net.seed, dev.name)
        pos = 0
        for p, _ in proj.post.parts():
            u = units[pos:pos + p.n]
            pos += p.n
            if u.size and not np.array_equal(u, np.arange(u[0], u[0] + u.size)):
                raise NotImplementedError("a population's drive units must be contiguous")
            u0 = int(u[0]) if u.size else 0
            pl.add_poisson_keyed(p.lib_pop, prm["rate"], w, ds, okey, u0, t_min, t_max,
                                 receptor=port)
            self.drives.append((p.lib_pop, prm["rate"], w, ds, okey, u0, t_min, t_max, port))

    def runner(self, batch=None, rng="independent"):
        return Runner(self, batch=batch, rng=rng)


class Recording(dict):
    """One observer's arrays: recordable -> (n_samples, n_columns), with the
    sample time stamps (window ends, ms) in ``times``."""


class Results:
    def __init__(self, recs):
        self._recs = recs

    def __getitem__(self, obs):
        return self._recs[obs.name if isinstance(obs, Observer) else obs]

    def __contains__(self, obs):
        return (obs.name if isinstance(obs, Observer) else obs) in self._recs


RNG_MODES = ("independent", "common")


def trial_indices(batch, rng="independent"):
    """Trial indices of a run (``_kernel/runner.py:84-113``): ``None`` -> trial
    0 (a uint32 scalar); ``B`` -> ``0 .. B-1`` ('independent') or ``B`` zeros
    ('common')."""
    if rng not in RNG_MODES:
        raise ValueError(f"rng must be one of {RNG_MODES}, got {rng!r}")
    if batch is None:
        return np.uint32(0)
    if isinstance(batch, bool) or not isinstance(batch, (int, np.integer)) or batch < 1:
        raise ValueError(f"batch must be a positive int or None, got {batch!r}")
    b = int(batch)
    return np.arange(b, dtype=np.uint32) if rng == "independent" else np.zeros(b, np.uint32)


class Runner:
    """Runs a program (``_kernel/runner.py:782-960``): ``simulate`` (from the
    initial state), ``cont`` (from the current state and time), ``reset``.

    ``batch=B`` runs B trials of the program: the same connectivity, weights,
    delays and initial state, with trial b's index folded into every
    ``poisson_generator`` step key ('independent'; 'common' gives every trial
    trial 0's numbers), so trial 0 equals the unbatched run.  Every recording
    then has a leading trial axis.  Each distinct trial index is one library
    plan run on the device after the other; 'common' runs one plan and repeats
    its recordings."""

    def __init__(self, program, batch=None, rng="independent"):
        if not isinstance(program, Program):
            raise TypeError(f"Runner needs a Program, got {type(program).__name__}")
        self._trials = trial_indices(batch, rng)
        if program.trial != 0:
            raise ValueError("a Runner starts from the program of trial 0")
        self.program = program
        self.batch = None if batch is None else int(batch)
        self.rng = rng
        self._progs = {0: program}
        if self.batch is not None:
            for t in sorted(set(int(x) for x in self._trials) - {0}):
                self._progs[t] = Program(program.net, program.precision,
                                         spike_capacity=program.spike_capacity, trial=t)
        self.n = 0
        self.h2d_bytes = self.d2h_bytes = 0

    @property
    def trials(self):
        """Trial indices (uint32; a scalar unbatched, ``(batch,)`` batched)."""
        return self._trials

    @property
    def t(self):
        return self.n * self.program.dt  # ms

    def reset(self):
        self.h2d_bytes = 0
        for prog in self._progs.values():
            prog.plan.restore(prog._ck0)
            self.h2d_bytes += int(prog._ck0.nbytes)
        self.n = 0

    def simulate(self, duration):
        self.reset()
        return self.cont(duration)

    def cont(self, duration):
        n_steps = _steps(duration, self.program.dt, "duration")
        for o in self.program.net.observers:
            o.n_samples(n_steps)
        self.d2h_bytes = 0
        per = {t: self._run_one(prog, n_steps) for t, prog in self._progs.items()}
        self.n += n_steps
        if self.batch is None:
            return Results(per[0])
        recs = {}
        for name, r0 in per[0].items():
            rec = Recording()
            for key in r0:
                rec[key] = np.stack([per[int(t)][name][key] for t in self._trials])
            rec.times = r0.times
            recs[name] = rec
        return Results(recs)

    def _run_one(self, prog, n_steps):
        pl = prog.plan
        pl.run(n_steps)
        st, g = pl.spikes(sort=False)  # binned into counts below: order is irrelevant
        v = pl.v_trace(np.float32 if prog.precision == 32 else np.float64) \
            if prog.rec_v.size else None
        # bytes read back from the device by this call (spike pairs, V_m)
        self.d2h_bytes += int(st.nbytes + g.nbytes + (v.nbytes if v is not None else 0))
        recs = {}
        for o in prog.net.observers:
            k, ns = o.interval, o.n_samples(n_steps)
            cols = prog.obs_cols[o.name]
            rec = Recording()
            if "spike" in o.recordables:
                counts = np.zeros((ns, cols.size), np.float64)
                pos = prog.obs_pos[o.name]
                col = pos[g] if g.size else np.zeros(0, np.int64)
                ok = col >= 0
                np.add.at(counts, ((st[ok] - self.n) // k, col[ok]), 1.0)
                rec["spike"] = counts
            if "V_m" in o.recordables:
                at = np.searchsorted(prog.rec_v, cols)
                vk = v[k - 1::k]
                # an observer of every recorded column in order takes the
                # trace as it is (no gather copy)
                full = at.size == v.shape[1] and np.array_equal(at, np.arange(at.size))
                rec["V_m"] = vk if full else vk[:, at]
            rec.times = (self.n + (np.arange(ns) + 1) * k) * prog.dt
            recs[o.name] = rec
        return recs
