"""The reference's random streams on the host: key chains and distributions.

Both front ends realise random parameters (distributed weights, per-edge
delays, initial states) with the reference's own draws for the same seed:
JAX's threefry PRNG in its partitionable layout, restated in the library
(``bspk_jax_fold_in`` / ``bspk_jax_uniform`` / ``bspk_jax_normal``).

Kernel path (``_kernel/rng.py:106-200``, ``_kernel/compiler.py:95-97,819-850``,
``_kernel/params.py:183-354``):

* ``root_key(seed) = PRNGKey(seed) = (0, seed)``;
* ``object_key(seed, name) = fold(fold(root, hi), lo)``, ``(hi, lo)`` the
  blake2b id of the object's name;
* a population's initial state ``s`` draws from
  ``name_key(fold(object_key, INIT_STREAM), s)``, ``name_key(k, s) =
  fold(k, crc32(s) & 0x7fffffff)``;
* a projection's weights draw from ``fold(object_key, WEIGHT_STREAM)`` and its
  delays from ``fold(object_key, DELAY_STREAM)``, one value per edge in the
  rule's canonical order (post-major, pre ascending).

Legacy ``Simulator`` path (``_nest_network/event_proj.py:148-149,286-291``,
``_dist.py:40-77``): ``k_conn, k_w, k_rec = split(key(seed), 3)``; weights draw
from ``k_w`` in the sampler's edge order (post-major, draw order), before the
CSR sort.

Distributions follow the kernel's ``_kernel/params.py`` forms (``Uniform(low,
high)`` draws ``jax.random.uniform(key, shape, dtype, low, high)`` and clips;
``Normal`` is ``mean + std * normal``; ``LogNormal`` is ``exp(mu + sigma *
normal)``) or, with ``legacy=True``, the legacy ``_dist.py`` forms
(``low + (high - low) * uniform01``).  Float32 arithmetic is done in numpy
float32 (IEEE, unfused), so uniform draws are bit-exact; normal draws use the
library's erfinv (XLA's float32 polynomial; float64 to an ulp or two) and
LogNormal numpy's exp, so their last bits may differ from XLA's.
"""
from __future__ import annotations

import hashlib
import zlib

import numpy as np

from . import _lib
from .units import Quantity, Unit, mantissa

INIT_STREAM = 0xFFFFFFFE
WEIGHT_STREAM = 0xFFFFFFFD
DELAY_STREAM = 0xFFFFFFFC
GID_BLOCK = 1024

__all__ = ["INIT_STREAM", "WEIGHT_STREAM", "DELAY_STREAM", "GID_BLOCK", "root_key", "fold_in",
           "split", "name_id", "object_key", "name_key", "Distribution", "Uniform", "Normal",
           "LogNormal", "delay_steps"]


def root_key(seed):
    """``jax.random.PRNGKey(seed)`` for a seed in [0, 2**32): (0, seed)."""
    if isinstance(seed, bool) or int(seed) != seed or not 0 <= int(seed) < 2 ** 32:
        raise ValueError(f"seed must be an int in [0, 2**32), got {seed!r}")
    return np.array([0, int(seed)], np.uint32)


def fold_in(key, data):
    return _lib.jax_fold_in(key, data)


def split(key, num):
    """``jax.random.split(key, num)`` (partitionable: subkey i = fold(key, i))."""
    return [fold_in(key, i) for i in range(int(num))]


def name_id(name):
    """Stable 64-bit id of an object name as (hi, lo): the first eight bytes
    of blake2b(name) read big-endian (``_kernel/rng.py:122-150``)."""
    if not isinstance(name, str) or not name:
        raise TypeError(f"object name must be a non-empty str, got {name!r}")
    d = hashlib.blake2b(name.encode("utf-8"), digest_size=8).digest()
    return int.from_bytes(d[:4], "big"), int.from_bytes(d[4:], "big")


def object_key(seed, name):
    hi, lo = name_id(name)
    return fold_in(fold_in(root_key(seed), hi), lo)


def name_key(key, name):
    """``fold_in(key, crc32(name) & 0x7fffffff)`` (``_kernel/params.py:348-354``)."""
    return fold_in(key, zlib.crc32(name.encode()) & 0x7FFFFFFF)


def _dtype(bits):
    return np.float32 if bits == 32 else np.float64


def _unit_of(x):
    return x.unit if isinstance(x, Quantity) else None


def _mant(x, unit):
    return None if x is None else float(mantissa(x, unit)) if unit is not None else float(x)


class Distribution:
    """Unit-aware random value specification (``_kernel/params.py:139-206``):
    ``sample(key, n, bits)`` gives mantissas in ``unit``, clipped to
    [low, high] when given, as float64 holding the draw dtype's values."""

    unit: Unit | None = None
    low = high = None
    legacy = False

    def _draw(self, key, n, bits):  # pragma: no cover - abstract
        raise NotImplementedError

    def sample(self, key, n, bits=32):
        m = np.asarray(self._draw(key, int(n), int(bits)), dtype=_dtype(bits))
        if self.low is not None or self.high is not None:
            lo = -np.inf if self.low is None else self.low
            hi = np.inf if self.high is None else self.high
            m = np.clip(m, _dtype(bits)(lo), _dtype(bits)(hi))
        return m.astype(np.float64)

    def sample_in(self, key, n, unit, bits=32):
        """Samples converted to ``unit`` (in the draw dtype)."""
        m = self.sample(key, n, bits)
        if self.unit is None or unit is None or self.unit.name == unit.name:
            return m
        f = _dtype(bits)(Quantity(1.0, self.unit).to(unit))
        return (m.astype(_dtype(bits)) * f).astype(np.float64)


class Uniform(Distribution):
    """Uniform on [low, high).  Kernel form: ``jax.random.uniform(key, shape,
    dtype, low, high)`` then clip; ``legacy=True``: ``low + (high - low) *
    jax.random.uniform(key, shape)`` (``_dist.py:66-77``)."""

    def __init__(self, low, high, *, legacy=False):
        self.unit = _unit_of(low) or _unit_of(high)
        self.low, self.high = _mant(low, self.unit), _mant(high, self.unit)
        if self.low > self.high:
            raise ValueError(f"low > high: {low} > {high}")
        self.legacy = bool(legacy)

    def sample(self, key, n, bits=32):
        if not self.legacy:
            return Distribution.sample(self, key, n, bits)
        t = _dtype(bits)
        u = _lib.jax_uniform(key, n, bits, 0.0, 1.0).astype(t)
        return (t(self.low) + t(self.high - self.low) * u).astype(np.float64)

    def _draw(self, key, n, bits):
        return _lib.jax_uniform(key, n, bits, self.low, self.high)


class Normal(Distribution):
    """``mean + std * jax.random.normal(key, shape, dtype)``, optionally clipped."""

    def __init__(self, mean, std, *, low=None, high=None, legacy=False):
        self.unit = _unit_of(mean) or _unit_of(std)
        self.mean, self.std = _mant(mean, self.unit), _mant(std, self.unit)
        if self.std < 0:
            raise ValueError(f"std must be non-negative, got {std}")
        self.low, self.high = _mant(low, self.unit), _mant(high, self.unit)
        self.legacy = bool(legacy)

    def _draw(self, key, n, bits):
        t = _dtype(bits)
        z = _lib.jax_normal(key, n, bits).astype(t)
        return t(self.mean) + t(self.std) * z


class LogNormal(Distribution):
    """``exp(mu + sigma * jax.random.normal(key, shape, dtype))`` in ``unit``."""

    def __init__(self, mu, sigma, *, unit=None, low=None, high=None, legacy=False):
        self.unit = unit
        self.mu, self.sigma = float(mu), float(sigma)
        if self.sigma < 0:
            raise ValueError(f"sigma must be non-negative, got {sigma}")
        self.low, self.high = _mant(low, unit), _mant(high, unit)
        self.legacy = bool(legacy)

    def _draw(self, key, n, bits):
        t = _dtype(bits)
        z = _lib.jax_normal(key, n, bits).astype(t)
        return np.exp(t(self.mu) + t(self.sigma) * z)


def delay_steps(d_ms, dt_ms, bits=64):
    """NEST's rounding of delays to steps (``_kernel/delays.py:50-98``):
    floor(d * steps_per_ms + 0.5) in float64, where values drawn in float32
    that lie within 8 float32 epsilons of a half step round half up as NEST
    does for the decimal the user wrote."""
    d = np.asarray(d_ms, dtype=np.float64)
    if d.size and (not np.all(np.isfinite(d)) or d.min() < 0):
        raise ValueError(f"delays must be finite and non-negative, got min {d.min()} ms")
    spm = 1.0 / float(dt_ms)
    k = np.rint(spm)
    if k >= 1 and abs(spm - k) <= 1e-6 * k:
        spm = float(k)
    y = d * spm + 0.5
    out = np.floor(y)
    if bits == 32:
        eps = float(np.finfo(np.float32).eps)
        r = np.rint(y)
        out = np.where(np.abs(y - r) <= 8 * eps * np.maximum(y, 1.0), r, out)
    return out.astype(np.int64)
