"""Minimal unit layer in NEST units (ms, mV, pA, pF, nS, Hz).

The reference takes brainunit Quantities (``1.5 * u.ms``).  When brainunit is
importable its Quantities are accepted directly; otherwise this module's own
``Quantity`` plays the same role.  Plain numbers are read as NEST units.
"""
from __future__ import annotations

import numpy as np

# scale of each unit relative to the NEST unit of its dimension
_DIMS = {
    "ms": ("time", 1.0), "second": ("time", 1000.0), "s": ("time", 1000.0),
    "us": ("time", 1e-3),
    "mV": ("voltage", 1.0), "V": ("voltage", 1000.0),
    "pA": ("current", 1.0), "nA": ("current", 1000.0),
    "pF": ("capacitance", 1.0), "nF": ("capacitance", 1000.0),
    "nS": ("conductance", 1.0), "uS": ("conductance", 1000.0),
    "Hz": ("rate", 1.0), "kHz": ("rate", 1000.0),
    "1": ("unitless", 1.0),
}


class Unit:
    def __init__(self, name):
        self.name = name
        self.dim, self.scale = _DIMS[name]

    def __rmul__(self, value):
        return Quantity(value, self)

    def __repr__(self):
        return self.name


class Quantity:
    """A value (scalar or array) with a unit; ``.to(unit)`` gives the mantissa."""

    def __init__(self, value, unit: Unit):
        self.value = np.asarray(value, dtype=np.float64) if not np.isscalar(value) else float(value)
        self.unit = unit

    def to(self, unit: Unit):
        if unit.dim != self.unit.dim:
            raise TypeError(f"unit mismatch: {self.unit.name} is not {unit.name}")
        return self.value * (self.unit.scale / unit.scale)

    def __mul__(self, other):
        return Quantity(self.value * other, self.unit)

    __rmul__ = __mul__

    def __neg__(self):
        return Quantity(-self.value, self.unit)

    def __repr__(self):
        return f"{self.value} * {self.unit.name}"


ms, second, mV, pA, pF, nS, Hz = (Unit(n) for n in ("ms", "second", "mV", "pA", "pF", "nS", "Hz"))
UNITLESS = Unit("1")

_DIM_OF_NEST = {"time": ms, "voltage": mV, "current": pA, "capacitance": pF,
                "conductance": nS, "rate": Hz, "unitless": UNITLESS}


def mantissa(x, unit: Unit):
    """Value of ``x`` in ``unit``; plain numbers are taken to be in ``unit``."""
    if x is None:
        return None
    if isinstance(x, Quantity):
        return x.to(unit)
    # brainunit Quantity (duck-typed: has .mantissa and .unit and to_decimal)
    if hasattr(x, "to_decimal") and hasattr(x, "mantissa"):
        import brainunit as bu  # only reachable when brainunit is installed
        return np.asarray(x.to_decimal(getattr(bu, unit.name)))
    return np.asarray(x, dtype=np.float64) if not np.isscalar(x) else float(x)
