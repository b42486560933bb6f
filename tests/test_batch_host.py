"""CPU checks of the batch description API: argument validation and the
sweep configuration.  Nothing here uploads or launches a kernel."""
import math

import numpy as np
import pytest

from brainpy.state_b200 import _lib, brunel

ALPHA = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]


def test_batch_rejects_unsupported_configs():
    with pytest.raises(NotImplementedError):
        _lib.Batch(0.1, "aeif_cond_alpha")
    with pytest.raises(ValueError):
        _lib.Batch(0.1, precision=16)


def test_batch_instance_validation():
    b = _lib.Batch(0.1, semantics=_lib.RING)
    k = b.add_instance()
    e = b.add_pop(k, 100, ALPHA)
    i = b.add_pop(k, 25, ALPHA)
    with pytest.raises(ValueError, match="Capacitance"):
        b.add_pop(k, 3, [0.0, -1.0] + ALPHA[2:])
    with pytest.raises(ValueError, match="out of range"):
        b.add_fixed_indegree(k, e, 7, 10, 1, 1.0, 15)
    with pytest.raises(ValueError, match="instance"):
        b.add_fixed_indegree(k + 5, e, i, 10, 1, 1.0, 15)
    with pytest.raises(ValueError, match="delay"):
        b.add_fixed_indegree(k, e, i, 10, 1, 1.0, 0)
    b.add_fixed_indegree(k, e, i, 10, 1, 1.0, 15)
    with pytest.raises(NotImplementedError, match="one delay"):
        b.add_fixed_indegree(k, i, e, 10, 1, 1.0, 12)
    with pytest.raises(NotImplementedError, match="64 steps"):
        k2 = b.add_instance()
        p2 = b.add_pop(k2, 10, ALPHA)
        b.add_fixed_indegree(k2, p2, p2, 2, 1, 1.0, 80)
    with pytest.raises(ValueError, match="rate"):
        b.add_poisson(k, e, -5.0, 1.0, 15, 3)
    with pytest.raises(RuntimeError, match="not uploaded"):
        b.run(10)
    b.close()


def test_sweep_configuration():
    specs = brunel.sweep_instances()
    assert len(specs) == 256
    ne = np.array([s["NE"] for s in specs])
    assert ne.min() >= 500 and ne.max() <= 8000
    assert all(s["NI"] == s["NE"] // 4 for s in specs)
    g = np.array([s["g"] for s in specs])
    eta = np.array([s["eta"] for s in specs])
    assert g.min() >= 3 and g.max() <= 8 and eta.min() >= 0.9 and eta.max() <= 4
    p = brunel._instance_params(specs[0])
    assert p["CE"] == int(0.1 * specs[0]["NE"]) and p["CI"] == int(0.1 * specs[0]["NI"])
    # external rate eta * nu_thr * CE is size independent
    q = brunel.brunel_params(2500, g=specs[0]["g"], eta=specs[0]["eta"])
    assert p["rate"] == q["rate"]
