"""CPU checks of the C ABI: the library loads, exports every declared symbol,
and its host logic (validation, connectivity sampling, Poisson tables) agrees
with the oracle.  Nothing here launches a kernel."""
import math
import os
import re

import numpy as np
import pytest

from brainpy.state_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bspk_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _declared("bspk.h")
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    for n in _declared("bspk_xla.h"):
        assert hasattr(L, n), n
    assert b"sm_100a" in L.bspk_version()


ALPHA = [0.0, 250.0, 20.0, 2.0, 20.0, 10.0, 0.5, 0.5, 0.0, -math.inf]


def test_validation_errors_match_reference_messages():
    pl = _lib.Plan(0.1)
    with pytest.raises(ValueError, match="Capacitance"):
        pl.add_pop(3, [0.0, -1.0] + ALPHA[2:])
    with pytest.raises(ValueError, match="Reset potential"):
        pl.add_pop(3, ALPHA[:4] + [10.0, 20.0] + ALPHA[6:])
    with pytest.raises(ValueError, match="refractory"):
        pl.add_pop(3, ALPHA[:3] + [-1.0] + ALPHA[4:])
    a = pl.add_pop(3, ALPHA)
    with pytest.raises(ValueError):
        pl.add_csr(a, 5, np.zeros(4, np.int64), np.zeros(0, np.int32), np.zeros(0), np.zeros(0))
    with pytest.raises(ValueError, match="post index"):
        pl.add_csr(a, a, np.array([0, 1, 1, 1]), np.array([7]), np.ones(1), np.ones(1))
    with pytest.raises(ValueError, match="indptr"):
        pl.add_csr(a, a, np.array([0, 2, 1, 1]), np.array([0]), np.ones(1), np.ones(1))
    with pytest.raises(ValueError, match="rate"):
        pl.add_poisson(a, 1e9, 1.0, 1, 0)
    with pytest.raises(NotImplementedError):
        _lib.Plan(0.1, precision=32, deterministic=True)
    with pytest.raises(RuntimeError, match="not uploaded"):
        pl.run(10)


def test_stdp_validation():
    pl = _lib.Plan(0.1)
    a = pl.add_pop(2, ALPHA)
    j = pl.add_csr(a, a, np.array([0, 1, 2]), np.array([1, 0]), np.array([1.0, 1.0]),
                   np.array([3, 3]))
    with pytest.raises(ValueError, match="same sign"):
        pl.attach_stdp(j, Wmax=-1.0)
    with pytest.raises(ValueError, match="tau_plus"):
        pl.attach_stdp(j, tau_plus=-1.0)
    k = pl.add_csr(a, a, np.array([0, 1, 2]), np.array([1, 0]), np.array([1.0, 1.0]),
                   np.array([3, 4]))
    with pytest.raises(NotImplementedError, match="homogeneous delay"):
        pl.attach_stdp(k)
    pl.attach_stdp(j)


@pytest.mark.parametrize("nbits,auto", [(32, True), (64, True), (32, False)])
def test_fixed_indegree_matches_oracle_sampler(oracle, nbits, auto):
    # library sampler (C++) == oracle restatement (C) of
    # _nest_network/connectivity.py:101-135 + csr_structure :39-53
    pl = _lib.Plan(0.1)
    e = pl.add_pop(300, ALPHA)
    i = pl.add_pop(75, ALPHA)
    seed = (1 * 1_000_003 + 2 + 1) & 0x7FFFFFFF
    pj = pl.add_fixed_indegree(e, i, 30, seed, 20.68, delay_const=15, allow_autapses=auto,
                               nbits=nbits)
    pk = pl.add_fixed_indegree(e, e, 30, seed + 1, 20.68, delay_const=15, allow_autapses=auto,
                               nbits=nbits)
    for proj, n_post, s, pre_is_post in ((pj, 75, seed, False), (pk, 300, seed + 1, True)):
        indptr, post, d, w = pl.csr(proj)
        pre_o, post_o = oracle.fixed_indegree(s, 300, n_post, 30, pre_is_post=pre_is_post,
                                              allow_autapses=auto, nbits=nbits)
        order, idx_o, indptr_o = oracle.csr_structure(pre_o, post_o, 300)
        np.testing.assert_array_equal(indptr, indptr_o)
        np.testing.assert_array_equal(post, idx_o)
        assert np.all(d == 15) and np.all(w == 20.68)
        if pre_is_post and not auto:
            pre_rows = np.repeat(np.arange(300), np.diff(indptr))
            assert np.all(pre_rows != post)


def test_poisson_cdf_counts_match_oracle(oracle):
    # host CDF table + device search == oracle sequential inversion; the
    # table itself is exercised through the oracle on boundary uniforms
    for lam in (0.05, 0.5, 1.7789, 30.0):
        for u in (0.0, 1e-300, 0.3, 0.999999, 1.0 - 2 ** -53):
            k = oracle.poisson(lam, u)
            F, p = [math.exp(-lam)], math.exp(-lam)
            for j in range(1, 4096):
                p = p * lam / j
                if not (F[-1] + p > F[-1]):
                    break
                F.append(F[-1] + p)
            ref = next((j for j, f in enumerate(F) if u <= f), len(F))
            assert k == ref, (lam, u)


def test_set_weights_on_library_drawn_connectivity():
    """Distributed weights on library-drawn fixed_indegree edges: the weights
    land in CSR order, the edges stay those of the sampler (host only)."""
    pl = _lib.Plan(0.1)
    a = pl.add_pop(50, ALPHA)
    j = pl.add_fixed_indegree(a, a, 7, 123, 1.0, delay_const=5)
    indptr, post, d, w = pl.csr(j)
    assert w.size == 350 and np.all(w == 1.0)
    new = np.linspace(0.5, 2.0, 350)
    pl.set_weights(j, new)
    indptr2, post2, d2, w2 = pl.csr(j)
    np.testing.assert_array_equal(w2, new)
    np.testing.assert_array_equal(post2, post)
    with pytest.raises(ValueError, match="every edge"):
        pl.set_weights(j, new[:10])
    pl.attach_stdp(j, Wmax=5.0)
    with pytest.raises(RuntimeError, match="before making the projection plastic"):
        pl.set_weights(j, new)
