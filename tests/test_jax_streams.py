"""The reference's random streams: JAX's threefry PRNG (partitionable layout),
jax.random.uniform / normal, and the key-derived streams of the reference's
kernel path, restated twice -- in the product library (host C++) and in the
oracle (C) -- and pinned to values JAX itself publishes.

Golden values (JAX's documentation of jax.random; JAX is not installed here):
  * jax.random.split(jax.random.key(0)) ==
        [[1797259609, 2579123966], [928981903, 3453687069]]
    (the partitionable split: subkey i = threefry(key, (0, i)), which is also
    fold_in(key, i));
  * jax.random.uniform(jax.random.key(0)) == 0.947667 (float32);
  * jax.random.normal(jax.random.key(0)) == 1.6226422 (float32).
The float32 printouts are shortest round-trip forms, so each names one float32.

Tolerances: uniform draws and fold_in are bit-exact (integer and exactly
rounded float operations); float32 normal draws equal between the two
restatements bit for bit (same polynomial, same libm log1p); float64 normal
draws agree to 4 ulp and erfinv to 1e-15 relative against scipy; Poisson
counts are integers and must be equal.
"""
import numpy as np
import pytest

from brainpy.state_b200 import _lib


@pytest.fixture(scope="module")
def O(oracle):
    return oracle


def test_split_and_fold_in_match_jax_published_keys(O):
    key0 = np.array([0, 0], np.uint32)
    want = [[1797259609, 2579123966], [928981903, 3453687069]]
    for i in range(2):
        assert list(_lib.jax_fold_in(key0, i)) == want[i]
        assert list(O.jax_fold_in(key0, i)) == want[i]
    assert [list(k) for k in O.jax_split(key0, 2)] == want


def test_uniform_and_normal_match_jax_published_values(O):
    key0 = np.array([0, 0], np.uint32)
    assert np.float32(_lib.jax_uniform(key0, 1, 32)[0]) == np.float32("0.947667")
    assert np.float32(O.jax_uniform(key0, 1, 32)[0]) == np.float32("0.947667")
    assert np.float32(_lib.jax_normal(key0, 1, 32)[0]) == np.float32("1.6226422")
    assert np.float32(O.jax_normal(key0, 1, 32)[0]) == np.float32("1.6226422")


@pytest.mark.parametrize("bits,lo,hi", [(32, 0.0, 1.0), (32, 0.0, 20.0), (32, 1.0, 3.0),
                                        (32, -7.5, 2.25), (64, 0.0, 20.0), (64, 1.0, 3.0),
                                        (64, -7.5, 2.25)])
def test_uniform_library_equals_oracle_bitwise(O, bits, lo, hi):
    key = np.array([123, 4567], np.uint32)
    a = _lib.jax_uniform(key, 300000, bits, lo, hi)
    b = O.jax_uniform(key, 300000, bits, lo, hi)
    np.testing.assert_array_equal(a, b)
    assert a.min() >= lo and a.max() < hi
    if bits == 32:
        np.testing.assert_array_equal(a, a.astype(np.float32).astype(np.float64))
    # the uniform of a key's element i does not depend on how many are drawn
    np.testing.assert_array_equal(_lib.jax_uniform(key, 17, bits, lo, hi), a[:17])


def test_normal_library_equals_oracle(O):
    key = np.array([9, 99], np.uint32)
    a32, b32 = _lib.jax_normal(key, 200000, 32), O.jax_normal(key, 200000, 32)
    np.testing.assert_array_equal(a32, b32)
    a64, b64 = _lib.jax_normal(key, 200000, 64), O.jax_normal(key, 200000, 64)
    ulp = np.spacing(np.abs(b64))
    assert np.max(np.abs(a64 - b64) / ulp) <= 4
    for a in (a32, a64):
        assert abs(a.mean()) < 0.01 and abs(a.std() - 1.0) < 0.01


def test_erfinv_f64_accuracy():
    from scipy.special import erfinv
    key = np.array([5, 6], np.uint32)
    u = _lib.jax_uniform(key, 50000, 64, np.nextafter(-1.0, 0.0), 1.0)
    z = _lib.jax_normal(key, 50000, 64)
    ref = np.sqrt(2.0) * erfinv(u)
    np.testing.assert_allclose(z, ref, rtol=1e-15, atol=1e-300)


@pytest.mark.parametrize("rate", [17789.0, 5000.0, 50000.0, 1.0, 95000.0])
def test_kernel_poisson_table_equals_literal_inversion(O, rate):
    """The library's integer thresholds give the counts of the reference's
    float32 inversion loop (restated literally in the oracle) for every draw,
    including the largest mantissa value."""
    dt = 0.1
    lam32 = np.float32(rate * dt / 1000.0)
    T = _lib.kernel_poisson_table(rate, dt)
    obj = np.array([0, 42], np.uint32)
    for step in (1, 2, 777):
        for block in (0, 3):
            sk = O.kernel_step_key(obj, block, step)
            for lane in range(0, 1024, 3):
                y0, y1 = O.threefry2x32(sk, (0, lane))
                m = (y0 ^ y1) >> 9
                cnt = int(np.sum(np.cumprod(m > T.astype(np.int64))))
                assert cnt == O.kernel_poisson_count(sk, lane, lam32)
    # the top draw m = 2^23 - 1 against the table's saturation
    top = (1 << 23) - 1
    cnt_top = int(np.sum(np.cumprod(top > T.astype(np.int64))))
    assert cnt_top <= T.size


def test_kernel_poisson_rejects_large_means():
    with pytest.raises(Exception):
        _lib.kernel_poisson_table(200000.0, 0.1)   # lam = 20: jax.random.poisson branch
