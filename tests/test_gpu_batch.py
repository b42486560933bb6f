"""GPU tests of the batched-instances kernel and the GPU connectivity builder.

  * connectivity: bit-exact against the oracle's fixed_indegree + csr_structure
    (the reference's key derivation), for the stand-alone builder and for
    every projection of every batch instance;
  * FP64 batch: identical spike rasters to the float64 oracle of each
    instance over a horizon shorter than the networks' divergence time
    (atomic accumulation order differs, so V_m agrees to 1e-9 mV, not
    bitwise), with runs split in the middle of windows;
  * FP32 batch: per-instance rate within 5 % (+ 0.5 Hz) of the FP64 batch
    over 1 s;
  * the autotuner restores the state it found.
"""
import numpy as np
import pytest

from brainpy.state_b200 import _lib, brunel

pytestmark = pytest.mark.gpu

RING = _lib.RING


def _specs():
    return [dict(NE=160, NI=40, g=5.0, eta=2.0, seed=3, delay_steps=15),
            dict(NE=333, NI=83, g=3.5, eta=1.4, seed=11, delay_steps=15),
            dict(NE=90, NI=22, g=6.0, eta=3.0, seed=17, delay_steps=15)]


def _oracle_instance(oracle, spec, semantics=RING):
    p = brunel._instance_params(spec)
    sim = oracle.OracleSim(0.1, "iaf_psc_alpha", semantics=semantics)
    e = sim.add_pop(p["NE"], p["neuron"])
    i = sim.add_pop(p["NI"], p["neuron"])
    sim.add_drive(e, p["rate"], p["J_ex"], 15, brunel.derive_seed(spec["seed"], 0))
    sim.add_drive(i, p["rate"], p["J_ex"], 15, brunel.derive_seed(spec["seed"], 1))
    sizes = (p["NE"], p["NI"])
    for pre, post, K, s, w in brunel._instance_projs(spec, p):
        pr, po = oracle.fixed_indegree(s, sizes[pre], sizes[post], K, pre == post, True, 32)
        _, idx, indptr = oracle.csr_structure(pr, po, sizes[pre])
        sim.add_proj(pre, post, indptr, idx, np.full(idx.size, w),
                     np.full(idx.size, spec["delay_steps"], np.int32))
    ve, vi = brunel._instance_v0(spec)
    sim.set_state(e, "V_m", ve)
    sim.set_state(i, "V_m", vi)
    return sim, p


@pytest.mark.parametrize("case", [(300, 200, 20, False, True, 32), (250, 250, 17, True, False, 32),
                                  (120, 90, 33, True, True, 64), (1, 5, 4, False, True, 32)])
def test_gpu_fixed_indegree_matches_oracle(oracle, case):
    n_pre, n_post, K, same, auto, nbits = case
    indptr, post = _lib.gen_fixed_indegree(77, n_pre, n_post, K, same, auto, nbits)
    pr, po = oracle.fixed_indegree(77, n_pre, n_post, K, same, auto, nbits)
    _, idx, optr = oracle.csr_structure(pr, po, n_pre)
    np.testing.assert_array_equal(indptr, optr)
    np.testing.assert_array_equal(post, idx)


def test_batch_edges_match_oracle(oracle):
    specs = _specs()
    b, params = brunel.build_batch(specs, precision=64, tile=64)
    for k, (spec, p) in enumerate(zip(specs, params)):
        pre, post, proj = b.edges(k)
        got = np.stack([proj, pre, post], 1)
        want = []
        off = (0, p["NE"])
        sizes = (p["NE"], p["NI"])
        for j, (a, c, K, s, w) in enumerate(brunel._instance_projs(spec, p)):
            pr, po = oracle.fixed_indegree(s, sizes[a], sizes[c], K, a == c, True, 32)
            want.append(np.stack([np.full(pr.size, j), pr + off[a], po + off[c]], 1))
        want = np.concatenate(want)
        key = lambda m: m[np.lexsort((m[:, 2], m[:, 1], m[:, 0]))]
        np.testing.assert_array_equal(key(got), key(want))
    b.close()


def _raster(st, ids):
    return set(zip(st.tolist(), ids.tolist()))


def test_batch_fp64_matches_oracle_with_split_runs(oracle):
    specs = _specs()
    b, params = brunel.build_batch(specs, precision=64, tile=64, record=(0, 1, 2))
    sims = [_oracle_instance(oracle, s)[0] for s in specs]
    total = {k: set() for k in range(len(specs))}
    want = {k: set() for k in range(len(specs))}
    for chunk in (37, 100, 63):  # windows of 15 steps: every run ends mid-window
        b.run(chunk)
        for k, sim in enumerate(sims):
            st, ids = b.spikes(k)
            total[k] |= _raster(st, ids)
            ost, og, _ = sim.run(chunk)
            want[k] |= _raster(ost, og)
    for k in range(len(specs)):
        assert len(want[k]) > 0
        assert total[k] == want[k]
        n = specs[k]["NE"]
        np.testing.assert_allclose(b.get_state(k, 0, "V_m"), sims[k].get_state(0, "V_m", n),
                                   rtol=0, atol=1e-9)
        counts = b.spike_counts(k)
        assert counts.sum() == len(want[k])
    b.close()


def test_batch_fp32_rates_track_fp64():
    specs = brunel.sweep_instances(n=12, seed=5, ne_range=(500, 2000))
    b64, _ = brunel.build_batch(specs, precision=64)
    b32, _ = brunel.build_batch(specs, precision=32)
    b64.run(10000)
    b32.run(10000)
    for k, s in enumerate(specs):
        n = s["NE"] + s["NI"]
        r64 = b64.spike_counts(k).sum() / n
        r32 = b32.spike_counts(k).sum() / n
        assert abs(r32 - r64) <= 0.05 * r64 + 0.5, (k, s, r32, r64)
    b64.close()
    b32.close()


def test_batch_tuner_restores_state():
    specs = _specs()
    b, _ = brunel.build_batch(specs, precision=64, record=(0, 1, 2))
    T, c, ms = b.tune(pilot_steps=60)
    assert T in (128, 256, 512) and c >= 1 and ms > 0
    assert b.step == 0
    b.run(150)
    ref, _ = brunel.build_batch(specs, precision=64, tile=T, ctas_per_sm=c, record=(0, 1, 2))
    ref.run(150)
    for k in range(len(specs)):
        assert _raster(*b.spikes(k)) == _raster(*ref.spikes(k))
    b.close()
    ref.close()
