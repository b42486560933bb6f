"""ctypes front end of the float64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
import this module; the product (``brainpy.state_b200``) never does.

What is pinned and what is not
------------------------------
* Pinned against the reference's own tests (``tests/test_oracle_golden.py``):
  the ``iaf_psc_alpha`` NEST trace and equation checks
  (``_nest_neuron/iaf_psc_alpha_test.py:57-127,200-245``), the ``iaf_psc_exp``
  first-spike time, the ``aeif_cond_alpha`` one-step current delay and RKF45
  reference loop, the STDP rule cases
  (``_nest_plasticity/stdp_synapse_rule_test.py``), the delay timing examples
  (``_nest_network/delay_test.py``, ``_kernel/delay_scatter.py:144-153``) and
  the CSR structure example (``_nest_network/connectivity_test.py:290-307``).
* Pinned against published known-answer vectors: the Threefry-2x32-20 block
  cipher (Random123).
* Parity unpinned: the JAX key-derivation layer (``fold_in``/``split``/
  ``randint`` on top of the cipher) and therefore concrete connectivity for a
  seed, because JAX cannot be installed or run in this build environment; and
  the Poisson stream, which is the library's own (JAX's ``poisson`` depends on
  XLA's float32 ``log``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MODEL_IDS = {"iaf_psc_alpha": 0, "iaf_psc_exp": 1, "aeif_cond_alpha": 2, "iaf_cond_exp": 3,
             "iaf_cond_alpha": 4, "iaf_psc_exp_multisynapse": 5}
LEGACY, RING = 0, 1


class BpttCfg(C.Structure):
    _fields_ = [("dt", C.c_double), ("n", C.c_int), ("n_in", C.c_int), ("batch", C.c_int),
                ("n_steps", C.c_int), ("n_readout", C.c_int), ("readout_tau", C.c_double),
                ("slope", C.c_double), ("relaxed", C.c_int), ("detach_reset", C.c_int),
                ("params", C.c_double * 9)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libbspk_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        i64, i32, u32, dbl, vp = C.c_int64, C.c_int32, C.c_uint32, C.c_double, C.c_void_p
        L.bo_create.restype = vp
        L.bo_create.argtypes = [dbl, C.c_int, C.c_int]
        L.bo_destroy.argtypes = [vp]
        L.bo_add_pop.argtypes = [vp, C.c_int, vp, C.c_int]
        L.bo_set_state.argtypes = [vp, C.c_int, C.c_char_p, vp]
        L.bo_get_state.argtypes = [vp, C.c_int, C.c_char_p, vp]
        L.bo_add_proj.argtypes = [vp, C.c_int, C.c_int, i64, vp, vp, vp, vp, C.c_int]
        L.bo_add_drive.argtypes = [vp, C.c_int, dbl, dbl, C.c_int, u32, i64, i64, C.c_int]
        L.bo_set_stdp.argtypes = [vp, C.c_int] + [dbl] * 7
        L.bo_set_stdp_triplet.argtypes = [vp, C.c_int] + [dbl] * 9
        L.bo_triplet_update.restype = dbl
        L.bo_triplet_update.argtypes = [dbl] * 12
        L.bo_get_weights.argtypes = [vp, C.c_int, vp]
        L.bo_record_v.argtypes = [vp, C.c_int, vp]
        L.bo_run.restype = i64
        L.bo_run.argtypes = [vp, i64, vp, vp, i64, vp]
        L.bo_step_neuron.argtypes = [vp, C.c_int, dbl, dbl, dbl]
        L.bo_step_neuron_ms.argtypes = [vp, C.c_int, vp, dbl]
        L.bo_set_ports.argtypes = [vp, C.c_int]
        L.bo_step_count.restype = i64
        L.bo_step_count.argtypes = [vp]
        L.bo_n_total.argtypes = [vp]
        L.bo_rk_substeps.restype = i64
        L.bo_rk_substeps.argtypes = [vp]
        L.bo_set_threads.argtypes = [vp, C.c_int]
        L.bo_threefry2x32.argtypes = [u32, u32, u32, u32, vp, vp]
        L.bo_jax_key.argtypes = [i64, vp]
        L.bo_jax_fold_in.argtypes = [vp, u32, vp]
        L.bo_jax_split.argtypes = [vp, C.c_int, vp]
        L.bo_jax_random_bits.argtypes = [vp, C.c_int, i64, vp]
        L.bo_jax_randint.argtypes = [vp, i64, i64, i64, C.c_int, vp]
        L.bo_fixed_indegree.argtypes = [i64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, vp, vp]
        L.bo_csr_structure.argtypes = [vp, vp, i64, C.c_int, vp, vp, vp]
        L.bo_jax_uniform.argtypes = [vp, C.c_int, i64, dbl, dbl, vp]
        L.bo_jax_normal.argtypes = [vp, C.c_int, i64, vp]
        L.bo_kernel_step_key.argtypes = [vp, u32, u32, vp]
        L.bo_kernel_poisson_count.restype = i64
        L.bo_kernel_poisson_count.argtypes = [vp, u32, C.c_float]
        L.bo_add_drive_keyed.argtypes = [vp, C.c_int, dbl, dbl, C.c_int, vp, i64, i64, i64,
                                         C.c_int]
        L.bo_set_trial.argtypes = [vp, u32]
        L.bo_set_trial.restype = None
        L.bo_uniform01.restype = dbl
        L.bo_uniform01.argtypes = [u32, u32, u32, u32]
        L.bo_poisson.argtypes = [dbl, dbl, dbl]
        L.bo_alpha_p31_p32.argtypes = [dbl, dbl, dbl, dbl, vp, vp]
        L.bo_propagator_exp.restype = dbl
        L.bo_propagator_exp.argtypes = [dbl, dbl, dbl, dbl]
        L.bo_lif_bptt.argtypes = [C.POINTER(BpttCfg), vp, vp, i64, vp, vp, vp, vp, vp, vp, vp,
                                  vp]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- RNG helpers

def threefry2x32(key, count):
    y0, y1 = C.c_uint32(), C.c_uint32()
    lib().bo_threefry2x32(int(key[0]), int(key[1]), int(count[0]), int(count[1]),
                          C.byref(y0), C.byref(y1))
    return y0.value, y1.value


def jax_key(seed):
    k = np.zeros(2, np.uint32)
    lib().bo_jax_key(int(seed), _p(k))
    return k


def jax_fold_in(key, data):
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(2, np.uint32)
    lib().bo_jax_fold_in(_p(k), int(data) & 0xFFFFFFFF, _p(out))
    return out


def jax_split(key, num):
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros((num, 2), np.uint32)
    lib().bo_jax_split(_p(k), int(num), _p(out))
    return out


def jax_randint(key, n, minval, maxval, nbits=32):
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(n, np.int64)
    lib().bo_jax_randint(_p(k), int(n), int(minval), int(maxval), int(nbits), _p(out))
    return out


def name_id(name):
    """(hi, lo) words of the first 8 bytes of blake2b(name) (_kernel/rng.py:122-150)."""
    import hashlib
    d = hashlib.blake2b(name.encode("utf-8"), digest_size=8).digest()
    return int.from_bytes(d[:4], "big"), int.from_bytes(d[4:], "big")


def kernel_fixed_indegree(seed, proj_name, parts, n_pre, self_pos, K):
    """Kernel-front-end fixed_indegree with multapses, one key per post neuron:
    object key fold(fold(PRNGKey(seed), hi), lo) of the projection name
    (_kernel/rng.py:152-175), then per part (population name, local ids)
    fold(fold(obj, hi_q), lo_q) and per local id l
    fold(fold(fold(., l // 1024), 0xFFFFFFFF), l % 1024) (rng.py:237-300);
    sources randint(key, (K,), 0, n_pre - has_self) shifted past the post's own
    position (_kernel/connectivity/rules.py:226-265).  Returns positions in the
    pre view, shape (n_post, K)."""
    hi, lo = name_id(proj_name)
    obj = jax_fold_in(jax_fold_in(jax_key(seed), hi), lo)
    rows = []
    j = 0
    for pop_name, local in parts:
        qh, ql = name_id(pop_name)
        pk = jax_fold_in(jax_fold_in(obj, qh), ql)
        for l in np.asarray(local, np.int64):
            kj = jax_fold_in(jax_fold_in(jax_fold_in(pk, int(l) // 1024), 0xFFFFFFFF),
                             int(l) % 1024)
            sp = int(self_pos[j]) if self_pos is not None else -1
            idx = jax_randint(kj, K, 0, n_pre - (1 if sp >= 0 else 0))
            if sp >= 0:
                idx = idx + (idx >= sp)
            rows.append(idx)
            j += 1
    return np.array(rows, np.int64).reshape(-1, K)


def fixed_indegree(seed, n_pre, n_post, K, pre_is_post=False, allow_autapses=True, nbits=32):
    pre = np.zeros(n_post * K, np.int32)
    post = np.zeros(n_post * K, np.int32)
    rc = lib().bo_fixed_indegree(int(seed), n_pre, n_post, K, int(pre_is_post),
                                 int(allow_autapses), int(nbits), _p(pre), _p(post))
    if rc != 0:
        raise ValueError("fixed_indegree failed")
    return pre, post


def csr_structure(pre, post, n_pre):
    pre = np.ascontiguousarray(pre, np.int32)
    post = np.ascontiguousarray(post, np.int32)
    n = pre.shape[0]
    order = np.zeros(n, np.int64)
    indices = np.zeros(n, np.int32)
    indptr = np.zeros(n_pre + 1, np.int64)
    rc = lib().bo_csr_structure(_p(pre), _p(post), n, int(n_pre), _p(order), _p(indices),
                                _p(indptr))
    if rc != 0:
        raise ValueError("csr_structure failed")
    return order, indices, indptr


def jax_uniform(key, n, bits=32, lo=0.0, hi=1.0):
    """jax.random.uniform(key, (n,), float32 / float64, lo, hi) as float64."""
    k = np.asarray(key, np.uint32).copy()
    out = np.zeros(int(n), np.float64)
    lib().bo_jax_uniform(_p(k), int(bits), int(n), float(lo), float(hi), _p(out))
    return out


def jax_normal(key, n, bits=32):
    """jax.random.normal(key, (n,), float32 / float64) as float64."""
    k = np.asarray(key, np.uint32).copy()
    out = np.zeros(int(n), np.float64)
    lib().bo_jax_normal(_p(k), int(bits), int(n), _p(out))
    return out


def kernel_step_key(obj_key, block, step):
    k = np.asarray(obj_key, np.uint32).copy()
    out = np.zeros(2, np.uint32)
    lib().bo_kernel_step_key(_p(k), int(block), int(step) & 0xFFFFFFFF, _p(out))
    return out


def kernel_poisson_count(step_key, lane, lam32):
    k = np.asarray(step_key, np.uint32).copy()
    return int(lib().bo_kernel_poisson_count(_p(k), int(lane), float(lam32)))


def uniform01(seed, stream, step, idx):
    return lib().bo_uniform01(seed, stream, step, idx)


def poisson(lam, u):
    return lib().bo_poisson(float(lam), float(np.exp(-lam)), float(u))


def alpha_p31_p32(tau_syn, tau_m, c_m, h):
    a, b = C.c_double(), C.c_double()
    lib().bo_alpha_p31_p32(tau_syn, tau_m, c_m, h, C.byref(a), C.byref(b))
    return a.value, b.value


def propagator_exp(tau_syn, tau_m, c_m, h):
    return lib().bo_propagator_exp(tau_syn, tau_m, c_m, h)


# ------------------------------------------------------------------ simulator

class OracleSim:
    """Serial float64 restatement of one network (test checker only)."""

    def __init__(self, dt, model="iaf_psc_alpha", semantics=LEGACY):
        self._L = lib()
        self.dt = float(dt)
        self.model = model
        self._h = self._L.bo_create(self.dt, int(semantics), MODEL_IDS[model])
        self._keep = []

    def set_threads(self, n):
        """OpenMP threads of the per-neuron phases (results do not change)."""
        self._L.bo_set_threads(self._h, int(n))

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.bo_destroy(self._h)
            self._h = None

    def add_pop(self, n, params):
        p = np.ascontiguousarray(params, np.float64)
        r = self._L.bo_add_pop(self._h, int(n), _p(p), int(p.size))
        if r < 0:
            raise ValueError("add_pop failed")
        return r

    def set_state(self, pop, name, values):
        v = np.ascontiguousarray(values, np.float64)
        if self._L.bo_set_state(self._h, pop, name.encode(), _p(v)) != 0:
            raise KeyError(name)

    def get_state(self, pop, name, n):
        v = np.zeros(n, np.float64)
        if self._L.bo_get_state(self._h, pop, name.encode(), _p(v)) != 0:
            raise KeyError(name)
        return v

    def add_proj(self, pre_pop, post_pop, indptr, post_local, w, delay_steps, receptor=0):
        indptr = np.ascontiguousarray(indptr, np.int64)
        post_local = np.ascontiguousarray(post_local, np.int32)
        w = np.ascontiguousarray(w, np.float64)
        d = np.ascontiguousarray(delay_steps, np.int32)
        r = self._L.bo_add_proj(self._h, pre_pop, post_pop, int(post_local.size), _p(indptr),
                                _p(post_local), _p(w), _p(d), int(receptor))
        if r < 0:
            raise ValueError(f"add_proj failed ({r})")
        return r

    def add_drive(self, post_pop, rate_hz, weight, delay_steps, seed, t_min=0,
                  t_max=2 ** 62, receptor=0):
        r = self._L.bo_add_drive(self._h, post_pop, float(rate_hz), float(weight),
                                 int(delay_steps), int(seed) & 0xFFFFFFFF, int(t_min),
                                 int(t_max), int(receptor))
        if r < 0:
            raise ValueError("add_drive failed")
        return r

    def set_trial(self, trial):
        """Trial index folded into the keyed drives' step keys (default 0)."""
        self._L.bo_set_trial(self._h, int(trial))

    def add_drive_keyed(self, post_pop, rate_hz, weight, delay_steps, obj_key, unit_off=0,
                        t_min=0, t_max=2 ** 62, receptor=0):
        k = np.asarray(obj_key, np.uint32).copy()
        r = self._L.bo_add_drive_keyed(self._h, post_pop, rate_hz, weight, delay_steps, _p(k),
                                       unit_off, t_min, t_max, receptor)
        if r < 0:
            raise ValueError("bad drive")
        return r

    def set_stdp(self, proj, tau_plus, tau_minus, lambda_, alpha, mu_plus, mu_minus, wmax):
        if self._L.bo_set_stdp(self._h, proj, tau_plus, tau_minus, lambda_, alpha, mu_plus,
                               mu_minus, wmax) != 0:
            raise ValueError("set_stdp failed")

    def set_stdp_triplet(self, proj, tau_plus, tau_plus_triplet, tau_minus, tau_minus_triplet,
                         Aplus, Aplus_triplet, Aminus, Aminus_triplet, Wmax):
        if self._L.bo_set_stdp_triplet(self._h, proj, tau_plus, tau_plus_triplet, tau_minus,
                                       tau_minus_triplet, Aplus, Aplus_triplet, Aminus,
                                       Aminus_triplet, Wmax) != 0:
            raise ValueError("set_stdp_triplet failed")

    def weights(self, proj, n_edges):
        w = np.zeros(n_edges, np.float64)
        self._L.bo_get_weights(self._h, proj, _p(w))
        return w

    def record_v(self, gids):
        self._rec = np.ascontiguousarray(gids, np.int32)
        self._L.bo_record_v(self._h, int(self._rec.size), _p(self._rec))

    def run(self, n_steps, cap=None):
        n_rec = int(getattr(self, "_rec", np.zeros(0)).size)
        if cap is None:
            cap = max(1024, self._L.bo_n_total(self._h) * n_steps // 20)
        st = np.zeros(cap, np.int64)
        gid = np.zeros(cap, np.int32)
        v = np.zeros((n_steps, n_rec), np.float64)
        n = self._L.bo_run(self._h, int(n_steps), _p(st), _p(gid), int(cap), _p(v))
        if n == -2:
            raise FloatingPointError(f"Numerical instability in {self.model} dynamics.")
        if n > cap:
            raise OverflowError("spike buffer too small")
        return st[:n], gid[:n], v

    def set_ports(self, separate):
        """iaf models: receptor ports 0 / 1 kept apart (signs kept)."""
        self._L.bo_set_ports(self._h, int(bool(separate)))

    def step_neuron_ms(self, gid, w, x_next=0.0):
        """One iaf_psc_exp_multisynapse update with weight w[k] into receptor k."""
        wv = np.zeros(4, np.float64)
        wv[:len(w)] = w
        r = self._L.bo_step_neuron_ms(self._h, int(gid), _p(wv), float(x_next))
        if r < 0:
            raise ValueError("step_neuron_ms failed")
        return r

    def step_neuron(self, gid, w0=0.0, w1=0.0, x_next=0.0):
        r = self._L.bo_step_neuron(self._h, int(gid), float(w0), float(w1), float(x_next))
        if r == -2:
            raise FloatingPointError(f"Numerical instability in {self.model} dynamics.")
        return r

    @property
    def step(self):
        return self._L.bo_step_count(self._h)

    @property
    def rk_substeps(self):
        return self._L.bo_rk_substeps(self._h)


def lif_bptt(cfg, row_ptr, col, w, w_in, inputs, targets, grad=True):
    """Surrogate-gradient BPTT restatement (bspk_oracle_bptt.c): returns
    (loss, dw, dw_in, n_spikes); dw/dw_in are None when grad is False.
    cfg: dt, n, n_in, batch, n_steps, n_readout, readout_tau, slope, relaxed,
    detach_reset, params (9 iaf_psc_exp parameters)."""
    c = BpttCfg(cfg["dt"], cfg["n"], cfg["n_in"], cfg["batch"], cfg["n_steps"],
                cfg["n_readout"], cfg["readout_tau"], cfg["slope"], int(cfg.get("relaxed", 0)),
                int(cfg.get("detach_reset", 0)), (C.c_double * 9)(*cfg["params"]))
    row_ptr = np.ascontiguousarray(row_ptr, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    w = np.ascontiguousarray(w, np.float64)
    w_in = np.ascontiguousarray(w_in, np.float64)
    inputs = np.ascontiguousarray(inputs, np.uint8)
    targets = np.ascontiguousarray(targets, np.float64)
    loss = np.zeros(1, np.float64)
    nsp = np.zeros(1, np.int64)
    dw = np.zeros(max(col.size, 1), np.float64) if grad else None
    dwi = np.zeros(max(w_in.size, 1), np.float64) if grad else None
    rc = lib().bo_lif_bptt(C.byref(c), _p(row_ptr), _p(col), int(col.size), _p(w), _p(w_in),
                           _p(inputs), _p(targets), _p(loss), _p(dw) if grad else None,
                           _p(dwi) if grad else None, _p(nsp))
    if rc != 0:
        raise ValueError("lif_bptt failed")
    if grad:
        return float(loss[0]), dw[:col.size], dwi[:w_in.size].reshape(w_in.shape), int(nsp[0])
    return float(loss[0]), None, None, int(nsp[0])


def triplet_update(w, pre_s, post_s, r, o, Aplus, Aplus_triplet, Aminus, Aminus_triplet, Wmax):
    """The oracle's triplet rule on one edge; r = (r1, r2), o = (o1, o2) are the
    substrate-fed traces that include this step's own spike."""
    return lib().bo_triplet_update(float(w), float(pre_s), float(post_s), float(r[0]),
                                    float(r[1]), float(o[0]), float(o[1]), float(Aplus),
                                    float(Aplus_triplet), float(Aminus), float(Aminus_triplet),
                                    float(Wmax))
