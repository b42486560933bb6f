"""ctypes binding of libbspk.so (the C ABI of include/bspk.h).

The library is built in-tree (``brainpy/state_b200/libbspk.so``).  There is no
fallback: if the shared object is missing or the GPU is absent, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbspk.so")

BSPK_OK = 0
ERRORS = {
    -1: ValueError, -2: RuntimeError, -3: RuntimeError, -4: NotImplementedError,
    -5: TimeoutError, -6: FloatingPointError, -7: OverflowError, -8: RuntimeError,
}
MODELS = {"iaf_psc_alpha": 0, "iaf_psc_exp": 1, "aeif_cond_alpha": 2, "iaf_cond_exp": 3,
          "iaf_cond_alpha": 4, "iaf_psc_exp_multisynapse": 5}
LEGACY, RING = 0, 1


class Config(C.Structure):
    _fields_ = [("dt", C.c_double), ("precision", C.c_int), ("semantics", C.c_int),
                ("deterministic", C.c_int), ("model", C.c_int), ("device", C.c_int),
                ("spike_capacity", C.c_int64)]


class AdjointConfig(C.Structure):
    _fields_ = [("dt", C.c_double), ("precision", C.c_int), ("n", C.c_int), ("n_in", C.c_int),
                ("batch", C.c_int), ("n_steps", C.c_int), ("ckpt_every", C.c_int),
                ("n_readout", C.c_int), ("readout_tau", C.c_double), ("slope", C.c_double),
                ("relaxed", C.c_int), ("detach_reset", C.c_int), ("device", C.c_int),
                ("params", C.c_double * 9)]


class StdpParams(C.Structure):
    _fields_ = [("tau_plus", C.c_double), ("tau_minus", C.c_double), ("lambda_", C.c_double),
                ("alpha", C.c_double), ("mu_plus", C.c_double), ("mu_minus", C.c_double),
                ("Wmax", C.c_double)]


class StdpTripletParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("tau_plus", "tau_plus_triplet", "tau_minus",
                                          "tau_minus_triplet", "Aplus", "Aplus_triplet",
                                          "Aminus", "Aminus_triplet", "Wmax")]


_lib = None


def lib():
    """Load libbspk.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libbspk.so not built ({LIB_PATH}); run "
                              "python -m brainpy.state_b200.csrc.build")
        L = C.CDLL(LIB_PATH)
        vp, i64, i32, dbl, u32 = C.c_void_p, C.c_int64, C.c_int32, C.c_double, C.c_uint32
        sig = {
            "bspk_version": (C.c_char_p, []),
            "bspk_last_error": (C.c_char_p, []),
            "bspk_plan_create": (C.c_int, [C.POINTER(Config), C.POINTER(vp)]),
            "bspk_plan_destroy": (C.c_int, [vp]),
            "bspk_pop_add": (C.c_int, [vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int)]),
            "bspk_proj_add_csr": (C.c_int, [vp, C.c_int, C.c_int, i64, vp, vp, vp, vp, C.c_int,
                                            C.POINTER(C.c_int)]),
            "bspk_proj_add_fixed_indegree": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, i64, C.c_int,
                                                       C.c_int, dbl, vp, C.c_int, C.c_int,
                                                       C.POINTER(C.c_int)]),
            "bspk_drive_add_poisson": (C.c_int, [vp, C.c_int, dbl, dbl, C.c_int, u32, i64, i64,
                                                 C.c_int, C.POINTER(C.c_int)]),
            "bspk_proj_add_fixed_indegree_w": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, i64,
                                                         C.c_int, C.c_int, dbl, vp, vp, C.c_int,
                                                         C.c_int, C.POINTER(C.c_int)]),
            "bspk_drive_add_poisson_keyed": (C.c_int, [vp, C.c_int, dbl, dbl, C.c_int, vp, i64,
                                                       i64, i64, C.c_int, C.POINTER(C.c_int)]),
            "bspk_jax_fold_in": (C.c_int, [vp, u32, vp]),
            "bspk_jax_uniform": (C.c_int, [vp, i64, C.c_int, dbl, dbl, vp]),
            "bspk_jax_normal": (C.c_int, [vp, i64, C.c_int, vp]),
            "bspk_kernel_poisson_table": (C.c_int, [dbl, dbl, C.c_int, vp, C.POINTER(C.c_int)]),
            "bspk_stdp_attach": (C.c_int, [vp, C.c_int, C.POINTER(StdpParams)]),
            "bspk_stdp_triplet_attach": (C.c_int, [vp, C.c_int, C.POINTER(StdpTripletParams)]),
            "bspk_proj_csr_get": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bspk_record_v": (C.c_int, [vp, C.c_int, vp]),
            "bspk_debug_withhold_record": (C.c_int, [vp, C.c_int, C.c_int]),
            "bspk_plan_set_ports": (C.c_int, [vp, C.c_int]),
            "bspk_proj_set_weights": (C.c_int, [vp, C.c_int, C.c_int64, vp]),
            "bspk_kernel_fixed_indegree": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                                     vp, vp, vp, vp, vp, C.c_int64, C.c_int, vp]),
            "bspk_record_spikes_of": (C.c_int, [vp, C.c_int, vp]),
            "bspk_plan_upload": (C.c_int, [vp, vp]),
            "bspk_run": (C.c_int, [vp, i64, vp]),
            "bspk_spikes_get": (C.c_int, [vp, i64, vp, vp, C.POINTER(i64)]),
            "bspk_v_get": (C.c_int, [vp, vp]),
            "bspk_v_get_f32": (C.c_int, [vp, vp]),
            "bspk_weights_get": (C.c_int, [vp, C.c_int, vp]),
            "bspk_state_get": (C.c_int, [vp, C.c_int, C.c_char_p, vp]),
            "bspk_state_set": (C.c_int, [vp, C.c_int, C.c_char_p, vp]),
            "bspk_step_count": (i64, [vp]),
            "bspk_plan_engine": (C.c_char_p, [vp]),
            "bspk_plan_set_trial": (C.c_int, [vp, C.c_uint32]),
            "bspk_plan_set_windowed": (C.c_int, [vp, C.c_int]),
            "bspk_plan_tune_tiled": (C.c_int, [vp, i64, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                               C.POINTER(dbl)]),
            "bspk_record_weights": (C.c_int, [vp, C.c_int, C.c_int]),
            "bspk_weight_trace_get": (C.c_int, [vp, C.c_int, C.POINTER(i64), vp]),
            "bspk_plan_ring_fraction_bits": (C.c_int, [vp, C.POINTER(C.c_int)]),
            "bspk_last_kernel_time": (C.c_int, [vp, C.POINTER(dbl), C.POINTER(i64)]),
            "bspk_rk_substeps": (C.c_int, [vp, C.POINTER(i64)]),
            "bspk_checkpoint_size": (C.c_int, [vp, C.POINTER(i64)]),
            "bspk_checkpoint_save": (C.c_int, [vp, vp, i64]),
            "bspk_checkpoint_restore": (C.c_int, [vp, vp, i64]),
            "bspk_host_alloc": (C.c_int, [i64, C.POINTER(vp)]),
            "bspk_host_free": (C.c_int, [vp]),
            "bspk_gen_fixed_indegree": (C.c_int, [C.c_int, i64, C.c_int, C.c_int, C.c_int,
                                                  C.c_int, C.c_int, C.c_int, vp, vp]),
            "bspk_batch_create": (C.c_int, [C.POINTER(Config), C.POINTER(vp)]),
            "bspk_batch_destroy": (C.c_int, [vp]),
            "bspk_batch_instance_add": (C.c_int, [vp, C.POINTER(C.c_int)]),
            "bspk_batch_pop_add": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_int,
                                             C.POINTER(C.c_int)]),
            "bspk_batch_fixed_indegree_add": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                                        i64, C.c_int, C.c_int, dbl, C.c_int]),
            "bspk_batch_drive_add_poisson": (C.c_int, [vp, C.c_int, C.c_int, dbl, dbl, C.c_int,
                                                       u32, i64, i64]),
            "bspk_batch_record_spikes": (C.c_int, [vp, C.c_int, C.c_int]),
            "bspk_batch_upload": (C.c_int, [vp, C.c_int, C.c_int, vp]),
            "bspk_batch_tune": (C.c_int, [vp, i64, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(dbl)]),
            "bspk_batch_shape": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_int), C.POINTER(i64)]),
            "bspk_batch_run": (C.c_int, [vp, i64, vp]),
            "bspk_batch_state_set": (C.c_int, [vp, C.c_int, C.c_int, C.c_char_p, vp]),
            "bspk_batch_state_get": (C.c_int, [vp, C.c_int, C.c_int, C.c_char_p, vp]),
            "bspk_batch_spike_counts": (C.c_int, [vp, C.c_int, vp]),
            "bspk_batch_spikes_get": (C.c_int, [vp, C.c_int, i64, vp, vp, C.POINTER(i64)]),
            "bspk_batch_edges_get": (C.c_int, [vp, C.c_int, i64, vp, vp, vp, C.POINTER(i64)]),
            "bspk_batch_step_count": (i64, [vp]),
            "bspk_batch_last_kernel_time": (C.c_int, [vp, C.POINTER(dbl), C.POINTER(i64)]),
            "bspk_adjoint_create": (C.c_int, [C.POINTER(AdjointConfig), vp, vp, i64,
                                              C.POINTER(vp)]),
            "bspk_adjoint_destroy": (C.c_int, [vp]),
            "bspk_adjoint_ctas_per_trial": (C.c_int, [vp]),
            "bspk_adjoint_set_contraction": (C.c_int, [vp, C.c_int]),
            "bspk_adjoint_contraction": (C.c_int, [vp]),
            "bspk_adjoint_status": (C.c_int, [vp]),
            "bspk_adjoint_forward": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp]),
            "bspk_adjoint_backward": (C.c_int, [vp, vp, vp, vp]),
            "bspk_xla_adjoint_forward": (None, [vp, vp, C.c_char_p, C.c_size_t]),
            "bspk_xla_adjoint_backward": (None, [vp, vp, C.c_char_p, C.c_size_t]),
            "bspk_xla_run": (None, [vp, vp, C.c_char_p, C.c_size_t]),
            "bspk_xla_step": (None, [vp, vp, C.c_char_p, C.c_size_t]),
            "bspk_step_fused": (C.c_int, [vp, vp]),
            "bspk_plan_set_tiled_options": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                                      C.c_int]),
            "bspk_plan_get_tiled_options": (C.c_int, [vp] + [C.POINTER(C.c_int)] * 5),
            "bspk_adjoint_sizes": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64),
                                             C.POINTER(C.c_int)]),
            "bspk_xla_batch_run": (None, [vp, vp, C.c_char_p, C.c_size_t]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def kernel_fixed_indegree(seed, proj_id, parts, n_pre, self_pos, K):
    """Source positions (n_post, K) in the pre view of the kernel front end's
    fixed_indegree with multapses; parts = [((hi, lo) population name id, local
    ids), ...] of the post view in order, self_pos = each post neuron's
    position in the pre view (-1 none) or None."""
    parts = list(parts)
    hi = np.array([p[0][0] for p in parts], np.uint32)
    lo = np.array([p[0][1] for p in parts], np.uint32)
    ln = np.array([len(p[1]) for p in parts], np.int64)
    loc = (np.ascontiguousarray(np.concatenate([np.asarray(p[1], np.int64) for p in parts]))
           if parts else np.zeros(0, np.int64))
    n_post = int(ln.sum())
    out = np.zeros(max(n_post * int(K), 1), np.int32)
    sp = None if self_pos is None else np.ascontiguousarray(self_pos, np.int64)
    check(lib().bspk_kernel_fixed_indegree(int(seed) & 0xFFFFFFFF, int(proj_id[0]), int(proj_id[1]),
                                          len(parts), ptr(hi), ptr(lo), ptr(ln), ptr(loc),
                                          ptr(sp) if sp is not None else None, int(n_pre), int(K),
                                          ptr(out)))
    return out[:n_post * int(K)].reshape(n_post, int(K)).astype(np.int64)


def _key(key):
    k = np.ascontiguousarray(np.asarray(key, dtype=np.uint32).reshape(2))
    return k


def jax_fold_in(key, data):
    """jax.random.fold_in(key, data) of a raw uint32[2] key."""
    out = np.zeros(2, np.uint32)
    check(lib().bspk_jax_fold_in(ptr(_key(key)), int(data) & 0xFFFFFFFF, ptr(out)))
    return out


def jax_uniform(key, n, bits=32, lo=0.0, hi=1.0):
    """jax.random.uniform(key, (n,), float32 / float64, lo, hi), widened to
    float64 (the float32 values are exact in it)."""
    out = np.zeros(int(n), np.float64)
    check(lib().bspk_jax_uniform(ptr(_key(key)), int(n), int(bits), float(lo), float(hi),
                                 ptr(out)))
    return out


def jax_normal(key, n, bits=32):
    """jax.random.normal(key, (n,), float32 / float64), widened to float64."""
    out = np.zeros(int(n), np.float64)
    check(lib().bspk_jax_normal(ptr(_key(key)), int(n), int(bits), ptr(out)))
    return out


def kernel_poisson_table(rate_hz, dt_ms):
    """Integer thresholds of the kernel path's float32 Poisson CDF inversion."""
    n = C.c_int()
    check(lib().bspk_kernel_poisson_table(float(rate_hz), float(dt_ms), 0, None, C.byref(n)))
    out = np.zeros(n.value, np.uint64)
    check(lib().bspk_kernel_poisson_table(float(rate_hz), float(dt_ms), n.value, ptr(out),
                                          C.byref(n)))
    return out


class _Pinned:
    """Owner of a page-locked host allocation (freed with the object)."""

    def __init__(self, nbytes):
        self.ptr = C.c_void_p()
        check(lib().bspk_host_alloc(int(nbytes), C.byref(self.ptr)))
        self.nbytes = int(nbytes)
        # held by the object: module globals may already be gone when the
        # last reference dies at interpreter exit
        self._free = lib().bspk_host_free

    def __del__(self):
        if getattr(self, "ptr", None) and self.ptr.value and getattr(self, "_free", None):
            self._free(self.ptr)
            self.ptr = None


def pinned_bytes(nbytes):
    """A uint8 numpy array over page-locked host memory; the allocation is
    freed when the array (and every view of it) is gone."""
    if nbytes == 0:
        return np.zeros(0, np.uint8)
    owner = _Pinned(nbytes)
    buf = (C.c_uint8 * int(nbytes)).from_address(owner.ptr.value)
    buf._owner = owner  # the ctypes array keeps the allocation alive
    return np.frombuffer(buf, dtype=np.uint8)


def check(rc):
    if rc != BSPK_OK:
        msg = lib().bspk_last_error().decode()
        raise ERRORS.get(rc, RuntimeError)(msg or f"libbspk error {rc}")
    return rc


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Plan:
    """Thin owner of one ``bspk_plan`` handle (one neuron model per plan)."""

    def __init__(self, dt, model="iaf_psc_alpha", precision=32, semantics=LEGACY,
                 deterministic=False, device=0, spike_capacity=1 << 22):
        self._L = lib()
        cfg = Config(float(dt), int(precision), int(semantics), int(bool(deterministic)),
                     MODELS[model], int(device), int(spike_capacity))
        h = C.c_void_p()
        check(self._L.bspk_plan_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.model = model
        self.precision = precision
        self.dt = float(dt)
        self.pop_sizes = []
        self.n_rec_v = 0
        self._proj_edges = []
        self._proj_pre_n = []

    def close(self):
        if getattr(self, "_h", None):
            self._L.bspk_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # -- building
    def add_pop(self, n, params):
        p = np.ascontiguousarray(params, np.float64)
        out = C.c_int()
        check(self._L.bspk_pop_add(self._h, int(n), ptr(p), int(p.size), C.byref(out)))
        self.pop_sizes.append(int(n))
        return out.value

    def add_csr(self, pre, post, indptr, post_local, w, delay_steps, receptor=0):
        indptr = np.ascontiguousarray(indptr, np.int64)
        post_local = np.ascontiguousarray(post_local, np.int32)
        w = np.ascontiguousarray(w, np.float64)
        d = np.ascontiguousarray(delay_steps, np.int32)
        out = C.c_int()
        check(self._L.bspk_proj_add_csr(self._h, pre, post, int(post_local.size), ptr(indptr),
                                        ptr(post_local), ptr(w), ptr(d), int(receptor),
                                        C.byref(out)))
        self._proj_edges.append(int(post_local.size))
        self._proj_pre_n.append(self.pop_sizes[pre])
        return out.value

    def add_fixed_indegree(self, pre, post, K, seed, weight, delay_steps=None, delay_const=0,
                           allow_autapses=True, nbits=32, receptor=0, w_draw=None):
        """``delay_steps`` and ``w_draw`` (per-edge weights) are in the
        sampler's edge order (post-major, before the CSR sort)."""
        d = None if delay_steps is None else np.ascontiguousarray(delay_steps, np.int32)
        wd = None if w_draw is None else np.ascontiguousarray(w_draw, np.float64)
        out = C.c_int()
        check(self._L.bspk_proj_add_fixed_indegree_w(self._h, pre, post, int(K), int(seed),
                                                     int(bool(allow_autapses)), int(nbits),
                                                     float(weight), ptr(wd), ptr(d),
                                                     int(delay_const), int(receptor),
                                                     C.byref(out)))
        self._proj_edges.append(int(K) * self.pop_sizes[post])
        self._proj_pre_n.append(self.pop_sizes[pre])
        return out.value

    def add_poisson(self, post, rate_hz, weight, delay_steps, seed, t_min=0, t_max=2 ** 62,
                    receptor=0):
        out = C.c_int()
        check(self._L.bspk_drive_add_poisson(self._h, post, float(rate_hz), float(weight),
                                             int(delay_steps), int(seed) & 0xFFFFFFFF,
                                             int(t_min), int(t_max), int(receptor),
                                             C.byref(out)))
        return out.value

    def add_poisson_keyed(self, post, rate_hz, weight, delay_steps, obj_key, unit_off=0,
                          t_min=0, t_max=2 ** 62, receptor=0):
        """Poisson drive on the reference kernel path's block-key stream of
        the device population with object key ``obj_key`` (uint32[2]); unit
        ``unit_off + i`` drives neuron i of ``post``."""
        out = C.c_int()
        check(self._L.bspk_drive_add_poisson_keyed(
            self._h, int(post), float(rate_hz), float(weight), int(delay_steps),
            ptr(_key(obj_key)), int(unit_off), int(t_min), int(t_max), int(receptor),
            C.byref(out)))
        return out.value

    def csr(self, proj):
        """(indptr, post_local, delay_steps, w) of a projection (host copy)."""
        E = self._proj_edges[proj]
        pre_n = self._proj_pre_n[proj]
        indptr = np.zeros(pre_n + 1, np.int64)
        post = np.zeros(E, np.int32)
        d = np.zeros(E, np.int32)
        w = np.zeros(E, np.float64)
        check(self._L.bspk_proj_csr_get(self._h, int(proj), ptr(indptr), ptr(post), ptr(d),
                                        ptr(w)))
        return indptr, post, d, w

    def attach_stdp(self, proj, tau_plus=20.0, tau_minus=20.0, lambda_=0.01, alpha=1.0,
                    mu_plus=1.0, mu_minus=1.0, Wmax=100.0):
        sp = StdpParams(tau_plus, tau_minus, lambda_, alpha, mu_plus, mu_minus, Wmax)
        check(self._L.bspk_stdp_attach(self._h, proj, C.byref(sp)))

    def attach_stdp_triplet(self, proj, tau_plus=16.8, tau_plus_triplet=101.0, tau_minus=20.0,
                            tau_minus_triplet=110.0, Aplus=5e-10, Aplus_triplet=0.0062,
                            Aminus=0.007, Aminus_triplet=0.00023, Wmax=100.0):
        tp = StdpTripletParams(tau_plus, tau_plus_triplet, tau_minus, tau_minus_triplet, Aplus,
                               Aplus_triplet, Aminus, Aminus_triplet, Wmax)
        check(self._L.bspk_stdp_triplet_attach(self._h, proj, C.byref(tp)))

    def set_weights(self, proj, w):
        """Per-edge weights of projection `proj` in its CSR order (before upload)."""
        w = np.ascontiguousarray(w, np.float64)
        check(self._L.bspk_proj_set_weights(self._h, int(proj), int(w.size), ptr(w)))

    def set_ports(self, separate):
        """iaf models: keep receptor ports 0 ('ex') and 1 ('in_') apart, signs
        kept (before any input is added)."""
        check(self._L.bspk_plan_set_ports(self._h, int(bool(separate))))

    def debug_withhold_record(self, cta, window):
        """Test hook: in the next run, tiled-kernel CTA `cta` withholds its
        record of `window`, so the run's next synchronising call (spikes(),
        v_trace(), ...) raises TimeoutError after about 2 s."""
        check(self._L.bspk_debug_withhold_record(self._h, int(cta), int(window)))

    def record_v(self, gids):
        g = np.ascontiguousarray(gids, np.int32)
        check(self._L.bspk_record_v(self._h, int(g.size), ptr(g)))
        self.n_rec_v = int(g.size)

    def record_spikes_of(self, gids):
        g = np.ascontiguousarray(gids, np.int32)
        check(self._L.bspk_record_spikes_of(self._h, int(g.size), ptr(g)))

    def upload(self, stream=None):
        check(self._L.bspk_plan_upload(self._h, stream))

    # -- running
    def run(self, n_steps, stream=None):
        check(self._L.bspk_run(self._h, int(n_steps), stream))
        self._last_steps = int(n_steps)

    def spikes(self, cap=None, sort=True):
        """(steps, gids) of the last run's recorded spikes, sorted by step then
        gid (``sort=False``: in the device's record order)."""
        n = C.c_int64()
        if cap is None:  # ask for the count first, then copy exactly that many
            check(self._L.bspk_spikes_get(self._h, 0, None, None, C.byref(n)))
            cap = n.value
        cap = max(int(cap), 1)
        st = np.empty(cap, np.int64)
        g = np.empty(cap, np.int32)
        check(self._L.bspk_spikes_get(self._h, cap, ptr(st), ptr(g), C.byref(n)))
        m = min(n.value, cap)
        if not sort:
            return st[:m], g[:m]
        order = np.lexsort((g[:m], st[:m]))
        return st[:m][order], g[:m][order]

    def v_trace(self, dtype=np.float64):
        """(steps, n_rec) V_m of the last run, float64 or float32."""
        if np.dtype(dtype) == np.float32:
            out = np.empty((self._last_steps, self.n_rec_v), np.float32)
            check(self._L.bspk_v_get_f32(self._h, ptr(out)))
        else:
            out = np.empty((self._last_steps, self.n_rec_v), np.float64)
            check(self._L.bspk_v_get(self._h, ptr(out)))
        return out

    def record_weights(self, proj, on=True):
        check(self._L.bspk_record_weights(self._h, int(proj), int(bool(on))))

    def weight_trace(self, proj):
        """(n_steps, n_edges) FP64 weights after every step of the last run."""
        n = C.c_int64()
        check(self._L.bspk_weight_trace_get(self._h, int(proj), C.byref(n), None))
        out = np.empty((n.value, self._proj_edges[proj]), np.float64)
        check(self._L.bspk_weight_trace_get(self._h, int(proj), C.byref(n), ptr(out)))
        return out

    def weights(self, proj):
        out = np.zeros(self._proj_edges[proj], np.float64)
        check(self._L.bspk_weights_get(self._h, int(proj), ptr(out)))
        return out

    def get_state(self, pop, name):
        out = np.zeros(self.pop_sizes[pop], np.float64)
        check(self._L.bspk_state_get(self._h, int(pop), name.encode(), ptr(out)))
        return out

    def set_state(self, pop, name, values):
        v = np.ascontiguousarray(np.broadcast_to(values, (self.pop_sizes[pop],)), np.float64)
        check(self._L.bspk_state_set(self._h, int(pop), name.encode(), ptr(v)))

    @property
    def step(self):
        return self._L.bspk_step_count(self._h)

    @property
    def engine(self):
        """Kernel family of the uploaded plan: 'tiled', 'global_ring', 'exact',
        'per_step' or 'windowed'."""
        return self._L.bspk_plan_engine(self._h).decode()

    def set_trial(self, trial):
        """Trial index folded into every keyed drive's step keys (the kernel
        path's batched trials); before upload."""
        check(self._L.bspk_plan_set_trial(self._h, int(trial)))

    def set_windowed(self, on):
        """Run a plan that can run windowed in the windowed (True) or the
        per-step (False) form."""
        check(self._L.bspk_plan_set_windowed(self._h, int(bool(on))))

    def kernel_time(self):
        ms, n = C.c_double(), C.c_int64()
        check(self._L.bspk_last_kernel_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def set_tiled_options(self, record_copies=1, poll_pause_ns=400, drive_overlap=True,
                          drive_chunk_steps=0, record_stride_bytes=64):
        """Options of the tiled path (results do not depend on them)."""
        check(self._L.bspk_plan_set_tiled_options(self._h, int(record_copies), int(poll_pause_ns),
                                                  int(bool(drive_overlap)),
                                                  int(drive_chunk_steps), int(record_stride_bytes)))

    def tune_tiled(self, pilot_steps=500):
        """Time pilot runs over CTA counts and poll pauses and keep the best
        (the state is restored after every pilot); returns (grid,
        poll_pause_ns, pilot_ms)."""
        g, pz, ms = C.c_int(), C.c_int(), C.c_double()
        check(self._L.bspk_plan_tune_tiled(self._h, int(pilot_steps), C.byref(g), C.byref(pz),
                                           C.byref(ms)))
        return g.value, pz.value, ms.value

    def tiled_options(self):
        v = [C.c_int() for _ in range(5)]
        check(self._L.bspk_plan_get_tiled_options(self._h, *[C.byref(x) for x in v]))
        return dict(record_copies=v[0].value, poll_pause_ns=v[1].value,
                    drive_overlap=bool(v[2].value), drive_chunk_steps=v[3].value,
                    record_stride_bytes=v[4].value)

    @property
    def ring_fraction_bits(self):
        """k of the tiled kernel's fixed-point ring (weights rint(w * 2^k))."""
        k = C.c_int()
        check(self._L.bspk_plan_ring_fraction_bits(self._h, C.byref(k)))
        return k.value

    def rk_substeps(self):
        """RKF45 substeps, accepted and rejected, of every conductance-model
        neuron since upload."""
        n = C.c_int64()
        check(self._L.bspk_rk_substeps(self._h, C.byref(n)))
        return n.value

    def checkpoint(self, pinned=False):
        """Host copy of every evolving device buffer; ``pinned`` puts it in
        page-locked memory (a restore from it needs no staging copy)."""
        n = C.c_int64()
        check(self._L.bspk_checkpoint_size(self._h, C.byref(n)))
        buf = pinned_bytes(n.value) if pinned else np.zeros(n.value, np.uint8)
        check(self._L.bspk_checkpoint_save(self._h, ptr(buf), n.value))
        return buf

    def restore(self, buf):
        buf = np.ascontiguousarray(buf, np.uint8)
        check(self._L.bspk_checkpoint_restore(self._h, ptr(buf), int(buf.size)))


def gen_fixed_indegree(seed, n_pre, n_post, K, pre_is_post=False, allow_autapses=True, nbits=32,
                       device=0):
    """fixed_indegree CSR drawn on the GPU: (indptr int64[n_pre+1], post int32[E])."""
    L = lib()
    indptr = np.zeros(int(n_pre) + 1, np.int64)
    post = np.zeros(max(int(n_post) * int(K), 1), np.int32)
    check(L.bspk_gen_fixed_indegree(int(device), int(seed), int(n_pre), int(n_post), int(K),
                                    int(bool(pre_is_post)), int(bool(allow_autapses)),
                                    int(nbits), ptr(indptr), ptr(post)))
    return indptr, post[:int(n_post) * int(K)]


class Batch:
    """Owner of one ``bspk_batch``: independent iaf networks of uneven sizes
    advanced by one persistent launch (instances, populations, fixed_indegree
    projections with one delay per instance, Poisson drives)."""

    def __init__(self, dt, model="iaf_psc_alpha", precision=32, semantics=LEGACY, device=0,
                 spike_capacity=1 << 22):
        self._L = lib()
        cfg = Config(float(dt), int(precision), int(semantics), 0, MODELS[model], int(device),
                     int(spike_capacity))
        h = C.c_void_p()
        check(self._L.bspk_batch_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.dt = float(dt)
        self.precision = precision
        self.sizes = []      # neurons per instance
        self.pop_sizes = []  # per instance: list of population sizes

    def close(self):
        if getattr(self, "_h", None):
            self._L.bspk_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def add_instance(self):
        i = C.c_int()
        check(self._L.bspk_batch_instance_add(self._h, C.byref(i)))
        self.sizes.append(0)
        self.pop_sizes.append([])
        return i.value

    def add_pop(self, inst, n, params):
        p = np.ascontiguousarray(params, np.float64)
        out = C.c_int()
        check(self._L.bspk_batch_pop_add(self._h, int(inst), int(n), ptr(p), p.size,
                                         C.byref(out)))
        self.sizes[inst] += int(n)
        self.pop_sizes[inst].append(int(n))
        return out.value

    def add_fixed_indegree(self, inst, pre, post, K, seed, weight, delay_steps,
                           allow_autapses=True, nbits=32):
        check(self._L.bspk_batch_fixed_indegree_add(self._h, int(inst), int(pre), int(post),
                                                    int(K), int(seed), int(bool(allow_autapses)),
                                                    int(nbits), float(weight), int(delay_steps)))

    def add_poisson(self, inst, post, rate_hz, weight, delay_steps, seed, t_min=0,
                    t_max=(1 << 62)):
        check(self._L.bspk_batch_drive_add_poisson(self._h, int(inst), int(post), float(rate_hz),
                                                   float(weight), int(delay_steps),
                                                   int(seed) & 0xFFFFFFFF, int(t_min), int(t_max)))

    def record_spikes(self, inst, on=True):
        check(self._L.bspk_batch_record_spikes(self._h, int(inst), int(bool(on))))

    def upload(self, tile=0, ctas_per_sm=0):
        check(self._L.bspk_batch_upload(self._h, int(tile), int(ctas_per_sm), None))

    def tune(self, pilot_steps=300):
        t, c, ms = C.c_int(), C.c_int(), C.c_double()
        check(self._L.bspk_batch_tune(self._h, int(pilot_steps), C.byref(t), C.byref(c),
                                      C.byref(ms)))
        return t.value, c.value, ms.value

    def shape(self):
        t, c, g, n = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        check(self._L.bspk_batch_shape(self._h, C.byref(t), C.byref(c), C.byref(g), C.byref(n)))
        return {"tile": t.value, "ctas_per_sm": c.value, "grid": g.value, "tiles": n.value}

    def run(self, n_steps, stream=None):
        check(self._L.bspk_batch_run(self._h, int(n_steps), stream))

    def set_state(self, inst, pop, name, values):
        v = np.ascontiguousarray(values, np.float64)
        check(self._L.bspk_batch_state_set(self._h, int(inst), int(pop), name.encode(), ptr(v)))

    def get_state(self, inst, pop, name):
        v = np.zeros(self.pop_sizes[inst][pop], np.float64)
        check(self._L.bspk_batch_state_get(self._h, int(inst), int(pop), name.encode(), ptr(v)))
        return v

    def spike_counts(self, inst):
        c = np.zeros(self.sizes[inst], np.int64)
        check(self._L.bspk_batch_spike_counts(self._h, int(inst), ptr(c)))
        return c

    def spikes(self, inst):
        n = C.c_int64()
        check(self._L.bspk_batch_spikes_get(self._h, int(inst), 0, None, None, C.byref(n)))
        st = np.zeros(max(n.value, 1), np.int64)
        ids = np.zeros(max(n.value, 1), np.int32)
        check(self._L.bspk_batch_spikes_get(self._h, int(inst), n.value, ptr(st), ptr(ids),
                                            C.byref(n)))
        return st[:n.value], ids[:n.value]

    def edges(self, inst):
        n = C.c_int64()
        check(self._L.bspk_batch_edges_get(self._h, int(inst), 0, None, None, None, C.byref(n)))
        pre = np.zeros(max(n.value, 1), np.int32)
        post = np.zeros_like(pre)
        proj = np.zeros_like(pre)
        check(self._L.bspk_batch_edges_get(self._h, int(inst), n.value, ptr(pre), ptr(post),
                                           ptr(proj), C.byref(n)))
        return pre[:n.value], post[:n.value], proj[:n.value]

    @property
    def step(self):
        return int(self._L.bspk_batch_step_count(self._h))

    def kernel_time(self):
        ms, n = C.c_double(), C.c_int64()
        check(self._L.bspk_batch_last_kernel_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value
