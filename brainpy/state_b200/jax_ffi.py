"""JAX bindings of libbspk.so: XLA custom calls over the targets of
``include/bspk_xla.h`` and a ``jax.custom_vjp`` over the hand-written adjoint.

Needs jax with a CUDA backend (``import jax`` fails without it; there is no CPU
path).  The targets use XLA's untyped GPU custom-call ABI
(``void(cudaStream_t, void **buffers, const char *opaque, size_t len)``), so they
register with ``api_version=0`` and take the library handle's address as the
opaque string.
"""
from __future__ import annotations

import struct

import jax
import jax.numpy as jnp

from . import _lib

_TARGETS = ("bspk_xla_adjoint_forward", "bspk_xla_adjoint_backward", "bspk_xla_run",
            "bspk_xla_step", "bspk_xla_batch_run")
_STATUS = jax.ShapeDtypeStruct((), jnp.int32)
_registered = False


def register():
    """Register every XLA target of libbspk.so for the CUDA platform (once)."""
    global _registered
    if _registered:
        return
    L = _lib.lib()
    for name in _TARGETS:
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(L, name)), platform="CUDA",
                                    api_version=0)
    _registered = True


def _opaque(handle, *ints):
    return struct.pack("<Q", handle.value) + b"".join(struct.pack("<q", int(i)) for i in ints)


def _call(name, result, opaque, *args):
    return jax.ffi.ffi_call(name, result, custom_call_api_version=1,
                            legacy_backend_config=opaque.decode("latin-1"),
                            has_side_effect=True)(*args)


def lif_bptt_loss(adj):
    """``loss_fn(w, w_in, inputs, targets)`` with gradients through the adjoint
    kernel of ``adj`` (a ``brainpy.state_b200.autograd.LifAdjoint``)."""
    register()
    op = _opaque(adj._h)
    real = jnp.float64 if adj.precision == 64 else jnp.float32

    @jax.custom_vjp
    def loss_fn(w, w_in, inputs, targets):
        loss, _status = _call("bspk_xla_adjoint_forward",
                              (jax.ShapeDtypeStruct((), jnp.float64), _STATUS), op,
                              w, w_in, inputs, targets)
        return loss.astype(real)   # NaN when the call failed

    def fwd(w, w_in, inputs, targets):
        return loss_fn(w, w_in, inputs, targets), (w, w_in, inputs, targets)

    def bwd(res, g):
        w, w_in, inputs, targets = res
        dw, dwi, _status = _call("bspk_xla_adjoint_backward",
                                 (jax.ShapeDtypeStruct(w.shape, real),
                                  jax.ShapeDtypeStruct(w_in.shape, real), _STATUS),
                                 op, w, w_in, inputs, targets)
        return dw * g, dwi * g, None, None

    loss_fn.defvjp(fwd, bwd)
    return loss_fn


def run(plan, n_steps):
    """Advance a plan inside a jitted program; returns (step counter, status)."""
    register()
    return _call("bspk_xla_run", (jax.ShapeDtypeStruct((), jnp.int64), _STATUS),
                 _opaque(plan._h, n_steps))


def step(plan):
    """One step of a plan (bspk_step_fused); returns (step counter, status)."""
    register()
    return _call("bspk_xla_step", (jax.ShapeDtypeStruct((), jnp.int64), _STATUS),
                 _opaque(plan._h))


def batch_run(batch, n_steps):
    """Advance a batch inside a jitted program; returns (step counter, status)."""
    register()
    return _call("bspk_xla_batch_run", (jax.ShapeDtypeStruct((), jnp.int64), _STATUS),
                 _opaque(batch._h, n_steps))
