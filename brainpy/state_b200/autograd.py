"""Surrogate-gradient BPTT through the hand-written adjoint kernel.

``LifAdjoint`` owns one ``bspk_adjoint`` handle (structure and sizes fixed at
creation); ``LifBpttLoss`` is the ``torch.autograd.Function`` over it:

    adj = LifAdjoint(cfg, row_ptr, col)              # cfg: lif_task.make_task()["cfg"]
    loss = LifBpttLoss.apply(w, w_in, inputs, targets, adj)
    loss.backward()                                   # w.grad, w_in.grad via the adjoint

The forward pass keeps a checkpoint every ``ckpt_every`` steps; backward
recomputes each segment from its checkpoint and sweeps the adjoint through
it (reference: BPTT._episode/_objective, _kernel/learn/bptt.py:437-491).
Operands live on the GPU; the kernels run on torch's current stream.  There is
no CPU path: without libbspk.so or a GPU these calls raise.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class LifAdjoint:
    def __init__(self, cfg, row_ptr, col, precision=32, ckpt_every=50, device=0):
        self._L = _lib.lib()
        c = _lib.AdjointConfig(float(cfg["dt"]), int(precision), int(cfg["n"]), int(cfg["n_in"]),
                               int(cfg["batch"]), int(cfg["n_steps"]), int(ckpt_every),
                               int(cfg["n_readout"]), float(cfg["readout_tau"]),
                               float(cfg["slope"]), int(cfg.get("relaxed", 0)),
                               int(cfg.get("detach_reset", 0)), int(device),
                               (C.c_double * 9)(*cfg["params"]))
        rp = np.ascontiguousarray(row_ptr, np.int64)
        cl = np.ascontiguousarray(col, np.int32)
        h = C.c_void_p()
        _lib.check(self._L.bspk_adjoint_create(C.byref(c), _lib.ptr(rp), _lib.ptr(cl),
                                               int(cl.size), C.byref(h)))
        self._h = h
        self.cfg = dict(cfg)
        self.precision = precision
        self.nnz = int(cl.size)
        self.forward_id = 0

    @property
    def ctas_per_trial(self):
        """1, or 2 when each trial runs on a two-CTA cluster."""
        return int(self._L.bspk_adjoint_ctas_per_trial(self._h))

    @property
    def contraction(self):
        """True when the weight gradients are dense contractions over (step,
        trial) (FP32 default); False: per-trial read-modify-writes."""
        return bool(self._L.bspk_adjoint_contraction(self._h))

    @contraction.setter
    def contraction(self, on):
        _lib.check(self._L.bspk_adjoint_set_contraction(self._h, int(bool(on))))

    def close(self):
        if getattr(self, "_h", None):
            self._L.bspk_adjoint_destroy(self._h)
            self._h = None

    __del__ = close

    def _check(self, t, dtype, shape, name):
        import torch
        if not t.is_cuda or t.dtype != dtype or tuple(t.shape) != tuple(shape) or not t.is_contiguous():
            raise ValueError(f"{name}: expected a contiguous CUDA {dtype} tensor of shape {shape}")

    def dtype(self):
        import torch
        return torch.float64 if self.precision == 64 else torch.float32

    def forward(self, w, w_in, inputs, targets, loss=None, n_spikes=None):
        """Loss (device float64 scalar tensor) of the episode; keeps checkpoints."""
        import torch
        c, dt = self.cfg, self.dtype()
        self._check(w, dt, (self.nnz,), "w")
        self._check(w_in, dt, (c["n"], c["n_in"]), "w_in")
        self._check(inputs, torch.uint8, (c["n_steps"], c["batch"], c["n_in"]), "inputs")
        self._check(targets, dt, (c["n_steps"], c["batch"], c["n_readout"]), "targets")
        if loss is None:
            loss = torch.zeros((), dtype=torch.float64, device=w.device)
        st = torch.cuda.current_stream(w.device).cuda_stream
        _lib.check(self._L.bspk_adjoint_forward(
            self._h, C.c_void_p(w.data_ptr()), C.c_void_p(w_in.data_ptr()),
            C.c_void_p(inputs.data_ptr()), C.c_void_p(targets.data_ptr()),
            C.c_void_p(loss.data_ptr()),
            C.c_void_p(n_spikes.data_ptr()) if n_spikes is not None else None, C.c_void_p(st)))
        self.forward_id += 1
        self._operands = (w, w_in, inputs, targets)  # keep alive while kernels may read them
        return loss

    def backward(self, dw=None, dw_in=None):
        """dL/dw and dL/dw_in of the last forward on this handle."""
        import torch
        w, w_in = self._operands[0], self._operands[1]
        dw = torch.empty_like(w) if dw is None else dw
        dw_in = torch.empty_like(w_in) if dw_in is None else dw_in
        st = torch.cuda.current_stream(w.device).cuda_stream
        _lib.check(self._L.bspk_adjoint_backward(self._h, C.c_void_p(dw.data_ptr()),
                                                 C.c_void_p(dw_in.data_ptr()), C.c_void_p(st)))
        return dw, dw_in

    def status(self):
        """Synchronise and raise if a bounded device wait of the gradient
        contraction ran out since the last check."""
        _lib.check(self._L.bspk_adjoint_status(self._h))


def _function():
    import torch

    class LifBpttLoss(torch.autograd.Function):
        """loss = LifBpttLoss.apply(w, w_in, inputs, targets, adj)."""

        @staticmethod
        def forward(ctx, w, w_in, inputs, targets, adj):
            loss = adj.forward(w, w_in, inputs, targets)
            ctx.adj = adj
            ctx.fid = adj.forward_id
            ctx.save_for_backward(w, w_in, inputs, targets)
            return loss.to(w.dtype)

        @staticmethod
        def backward(ctx, gloss):
            adj = ctx.adj
            w, w_in, inputs, targets = ctx.saved_tensors
            if adj.forward_id != ctx.fid:  # another forward ran on the handle: redo ours
                adj.forward(w, w_in, inputs, targets)
                ctx.fid = adj.forward_id
            dw, dw_in = adj.backward()
            g = gloss.to(w.dtype)
            return dw * g, dw_in * g, None, None, None

    return LifBpttLoss


class _Lazy:
    _f = None

    def __getattr__(self, k):
        if _Lazy._f is None:
            _Lazy._f = _function()
        return getattr(_Lazy._f, k)


LifBpttLoss = _Lazy()
