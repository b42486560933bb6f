/*
 * bspk_xla.h -- XLA GPU custom-call targets exported by libbspk.so.
 *
 * Untyped custom-call ABI (register with jax.ffi.register_ffi_target(name,
 * jax.ffi.pycapsule(fn), platform="CUDA", api_version=0)); `stream` is the
 * cudaStream_t XLA passes.  The reference has no FFI: its hot path is JAX
 * with brainevent primitives (_nest_network/projections.py:56-59,
 * _kernel/delay_scatter.py:243-347); these targets put the library's kernels
 * inside a jitted JAX program instead.  `opaque` holds the 8-byte address of a
 * handle made through bspk.h, followed by the per-target integers below.
 */
#ifndef BSPK_XLA_H
#define BSPK_XLA_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every target ends its outputs with an int32 status (0 = ok, else a BSPK_ERR_*
 * code), written on the call's stream; on failure the other outputs hold NaN
 * (losses, gradients) or -1 (step counters).  No target synchronises. */
/* buffers [w, w_in, inputs, targets | loss, status];  opaque: bspk_adjoint* */
void bspk_xla_adjoint_forward(void *stream, void **buffers, const char *opaque, size_t len);
/* buffers [w, w_in, inputs, targets | dw, dw_in, status];  opaque: bspk_adjoint* (the
 * forward pass is recomputed inside the call) */
void bspk_xla_adjoint_backward(void *stream, void **buffers, const char *opaque, size_t len);
/* buffers [| step, status];  opaque: bspk_plan*, int64 n_steps (Simulator.simulate/cont,
 * _nest_network/simulator.py:1790-1883) */
void bspk_xla_run(void *stream, void **buffers, const char *opaque, size_t len);
/* buffers [| step, status];  opaque: bspk_plan*.  One step (bspk_step_fused): the
 * single-step target for programs whose time loop stays in JAX (the reference's
 * scan body, _kernel/runner.py:571-674) */
void bspk_xla_step(void *stream, void **buffers, const char *opaque, size_t len);
/* buffers [| step, status];  opaque: bspk_batch*, int64 n_steps */
void bspk_xla_batch_run(void *stream, void **buffers, const char *opaque, size_t len);

#ifdef __cplusplus
}
#endif
#endif
