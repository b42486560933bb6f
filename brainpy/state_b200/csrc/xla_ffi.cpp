// xla_ffi.cpp -- XLA GPU custom-call targets (the untyped custom-call ABI,
// registered from Python with jax.ffi.register_ffi_target(..., api_version=0)):
//     void target(cudaStream_t stream, void **buffers, const char *opaque, size_t len)
// `opaque` carries the 8-byte address of a library handle (plan, batch or
// adjoint) created beforehand through the C ABI, plus per-call integers.
// The reference has no FFI (its operators are brainevent/JAX primitives);
// these targets let the same kernels sit inside a jitted JAX program.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../../include/bspk.h"

namespace {

template <typename T>
bool read_opaque(const char *opaque, size_t len, size_t at, T *out) {
    if (!opaque || len < at + sizeof(T)) return false;
    std::memcpy(out, opaque + at, sizeof(T));
    return true;
}

}  // namespace

extern "C" {

// buffers: [w, w_in, inputs, targets] -> [loss (f64 scalar)]; opaque: adjoint handle.
void bspk_xla_adjoint_forward(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_adjoint *h = nullptr;
    if (!read_opaque(opaque, len, 0, &h) || !h) return;
    bspk_adjoint_forward(h, buffers[0], buffers[1], static_cast<const uint8_t *>(buffers[2]),
                         buffers[3], static_cast<double *>(buffers[4]), nullptr, stream);
}

// buffers: [w, w_in, inputs, targets] -> [dw, dw_in]; the forward pass is
// recomputed here (XLA does not order this call after a particular forward),
// its loss kept inside the handle.
void bspk_xla_adjoint_backward(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_adjoint *h = nullptr;
    if (!read_opaque(opaque, len, 0, &h) || !h) return;
    if (bspk_adjoint_forward(h, buffers[0], buffers[1], static_cast<const uint8_t *>(buffers[2]),
                             buffers[3], nullptr, nullptr, stream) != BSPK_OK)
        return;
    bspk_adjoint_backward(h, buffers[4], buffers[5], stream);
}

// buffers: [] -> [step counter (i64 scalar, device)]; opaque: plan handle, n_steps (i64).
void bspk_xla_run(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_plan *p = nullptr;
    int64_t n = 0;
    if (!read_opaque(opaque, len, 0, &p) || !p || !read_opaque(opaque, len, 8, &n)) return;
    if (bspk_run(p, n, stream) != BSPK_OK) return;
    const int64_t step = bspk_step_count(p);
    cudaMemcpyAsync(buffers[0], &step, sizeof(step), cudaMemcpyHostToDevice, stream);
    cudaStreamSynchronize(stream);  // `step` lives on this stack frame
}

// buffers: [] -> [step counter]; opaque: batch handle, n_steps.
void bspk_xla_batch_run(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_batch *b = nullptr;
    int64_t n = 0;
    if (!read_opaque(opaque, len, 0, &b) || !b || !read_opaque(opaque, len, 8, &n)) return;
    if (bspk_batch_run(b, n, stream) != BSPK_OK) return;
    const int64_t step = bspk_batch_step_count(b);
    cudaMemcpyAsync(buffers[0], &step, sizeof(step), cudaMemcpyHostToDevice, stream);
    cudaStreamSynchronize(stream);
}

}  // extern "C"
