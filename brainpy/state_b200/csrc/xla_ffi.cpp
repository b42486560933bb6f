// xla_ffi.cpp -- XLA GPU custom-call targets (the untyped custom-call ABI,
// registered from Python with jax.ffi.register_ffi_target(..., api_version=0)):
//     void target(cudaStream_t stream, void **buffers, const char *opaque, size_t len)
// `opaque` carries the 8-byte address of a library handle (plan, batch or
// adjoint) created beforehand through the C ABI, plus per-call integers.
// The reference has no FFI (its operators are brainevent/JAX primitives);
// these targets let the same kernels sit inside a jitted JAX program.
//
// A custom call has no way to return an error to XLA, so every target ends
// with an int32 status buffer (0 = ok, else a BSPK_ERR_* code) that a small
// kernel writes on the call's stream, and on failure the other outputs are
// filled with NaN (floating point) or -1 (step counters) so that no consumer
// reads uninitialised memory.  Scalars reach the device as kernel arguments
// (copied at launch), so no call copies from host memory or synchronises.
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

__global__ void k_set_i64_i32(int64_t *a, int64_t va, int *b, int vb) {
    if (a) *a = va;
    if (b) *b = vb;
}

// NaN in every element of a float (elt 4) or double (elt 8) buffer
__global__ void k_fill_nan(void *p, int64_t n, int elt) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (elt == 8) static_cast<double *>(p)[i] = __longlong_as_double(0x7FF8000000000000ll);
        else static_cast<float *>(p)[i] = __int_as_float(0x7FC00000);
    }
}

void fill_nan(void *p, int64_t n, int elt, cudaStream_t st) {
    if (!p || n <= 0) return;
    const int64_t blocks = (n + 255) / 256;
    k_fill_nan<<<static_cast<int>(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(p, n, elt);
}

void put(cudaStream_t st, int64_t *i64, int64_t v64, int *status, int rc) {
    k_set_i64_i32<<<1, 1, 0, st>>>(i64, v64, status, rc);
}

}  // namespace

extern "C" {

// buffers: [w, w_in, inputs, targets] -> [loss (f64 scalar), status (i32)];
// opaque: adjoint handle.
void bspk_xla_adjoint_forward(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_adjoint *h = nullptr;
    int rc = BSPK_ERR_ARG;
    if (read_opaque(opaque, len, 0, &h) && h)
        rc = bspk_adjoint_forward(h, buffers[0], buffers[1], static_cast<const uint8_t *>(buffers[2]),
                                  buffers[3], static_cast<double *>(buffers[4]), nullptr, stream);
    if (rc != BSPK_OK) fill_nan(buffers[4], 1, 8, stream);
    put(stream, nullptr, 0, static_cast<int *>(buffers[5]), rc);
}

// buffers: [w, w_in, inputs, targets] -> [dw, dw_in, status]; the forward
// pass is recomputed here (XLA does not order this call after a particular
// forward), its loss kept inside the handle.
void bspk_xla_adjoint_backward(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_adjoint *h = nullptr;
    int rc = BSPK_ERR_ARG;
    if (read_opaque(opaque, len, 0, &h) && h) {
        rc = bspk_adjoint_forward(h, buffers[0], buffers[1], static_cast<const uint8_t *>(buffers[2]),
                                  buffers[3], nullptr, nullptr, stream);
        if (rc == BSPK_OK) rc = bspk_adjoint_backward(h, buffers[4], buffers[5], stream);
        if (rc != BSPK_OK) {
            int64_t nnz = 0, nwin = 0;
            int prec = 32;
            if (bspk_adjoint_sizes(h, &nnz, &nwin, &prec) == BSPK_OK) {
                fill_nan(buffers[4], nnz, prec == 64 ? 8 : 4, stream);
                fill_nan(buffers[5], nwin, prec == 64 ? 8 : 4, stream);
            }
        }
    }
    put(stream, nullptr, 0, static_cast<int *>(buffers[6]), rc);
}

// buffers: [] -> [step counter (i64 scalar), status (i32)]; opaque: plan
// handle, n_steps (i64).
void bspk_xla_run(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_plan *p = nullptr;
    int64_t n = 0;
    int rc = BSPK_ERR_ARG;
    if (read_opaque(opaque, len, 0, &p) && p && read_opaque(opaque, len, 8, &n))
        rc = bspk_run(p, n, stream);
    put(stream, static_cast<int64_t *>(buffers[0]), rc == BSPK_OK ? bspk_step_count(p) : -1,
        static_cast<int *>(buffers[1]), rc);
}

// buffers: [] -> [step counter, status]; opaque: plan handle.  One step
// (bspk_step_fused), for programs that keep the time loop in JAX.
void bspk_xla_step(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_plan *p = nullptr;
    int rc = BSPK_ERR_ARG;
    if (read_opaque(opaque, len, 0, &p) && p) rc = bspk_step_fused(p, stream);
    put(stream, static_cast<int64_t *>(buffers[0]), rc == BSPK_OK ? bspk_step_count(p) : -1,
        static_cast<int *>(buffers[1]), rc);
}

// buffers: [] -> [step counter, status]; opaque: batch handle, n_steps.
void bspk_xla_batch_run(cudaStream_t stream, void **buffers, const char *opaque, size_t len) {
    bspk_batch *b = nullptr;
    int64_t n = 0;
    int rc = BSPK_ERR_ARG;
    if (read_opaque(opaque, len, 0, &b) && b && read_opaque(opaque, len, 8, &n))
        rc = bspk_batch_run(b, n, stream);
    put(stream, static_cast<int64_t *>(buffers[0]), rc == BSPK_OK ? bspk_batch_step_count(b) : -1,
        static_cast<int *>(buffers[1]), rc);
}

}  // extern "C"
