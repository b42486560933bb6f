// jax_rng.cpp -- C ABI over jax_rng.h: the reference's random draws on the
// host, for the front ends that realise distributed weights, delays and
// initial states on the reference's keys.
#include <string>

#include "bspk.h"
#include "jax_rng.h"
#include "plan_internal.h"

using namespace bspk;

extern "C" {

int bspk_jax_fold_in(const uint32_t *key, uint32_t data, uint32_t *out) {
    if (!key || !out) return fail(BSPK_ERR_ARG, "null key");
    const JaxKey k = jax_fold(JaxKey{key[0], key[1]}, data);
    out[0] = k.k0;
    out[1] = k.k1;
    return BSPK_OK;
}

int bspk_jax_uniform(const uint32_t *key, int64_t n, int bits, double lo, double hi,
                     double *out) {
    if (!key || (n > 0 && !out) || n < 0) return fail(BSPK_ERR_ARG, "bad argument");
    if (bits != 32 && bits != 64) return fail(BSPK_ERR_ARG, "bits must be 32 or 64");
    const JaxKey k{key[0], key[1]};
    if (bits == 32) {
        const float l = static_cast<float>(lo), h = static_cast<float>(hi);
        parallel_for(n, [&](int64_t i) { out[i] = jax_uniform_f32_at(k, i, l, h); });
    } else {
        parallel_for(n, [&](int64_t i) { out[i] = jax_uniform_f64_at(k, i, lo, hi); });
    }
    return BSPK_OK;
}

int bspk_jax_normal(const uint32_t *key, int64_t n, int bits, double *out) {
    if (!key || (n > 0 && !out) || n < 0) return fail(BSPK_ERR_ARG, "bad argument");
    if (bits != 32 && bits != 64) return fail(BSPK_ERR_ARG, "bits must be 32 or 64");
    const JaxKey k{key[0], key[1]};
    if (bits == 32) parallel_for(n, [&](int64_t i) { out[i] = jax_normal_f32_at(k, i); });
    else parallel_for(n, [&](int64_t i) { out[i] = jax_normal_f64_at(k, i); });
    return BSPK_OK;
}

int bspk_kernel_poisson_table(double rate_hz, double dt_ms, int cap, uint64_t *thresholds,
                              int *n_out) {
    if (!n_out || cap < 0 || (cap > 0 && !thresholds)) return fail(BSPK_ERR_ARG, "bad argument");
    const float lam = kernel_poisson_lam(rate_hz, dt_ms);
    if (!(lam >= 0.0f) || lam >= 10.0f)
        return fail(BSPK_ERR_UNSUPPORTED, "the kernel stream's CDF inversion needs rate*dt < 10");
    const std::vector<uint64_t> t = kernel_poisson_table(lam);
    *n_out = static_cast<int>(t.size());
    for (int i = 0; i < cap && i < static_cast<int>(t.size()); ++i) thresholds[i] = t[i];
    return BSPK_OK;
}

}  // extern "C"
