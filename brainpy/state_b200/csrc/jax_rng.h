// jax_rng.h -- the reference's random streams on the host: JAX's threefry
// PRNG in its partitionable layout (jax >= 0.5 default), jax.random.uniform
// and jax.random.normal for float32 and float64, the key chain of the
// reference's kernel path (_kernel/rng.py, _kernel/compiler.py:95-97,
// _kernel/params.py:348-354), and the CDF-inversion table of its
// poisson_generator (_kernel/models/devices.py:49-139).
//
// Layout facts restated here (JAX, jax/_src/prng.py and jax/_src/random.py):
//  * key(seed) = (seed >> 32, seed & 0xffffffff);
//  * fold_in(k, d) = threefry(k, (0, d)); split(k, n)[i] = threefry(k, (0, i));
//  * random_bits(k, shape)[i] = threefry(k, (i >> 32, i & 0xffffffff)),
//    32-bit: y0 ^ y1, 64-bit: y0 << 32 | y1;
//  * uniform: mantissa bits (bits >> (nbits - nmant)) under the exponent of
//    1.0, minus 1.0, then floats * (hi - lo) + lo, then max(lo, .);
//  * normal: uniform on [nextafter(-1, 0), 1), then sqrt(2) * erfinv(u).
// XLA evaluates float32 erfinv with M. Giles' single-precision polynomial
// ("Approximating the erfinv function", GPU Computing Gems Jade, 2011) on
// w = -log1p(-x * x); that is restated below.  The float64 erfinv is
// evaluated to within an ulp or two by Newton steps on erf / erfc.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "host_rng.h"

namespace bspk {

inline uint32_t jax_bits32(JaxKey k, uint64_t i) {
    uint32_t y0, y1;
    tf2x32(k.k0, k.k1, static_cast<uint32_t>(i >> 32), static_cast<uint32_t>(i), y0, y1);
    return y0 ^ y1;
}
inline uint64_t jax_bits64(JaxKey k, uint64_t i) {
    uint32_t y0, y1;
    tf2x32(k.k0, k.k1, static_cast<uint32_t>(i >> 32), static_cast<uint32_t>(i), y0, y1);
    return (static_cast<uint64_t>(y0) << 32) | y1;
}

// [0, 1) from the draw's bits: the top mantissa bits under 1.0's exponent.
inline float jax_unit_f32(uint32_t bits) {
    const uint32_t b = (bits >> 9) | 0x3F800000u;
    float f;
    std::memcpy(&f, &b, 4);
    return f - 1.0f;
}
inline double jax_unit_f64(uint64_t bits) {
    const uint64_t b = (bits >> 12) | 0x3FF0000000000000ull;
    double f;
    std::memcpy(&f, &b, 8);
    return f - 1.0;
}

// One element of jax.random.uniform(key, (n,), dtype, lo, hi).  The
// multiply and the add are separate roundings (no fused multiply-add).
inline float jax_uniform_f32_at(JaxKey k, uint64_t i, float lo, float hi) {
    const float span = hi - lo;
    volatile float prod = jax_unit_f32(jax_bits32(k, i)) * span;
    const float v = prod + lo;
    return v > lo ? v : lo;
}
inline double jax_uniform_f64_at(JaxKey k, uint64_t i, double lo, double hi) {
    const double span = hi - lo;
    volatile double prod = jax_unit_f64(jax_bits64(k, i)) * span;
    const double v = prod + lo;
    return v > lo ? v : lo;
}

// erfinv in float32 as XLA evaluates it (Giles' single-precision form).
inline float erfinv_f32(float x) {
    static const float kLt5[9] = {2.81022636e-08f,  3.43273939e-07f, -3.5233877e-06f,
                                  -4.39150654e-06f, 0.00021858087f,  -0.00125372503f,
                                  -0.00417768164f,  0.246640727f,    1.50140941f};
    static const float kGe5[9] = {-0.000200214257f, 0.000100950558f, 0.00134934322f,
                                  -0.00367342844f,  0.00573950773f,  -0.0076224613f,
                                  0.00943887047f,   1.00167406f,     2.83297682f};
    if (std::fabs(x) == 1.0f) return x * INFINITY;
    volatile float xx = x * x;
    float w = -std::log1p(-static_cast<float>(xx));
    const float *c;
    if (w < 5.0f) {
        w = w - 2.5f;
        c = kLt5;
    } else {
        w = std::sqrt(w) - 3.0f;
        c = kGe5;
    }
    float p = c[0];
    for (int i = 1; i < 9; ++i) {
        volatile float pw = p * w;
        p = c[i] + static_cast<float>(pw);
    }
    return p * x;
}

// erfinv in float64: the float32 form as a start, then Newton steps on erf
// (|x| < 0.5) or erfc (|x| >= 0.5, where 1 - |x| is exact).
inline double erfinv_f64(double x) {
    if (std::fabs(x) == 1.0) return x * INFINITY;
    if (x == 0.0) return x;
    const double ax = std::fabs(x);
    double y = std::fabs(static_cast<double>(erfinv_f32(static_cast<float>(ax))));
    if (!std::isfinite(y)) y = 6.0;
    const double k = 1.1283791670955125739;  // 2 / sqrt(pi)
    for (int it = 0; it < 4; ++it) {
        const double d = k * std::exp(-y * y);
        double step;
        if (ax < 0.5) step = (std::erf(y) - ax) / d;
        else step = ((1.0 - ax) - std::erfc(y)) / d;
        y -= step;
        if (std::fabs(step) <= 1e-17 * y) break;
    }
    return x < 0 ? -y : y;
}

inline float jax_normal_f32_at(JaxKey k, uint64_t i) {
    const float lo = std::nextafter(-1.0f, 0.0f);
    const float u = jax_uniform_f32_at(k, i, lo, 1.0f);
    return 1.41421354f * erfinv_f32(u);  // np.sqrt(2) as float32
}
inline double jax_normal_f64_at(JaxKey k, uint64_t i) {
    const double lo = std::nextafter(-1.0, 0.0);
    const double u = jax_uniform_f64_at(k, i, lo, 1.0);
    return 1.4142135623730951 * erfinv_f64(u);
}

// Run f(i) for i in [0, n) on up to 32 host threads (large draws only).
template <typename F>
void parallel_for(int64_t n, F f) {
    unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 100000) nth = 1;
    if (nth == 1) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> ts;
    const int64_t chunk = (n + nth - 1) / nth;
    for (unsigned t = 0; t < nth; ++t) {
        const int64_t a = t * chunk, b = std::min<int64_t>(n, a + chunk);
        if (a >= b) break;
        ts.emplace_back([=]() {
            for (int64_t i = a; i < b; ++i) f(i);
        });
    }
    for (auto &th : ts) th.join();
}

// Kernel-path poisson_generator: the mean per unit and step in float32,
// lam = rate [kHz] * dt [ms] (devices.py:203), and the table of the CDF
// inversion (devices.py:46-67): p_0 = exp(-lam), p_k = p_{k-1} * lam / k,
// F_k = F_{k-1} + p_k, all in float32 with denormals flushed to zero (XLA's
// CPU setting); the count of a draw u = m * 2^-23 is #{k : u >= F_k} over the
// terms with p_k > 0 (the first 12 unconditionally).  Returned as integer
// thresholds t_k = ceil(F_k * 2^23) - 1, so that the count is the number of
// leading k with m > t_k (the library's table search).
inline float kernel_poisson_lam(double rate_hz, double dt_ms) {
    return static_cast<float>(rate_hz * dt_ms / 1000.0);
}
inline std::vector<uint64_t> kernel_poisson_table(float lam) {
    std::vector<uint64_t> t;
    auto ftz = [](float v) { return std::fabs(v) < 1.17549435e-38f ? 0.0f : v; };
    float p = ftz(static_cast<float>(std::exp(-static_cast<double>(lam))));
    float F = p;
    for (int k = 0; k < 4096; ++k) {
        if (k >= 12 && !(p > 0.0f)) break;
        t.push_back(static_cast<uint64_t>(std::ceil(std::ldexp(static_cast<double>(F), 23))) - 1);
        volatile float pl = p * lam;
        p = ftz(ftz(static_cast<float>(pl)) / static_cast<float>(k + 1));
        volatile float Fn = F + p;
        F = Fn;
    }
    return t;
}

}  // namespace bspk
