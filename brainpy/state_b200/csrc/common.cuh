// common.cuh -- device building blocks shared by the sm_100a kernels.
//
//  * threefry2x32_20: counter-based RNG of the Poisson drive (no state in HBM).
//  * poisson_from_table: inversion against a per-drive CDF table built on the
//    host in float64 (identical doubles on host and device, so the FP64 path
//    reproduces the CPU restatement count for count).
//  * grid_barrier: bounded-spin barrier for co-resident (cooperative) grids;
//    it gives up after ~2 s of globaltimer and raises an error flag instead of
//    hanging the GPU.
//  * neuron steps in the NEST update order of the reference models.
#pragma once
#include <cstdint>

#include "device_types.h"

namespace bspk {

__device__ __forceinline__ uint32_t rotl32(uint32_t v, int r) { return __funnelshift_l(v, v, r); }

// Threefry-2x32-20 (Salmon et al., SC'11): 5 groups of 4 rounds with key
// injection after each group.
__device__ __forceinline__ void threefry2x32(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1,
                                             uint32_t &y0, uint32_t &y1) {
    const uint32_t k2 = k0 ^ k1 ^ 0x1BD11BDAu;
    uint32_t a = x0 + k0, b = x1 + k1;
#define BSPK_R(r) a += b; b = rotl32(b, r); b ^= a;
    BSPK_R(13) BSPK_R(15) BSPK_R(26) BSPK_R(6)  a += k1; b += k2 + 1u;
    BSPK_R(17) BSPK_R(29) BSPK_R(16) BSPK_R(24) a += k2; b += k0 + 2u;
    BSPK_R(13) BSPK_R(15) BSPK_R(26) BSPK_R(6)  a += k0; b += k1 + 3u;
    BSPK_R(17) BSPK_R(29) BSPK_R(16) BSPK_R(24) a += k1; b += k2 + 4u;
    BSPK_R(13) BSPK_R(15) BSPK_R(26) BSPK_R(6)  a += k2; b += k0 + 5u;
#undef BSPK_R
    y0 = a;
    y1 = b;
}

// 53-bit uniform in [0, 1) from threefry((seed, stream), (step, idx)).
__device__ __forceinline__ double uniform01(uint32_t seed, uint32_t stream, uint32_t step,
                                            uint32_t idx) {
    uint32_t y0, y1;
    threefry2x32(seed, stream, step, idx, y0, y1);
    const uint64_t b = (static_cast<uint64_t>(y0) << 32) | y1;
    return static_cast<double>(b >> 11) * 0x1.0p-53;
}

// The same draw as an integer: b53 = top 53 bits, u = b53 * 2^-53.
__device__ __forceinline__ uint64_t bits53(uint32_t seed, uint32_t stream, uint32_t step,
                                           uint32_t idx) {
    uint32_t y0, y1;
    threefry2x32(seed, stream, step, idx, y0, y1);
    return ((static_cast<uint64_t>(y0) << 32) | y1) >> 11;
}

// fold_in(k, d) = threefry(k, (0, d)) (JAX's key derivation).
__device__ __forceinline__ void fold_key(uint32_t &k0, uint32_t &k1, uint32_t d) {
    uint32_t y0, y1;
    threefry2x32(k0, k1, 0u, d, y0, y1);
    k0 = y0;
    k1 = y1;
}

// The draw of drive `d` for neuron idx of its population at emission step
// `step`, as the integer its threshold table is searched with:
//  kind 0: the library's stream, 53 bits of threefry((seed, 0), (step, idx));
//  kind 1: the reference kernel path's poisson_generator stream
//    (_kernel/models/devices.py:103-145, _kernel/rng.py:338-420): unit
//    u = unit_off + idx of the device population, block key
//    fold(obj, u >> 10), step key fold(fold(block, step), trial) (trial 0
//    for an unbatched run), and the 23 mantissa bits of
//    jax.random.uniform's float32 draw at lane u & 1023.
__device__ __forceinline__ uint64_t drive_draw(const DriveDev &d, uint32_t step, uint32_t idx) {
    if (d.kind == 0) return bits53(d.seed, 0u, step, idx);
    const uint64_t unit = static_cast<uint64_t>(d.unit_off) + idx;
    uint32_t k0 = d.key0, k1 = d.key1;
    fold_key(k0, k1, static_cast<uint32_t>(unit >> 10));
    fold_key(k0, k1, step);
    fold_key(k0, k1, d.trial);
    uint32_t y0, y1;
    threefry2x32(k0, k1, 0u, static_cast<uint32_t>(unit & 1023u), y0, y1);
    return (y0 ^ y1) >> 9;
}

// Smallest k with u <= F[k] (table length if none).  The table holds the CDF
// as integer thresholds T[k] = floor(F[k] * 2^53), so u <= F[k] is exactly
// b53 <= T[k]: no floating point in the search.
__device__ __forceinline__ int poisson_from_table(const uint64_t *T, int n, uint64_t b53) {
    int k = 0;
    while (k < n && b53 > T[k]) ++k;
    return k;
}

// Split-phase grid barrier over a monotonically increasing arrival counter
// that the host zeroes before each launch (`epoch` is 1-based): arrive, do
// independent work, then wait.  The wait gives up after 2 s of globaltimer,
// raises the error flag and returns false instead of hanging.
__device__ __forceinline__ void grid_arrive(unsigned int *counter) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(counter, 1u);
    }
}

__device__ __forceinline__ bool grid_wait(unsigned int *counter, unsigned int epoch, int *err) {
    __shared__ int timed_out_w;
    if (threadIdx.x == 0) {
        timed_out_w = 0;
        const unsigned int target = epoch * gridDim.x;
        uint64_t t0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        unsigned int seen;
        while (true) {
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(counter) : "memory");
            if (seen >= target) break;
            if (*(volatile int *)err) { timed_out_w = 1; break; }
            uint64_t t1;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > 2000000000ull) {  // 2 s
                atomicExch(err, BSPK_DEV_ERR_TIMEOUT);
                timed_out_w = 1;
                break;
            }
            __nanosleep(20);
        }
        __threadfence();
    }
    __syncthreads();
    return timed_out_w == 0;
}

// Bounded grid barrier over a monotonically increasing arrival counter that
// the host zeroes before each launch.  `epoch` is 1-based.
__device__ __forceinline__ bool grid_barrier(unsigned int *counter, unsigned int epoch,
                                             int *err) {
    __syncthreads();
    __shared__ int timed_out;
    if (threadIdx.x == 0) {
        timed_out = 0;
        __threadfence();
        atomicAdd(counter, 1u);
        const unsigned int target = epoch * gridDim.x;
        uint64_t t0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        unsigned int seen;
        while (true) {
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(counter) : "memory");
            if (seen >= target) break;
            if (*(volatile int *)err) { timed_out = 1; break; }
            uint64_t t1;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > 2000000000ull) {  // 2 s
                atomicExch(err, BSPK_DEV_ERR_TIMEOUT);
                timed_out = 1;
                break;
            }
            __nanosleep(20);
        }
        __threadfence();
    }
    __syncthreads();
    return timed_out == 0;
}

// ---------------------------------------------------------------- neurons

// iaf_psc_alpha, NEST order (_nest_neuron/iaf_psc_alpha.py:558-684).
// s: V, I_ex, dI_ex, I_in, dI_in, y0.  w_all: summed delta input (pA).
// Two-port form: w_ex / w_in are the jumps of this step's excitatory and
// inhibitory receptor ports, signs kept (_kernel/models/iaf_psc_alpha.py
// ports 'ex' / 'in_'); iaf_alpha_step below splits one summed input by sign.
template <typename Real>
__device__ __forceinline__ bool iaf_alpha_step_ports(const PopCoef<Real> &c, Real (&s)[6], int &r,
                                                     Real w_ex, Real w_in) {
    Real y3 = s[0] - c.E_L;
    if (r == 0) {
        Real v = c.P30 * (s[5] + c.I_e) + c.P31ex * s[2] + c.P32ex * s[1] + c.P31in * s[4] +
                 c.P32in * s[3] + c.expm1_tm * y3 + y3;
        if (!(v >= c.lower)) v = c.lower;
        y3 = v;
    } else {
        r = r - 1;
    }
    const Real Iex = c.P21ex * s[2] + c.P22ex * s[1];
    Real dIex = s[2] * c.P11ex;
    dIex = dIex + c.epsc * w_ex;
    const Real Iin = c.P21in * s[4] + c.P22in * s[3];
    Real dIin = s[4] * c.P11in;
    dIin = dIin + c.ipsc * w_in;
    const bool spike = y3 >= c.theta;
    if (spike) {
        r = c.ref_count;
        y3 = c.vreset;
    }
    s[0] = y3 + c.E_L;
    s[1] = Iex;
    s[2] = dIex;
    s[3] = Iin;
    s[4] = dIin;
    s[5] = Real(0);  // no current injector on this path: y0 <- 0
    return spike;
}
template <typename Real>
__device__ __forceinline__ bool iaf_alpha_step(const PopCoef<Real> &c, Real (&s)[6], int &r,
                                               Real w_all) {
    return iaf_alpha_step_ports<Real>(c, s, r, w_all > Real(0) ? w_all : Real(0),
                                      w_all < Real(0) ? w_all : Real(0));
}

// iaf_psc_exp, deterministic threshold (_nest_neuron/iaf_psc_exp.py:552-682).
// s: V, i_syn_ex, i_syn_in, i_0, i_1.
template <typename Real>
__device__ __forceinline__ bool iaf_exp_step_ports(const PopCoef<Real> &c, Real (&s)[6], int &r,
                                                   Real w_ex, Real w_in) {
    Real V_rel = s[0] - c.E_L;
    if (r == 0) {
        V_rel = V_rel * c.eP22 + s[1] * c.eP21ex + s[2] * c.eP21in + (c.I_e + s[3]) * c.eP20;
    } else {
        r = r - 1;
    }
    Real iex = s[1] * c.eP11ex;
    Real iin = s[2] * c.eP11in;
    iex = iex + c.one_m_eP11ex * s[4];
    iex = iex + w_ex;
    iin = iin + w_in;
    const bool spike = V_rel >= c.theta;
    if (spike) {
        r = c.ref_count;
        V_rel = c.vreset;
    }
    s[0] = V_rel + c.E_L;
    s[1] = iex;
    s[2] = iin;
    s[3] = Real(0);
    s[4] = Real(0);
    return spike;
}
template <typename Real>
__device__ __forceinline__ bool iaf_exp_step(const PopCoef<Real> &c, Real (&s)[6], int &r,
                                             Real w_all) {
    return iaf_exp_step_ports<Real>(c, s, r, w_all > Real(0) ? w_all : Real(0),
                                    w_all < Real(0) ? w_all : Real(0));
}

}  // namespace bspk
