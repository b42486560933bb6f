// device_types.h -- plain structs shared by the host plan and the kernels.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

namespace bspk {

enum {
    BSPK_DEV_OK = 0,
    BSPK_DEV_ERR_TIMEOUT = 1,
    BSPK_DEV_ERR_OVERFLOW = 2,
    BSPK_DEV_ERR_BOUNDS = 3,
    BSPK_DEV_ERR_UNSTABLE = 4,
    BSPK_DEV_ERR_RKCAP = 5,
};

// Conductance models (ids 2..4 of bspk.h: aeif_cond_alpha, iaf_cond_exp,
// iaf_cond_alpha) run on the RKF45 per-step engine with two receptor ports.
// Their state slots are the ODE leaves, then the integration step h and the
// buffered current I_stim.
__host__ __device__ constexpr bool model_is_cond(int model) { return model >= 2 && model <= 4; }
__host__ __device__ constexpr int cond_n_ode(int model) {
    return model == 2 ? 6 : (model == 3 ? 3 : 5);
}
// iaf_psc_exp_multisynapse (id 5): V_m, i_const, then one synaptic current
// per receptor (kMaxReceptors slots whatever the population's count)
constexpr int kMaxReceptors = 4;
__host__ __device__ constexpr int model_n_slots(int model) {
    return model_is_cond(model) ? cond_n_ode(model) + 2 : (model == 5 ? 2 + kMaxReceptors : 6);
}
// models stepped by the per-step engine (one launch sequence per step)
__host__ __device__ constexpr bool model_per_step(int model) { return model >= 2; }
// input channels of the ring: the receptor ports of the model
__host__ __device__ constexpr int model_n_receptors(int model) {
    return model_is_cond(model) ? 2 : (model == 5 ? kMaxReceptors : 1);
}

constexpr int kMaxPops = 64;
constexpr int kMaxInputs = 64;   // drives + projections per plan
constexpr int kMaxWindow = 32;   // d_min batching window (steps)
constexpr int kEdgeDelayShift = 24;
constexpr uint32_t kEdgePostMask = (1u << kEdgeDelayShift) - 1u;

// Per-population coefficients, computed on the host in float64 and cast to
// the compute type.  Covers iaf_psc_alpha (P11..P32, epsc/ipsc) and
// iaf_psc_exp (eP*); the aeif fields hold the NEST parameters directly.
template <typename Real>
struct PopCoef {
    Real E_L, I_e, lower, theta, vreset;
    Real P11ex, P21ex, P22ex, P11in, P21in, P22in, expm1_tm, P30, P31ex, P32ex, P31in, P32in,
        epsc, ipsc;
    Real eP11ex, eP11in, eP22, eP21ex, eP21in, eP20, one_m_eP11ex;
    // aeif_cond_alpha
    Real V_peak, V_reset, g_L, C_m, E_ex, E_in, Delta_T, tau_w, a, b, V_th, tau_syn_ex,
        tau_syn_in, atol, pscon_ex, pscon_in, v_peak_detect;
    // reciprocals taken once on the host in FP64: the RKF45 stages multiply
    // instead of dividing (a division is a long dependent sequence on the
    // substep chain); inv_Delta_T and inv_atol stay FP64 for the exponential
    // term and the error norm
    Real inv_C_m, inv_tau_syn_ex, inv_tau_syn_in, inv_tau_w;
    double inv_Delta_T, inv_atol;
    // 1 / Delta_T as an unevaluated FP32 sum hi + lo (|lo| <= ulp(hi) / 2):
    // an FP32 state forms the exponent d / Delta_T to FP64 accuracy in FP32
    float inv_Delta_T_hi, inv_Delta_T_lo;
    // iaf_psc_exp_multisynapse: per-receptor decay and membrane coupling
    // (eP22 / eP20 hold the membrane propagators)
    Real msP11[4], msP21[4];
    int nrec;
    int ref_count;
    int off, n;  // gid range of the population
};

// Poisson drive of one population.
struct DriveDev {
    int pop;
    int lag;           // arrival lag in steps (LEGACY: delay + 1)
    uint32_t seed;
    int cdf_off, cdf_n;
    int receptor;
    double weight;
    int64_t tmin, tmax;
    // stream: 0 = the library's counter stream (53-bit thresholds);
    // 1 = the reference kernel path's block-key stream (23-bit thresholds)
    // of the device population with object key (key0, key1), whose unit
    // unit_off + i drives neuron i of `pop`
    int kind;
    uint32_t key0, key1;
    int64_t unit_off;
    uint32_t trial;    // kind 1: trial index folded into every step key
};

// One projection (CSR over the pre population's local indices).
template <typename Real>
struct ProjDev {
    int pre_pop, post_pop, post_off, receptor;
    int homogeneous;     // 1: every edge carries w0
    Real w0;
    const int64_t *indptr;   // n_pre + 1
    const uint32_t *edges;   // post_local | (arrival lag << 24)
    const Real *w;           // per edge (nullptr when homogeneous)
    // deterministic pull (CSC over post local indices, sorted by pre)
    const int64_t *cindptr;  // n_post + 1
    const uint32_t *cedges;  // pre_local | (arrival lag << 24)
    const double *cw;        // per in-edge weight (nullptr when homogeneous)
};

// An arrival of a window: CSR edge and pre.
struct WinArrival {
    uint32_t e, pre;
};

}  // namespace bspk
