// per_step.cu -- per-step engine: the conductance models (aeif_cond_alpha,
// iaf_cond_exp, iaf_cond_alpha) with adaptive RKF45, iaf_psc_exp_multisynapse
// (one input channel per receptor), and networks with plastic
// stdp_synapse / stdp_triplet_synapse projections (any neuron model).
//
// One step n is this kernel sequence (the reference Simulator's phase order,
// _nest_network/simulator.py:1719-1788):
//   memset of the step's counters;
//   per plastic projection: traces (decay-then-add), facilitation on the
//   in-edges of neurons that fired at n-1, depression + delivery on the
//   out-edges of pres whose delayed spike arrives at n (the order of
//   _nest_plasticity/stdp_synapse.py:171-179), adding into ring slot n;
//   neuron update (one neuron per thread; RKF45 per neuron with FP64 error
//   norm and step control, FP64 exponential term);
//   static delivery of step n's spikes into ring slots n + lag (warp per row);
//   step counter += 1.
// The step index lives in device memory, so a CUDA graph captured over K
// steps is replayed for every chunk of K steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "aeif_args.h"
#include "common.cuh"
#include "plan_internal.h"

namespace bspk {

namespace {

template <typename Real>
__device__ __forceinline__ int find_pop_t(const PopCoef<Real> *c, int npop, int g) {
    int p = 0;
    while (p + 1 < npop && c[p + 1].off <= g) ++p;
    return p;
}

// Edge work items of the delivery and STDP kernels: kEdgeU edges per lane,
// kChunkEdges = 32 kEdgeU per warp-sized item.
constexpr int kEdgeU = 8;
constexpr int kChunkEdges = 32 * kEdgeU;
// plastic arrivals of one window step taken together by a neuron thread
constexpr int kWinArrU = 8;

__device__ __forceinline__ bool fired(const uint64_t *hist, int gid, int64_t m) {
    if (m < 0) return false;
    return (hist[gid] >> (m & 63)) & 1ull;
}

// ------------------------------------------------ aeif_cond_alpha + RKF45

// RKF45 tableau (_nest_base/utils.py:266-279); b_err = b - b_hat.
__device__ constexpr double kA[6][5] = {
    {0, 0, 0, 0, 0},
    {1.0 / 4, 0, 0, 0, 0},
    {3.0 / 32, 9.0 / 32, 0, 0, 0},
    {1932.0 / 2197, -7200.0 / 2197, 7296.0 / 2197, 0, 0},
    {439.0 / 216, -8.0, 3680.0 / 513, -845.0 / 4104, 0},
    {-8.0 / 27, 2.0, -3544.0 / 2565, 1859.0 / 4104, -11.0 / 40},
};
__device__ constexpr double kB[6] = {16.0 / 135, 0.0, 6656.0 / 12825, 28561.0 / 56430, -9.0 / 50, 2.0 / 55};
__device__ constexpr double kBhat[6] = {25.0 / 216, 0.0, 1408.0 / 2565, 2197.0 / 4104, -1.0 / 5, 0.0};

// Vector field (_nest_neuron/aeif_cond_alpha.py:554-592).
//
// The exponential spike current g_L Delta_T exp((V - V_th) / Delta_T) in an
// FP64 state is FP64 throughout.  In an FP32 state it is FP32 arithmetic to
// the accuracy of FP32 rounding: the exponent d / Delta_T is carried as the
// unevaluated sum arg + lo (arg = d * hi rounded, lo = the product's rounding
// error plus d * lo(1 / Delta_T), both exact to a few ulp of lo), and
// exp(arg + lo) = expf(arg) (1 + lo) to O(lo^2) (|lo| < 1e-5, so lo^2 is far
// below FP32's 6e-8).  expf's own error is at most 2 ulp, so the current is
// within about 3 ulp of the correctly rounded value at every V, including the
// spike-initiation zone where the term grows without bound and the adaptive
// step control spends most of a spiking neuron's trial steps.  The exponent is
// clamped to [-500, 88] (expf(88) is finite; a zero Delta_T then still gives a
// zero term).
template <typename Real>
__device__ __forceinline__ void aeif_vf(const PopCoef<Real> &c, int r, Real i_stim, const Real *y,
                                        Real *dy) {
    const bool refr = r > 0;
    const Real v = y[0];
    const Real v_eff = refr ? c.V_reset : (v < c.V_peak ? v : (v != v ? v : c.V_peak));
    const Real i_ex = y[2] * (v_eff - c.E_ex);
    const Real i_in = y[4] * (v_eff - c.E_in);
    Real i_spike;
    if constexpr (sizeof(Real) == 4) {
        const float d = v_eff - c.V_th;
        const float arg = d * c.inv_Delta_T_hi;
        const float lo = fmaf(d, c.inv_Delta_T_hi, -arg) + d * c.inv_Delta_T_lo;
        const float ac = arg < -500.0f ? -500.0f : (arg > 88.0f ? 88.0f : arg);
        const float e = expf(ac);
        i_spike = (c.g_L * c.Delta_T) * fmaf(e, lo, e);
    } else {
        double arg = static_cast<double>(v_eff - c.V_th) * c.inv_Delta_T;
        arg = arg < -500.0 ? -500.0 : (arg > 500.0 ? 500.0 : arg);
        i_spike = static_cast<Real>(static_cast<double>(c.g_L) * static_cast<double>(c.Delta_T) *
                                    exp(arg));
    }
    Real dV;
    if constexpr (sizeof(Real) == 4) {
        // FP32: the terms that do not wait for the exponential are summed
        // while it is evaluated, and the spike current joins last
        const Real rest = -c.g_L * (v_eff - c.E_L) - i_ex - i_in - y[5] + c.I_e + i_stim;
        dV = (rest + i_spike) * c.inv_C_m;
    } else {
        // FP64: the reference's order of the sum
        dV = (-c.g_L * (v_eff - c.E_L) + i_spike - i_ex - i_in - y[5] + c.I_e + i_stim) * c.inv_C_m;
    }
    dy[0] = refr ? Real(0) : dV;
    dy[1] = -y[1] * c.inv_tau_syn_ex;
    dy[2] = y[1] - y[2] * c.inv_tau_syn_ex;
    dy[3] = -y[3] * c.inv_tau_syn_in;
    dy[4] = y[3] - y[4] * c.inv_tau_syn_in;
    dy[5] = (c.a * (v_eff - c.E_L) - y[5]) * c.inv_tau_w;
}

// Vector fields of the iaf conductance models: iaf_cond_exp
// (_nest_neuron/iaf_cond_exp.py:456-490; y = V, g_ex, g_in) and
// iaf_cond_alpha (_nest_neuron/iaf_cond_alpha.py:459-491; y = V, dg_ex, g_ex,
// dg_in, g_in).  The membrane sees min(V, V_th), or V_reset while refractory.
template <typename Real, int MODEL>
__device__ __forceinline__ void iaf_cond_vf(const PopCoef<Real> &c, int r, Real i_stim,
                                            const Real *y, Real *dy) {
    const bool refr = r > 0;
    const Real v = y[0];
    const Real v_eff = refr ? c.V_reset : (v < c.V_th ? v : (v != v ? v : c.V_th));
    const Real gex = MODEL == 3 ? y[1] : y[2];
    const Real gin = MODEL == 3 ? y[2] : y[4];
    const Real i_syn_exc = gex * (v_eff - c.E_ex);
    const Real i_syn_inh = gin * (v_eff - c.E_in);
    const Real i_leak = c.g_L * (v_eff - c.E_L);
    const Real dV = (-i_leak - i_syn_exc - i_syn_inh + c.I_e + i_stim) * c.inv_C_m;
    dy[0] = refr ? Real(0) : dV;
    if constexpr (MODEL == 3) {
        dy[1] = -y[1] * c.inv_tau_syn_ex;
        dy[2] = -y[2] * c.inv_tau_syn_in;
    } else {
        dy[1] = -y[1] * c.inv_tau_syn_ex;
        dy[2] = y[1] - y[2] * c.inv_tau_syn_ex;
        dy[3] = -y[3] * c.inv_tau_syn_in;
        dy[4] = y[3] - y[4] * c.inv_tau_syn_in;
    }
}

// err^(-q) of the step-size factor 0.9 (1 / err)^q, as exp(-q log err): no
// division and a shorter chain than pow on the substep's critical path.  An
// FP32 state takes it in FP32: the factor only sizes the next trial step,
// whose error the FP64 norm then tests, so acceptance stays FP64.
template <typename Real>
__device__ __forceinline__ double err_pow(double err, double q) {
    if constexpr (sizeof(Real) == 4)
        return static_cast<double>(
            exp2f(-static_cast<float>(q) * log2f(static_cast<float>(err))));
    else
        return exp(-q * log(err));
}

// One dt of the adaptive RKF45 loop (_nest_base/utils.py:583-718) for a
// conductance model (MODEL 2: aeif_cond_alpha, 3: iaf_cond_exp,
// 4: iaf_cond_alpha), with the model's in-loop spike/reset event
// (aeif_cond_alpha.py:594-625, iaf_cond_exp.py:487-517,
// iaf_cond_alpha.py:493-521) and the synaptic jumps after integration
// (aeif_cond_alpha.py:709-728, iaf_cond_exp.py:594-614,
// iaf_cond_alpha.py:602-624).  s: the NS ODE leaves, then h and I_stim.
// The step is split into rk_begin, rk_substep (one trial step of the loop),
// rk_done and rk_end (cond_step runs the four in sequence).
template <typename Real, int MODEL>
struct RkState {
    static constexpr int NS = cond_n_ode(MODEL);
    Real y[NS];
    double h, t_loc;
    Real i_stim;
    int iters;
    bool spiked, unstable;
};
template <int MODEL>
__host__ __device__ constexpr int rk_max_iters() {
    return MODEL == 3 ? 10000 : 100000;  // the models' _MAX_ITERS
}
constexpr double kRkMinH = 1e-8;

template <typename Real, int MODEL>
__device__ __forceinline__ void rk_begin(RkState<Real, MODEL> &q, const Real *s) {
    constexpr int NS = RkState<Real, MODEL>::NS;
#pragma unroll
    for (int i = 0; i < NS; ++i) q.y[i] = s[i];
    q.h = static_cast<double>(s[NS]);
    q.i_stim = s[NS + 1];
    q.spiked = false;
    q.unstable = false;
    q.t_loc = 0.0;
    if (q.h < kRkMinH) q.h = kRkMinH;
    q.iters = 0;
}
template <typename Real, int MODEL>
__device__ __forceinline__ bool rk_done(const RkState<Real, MODEL> &q, double dt) {
    return !(q.t_loc < dt && q.iters < rk_max_iters<MODEL>());
}
template <typename Real, int MODEL>
__device__ __forceinline__ void rk_substep(const PopCoef<Real> &c, RkState<Real, MODEL> &q, int &r,
                                           double dt) {
    constexpr int NS = RkState<Real, MODEL>::NS;
    const double inv_atol = c.inv_atol;
    Real k[6][NS];
    {
        const double hh = q.h < dt - q.t_loc ? q.h : dt - q.t_loc;
        q.h = hh > kRkMinH ? hh : kRkMinH;
        const Real hR = static_cast<Real>(q.h);
#pragma unroll
        for (int st = 0; st < 6; ++st) {
            Real yi[NS];
            if (st == 0) {
#pragma unroll
                for (int i = 0; i < NS; ++i) yi[i] = q.y[i];
            } else {
#pragma unroll
                for (int i = 0; i < NS; ++i) {
                    Real acc = Real(0);
                    bool first = true;
#pragma unroll
                    for (int j = 0; j < st; ++j) {
                        const double aij = kA[st][j];
                        if (aij == 0.0) continue;
                        const Real term = static_cast<Real>(aij) * k[j][i];
                        acc = first ? term : acc + term;
                        first = false;
                    }
                    yi[i] = q.y[i] + hR * acc;
                }
            }
            if constexpr (MODEL == 2) aeif_vf<Real>(c, r, q.i_stim, yi, k[st]);
            else iaf_cond_vf<Real, MODEL>(c, r, q.i_stim, yi, k[st]);
        }
        Real yh[NS];
        double ev[NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            Real acc = Real(0), eacc = Real(0);
            bool first = true, efirst = true;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                if (kB[j] != 0.0) {
                    const Real term = static_cast<Real>(kB[j]) * k[j][i];
                    acc = first ? term : acc + term;
                    first = false;
                }
                const double be = kB[j] - kBhat[j];
                if (be != 0.0) {
                    const Real term = static_cast<Real>(be) * k[j][i];
                    eacc = efirst ? term : eacc + term;
                    efirst = false;
                }
            }
            yh[i] = q.y[i] + hR * acc;
            const Real ye = hR * eacc;
            const double ay = fabs(static_cast<double>(q.y[i])) > fabs(static_cast<double>(yh[i]))
                                  ? fabs(static_cast<double>(q.y[i]))
                                  : fabs(static_cast<double>(yh[i]));
            // |err| / atol (rtol = 0); the 0 * |y| term carries a NaN or an
            // infinite state into the norm as the reference's scale does
            ev[i] = fabs(static_cast<double>(ye)) * inv_atol + 0.0 * ay;
        }
        // the largest component (NaN if any is NaN), folded as a tree: the
        // same value as the sequential fold in fewer dependent steps
#pragma unroll
        for (int span = 1; span < NS; span <<= 1) {
#pragma unroll
            for (int i = 0; i + span < NS; i += 2 * span) {
                const double x = ev[i], y = ev[i + span];
                ev[i] = (x != x || y != y) ? NAN : (x > y ? x : y);
            }
        }
        double err = ev[0];
        if (err != err) err = INFINITY;
        const bool accept = (err <= 1.0) || (q.h <= kRkMinH);
        if (accept) {
#pragma unroll
            for (int i = 0; i < NS; ++i) q.y[i] = yh[i];
            q.t_loc = q.t_loc + q.h;
            if constexpr (MODEL == 2) {
                if (q.y[0] < Real(-1e3) || q.y[5] < Real(-1e6) || q.y[5] > Real(1e6)) q.unstable = true;
            } else if constexpr (MODEL == 3) {
                if (q.y[0] < Real(-1e3)) q.unstable = true;
            }
            if (r > 0) q.y[0] = c.V_reset;
            if (r <= 0 && q.y[0] >= c.v_peak_detect) {
                q.spiked = true;
                q.y[0] = c.V_reset;
                if constexpr (MODEL == 2) q.y[5] = q.y[5] + c.b;
                if (c.ref_count > 0) r = c.ref_count + 1;
            }
        }
        const double err_sg = err > 1e-30 ? err : 1e-30;
        double fac;
        if (accept) {
            fac = err_sg <= 1e-30 ? 5.0 : 0.9 * err_pow<Real>(err_sg, 0.2);
            if (!(err_sg <= 1e-30)) fac = fac < 0.2 ? 0.2 : (fac > 5.0 ? 5.0 : fac);
        } else {
            fac = 0.9 * err_pow<Real>(err_sg, 0.25);
            fac = fac < 0.2 ? 0.2 : (fac > 1.0 ? 1.0 : fac);
        }
        const double hn = q.h * fac;
        q.h = hn > kRkMinH ? hn : kRkMinH;
        ++q.iters;
    }
}
template <typename Real, int MODEL>
__device__ __forceinline__ bool rk_end(const PopCoef<Real> &c, RkState<Real, MODEL> &q, Real *s, int &r,
                                       Real w_ex, Real w_in, double dt, int *err,
                                       unsigned long long *rk_iters) {
    constexpr int NS = RkState<Real, MODEL>::NS;
    if (q.iters >= rk_max_iters<MODEL>() && q.t_loc < dt) atomicExch(err, BSPK_DEV_ERR_RKCAP);
    if (q.unstable) atomicExch(err, BSPK_DEV_ERR_UNSTABLE);
    if (rk_iters) {
        // one atomic per group of converged lanes, not one per neuron
        const unsigned m = __activemask();
        const unsigned sum = __reduce_add_sync(m, static_cast<unsigned>(q.iters));
        if ((threadIdx.x & 31) == __ffs(m) - 1)
            atomicAdd(rk_iters, static_cast<unsigned long long>(sum));
    }
    if (r > 0) r = r - 1;
    if constexpr (MODEL == 3) {
        q.y[1] = q.y[1] + w_ex;
        q.y[2] = q.y[2] + w_in;
    } else {
        q.y[1] = q.y[1] + c.pscon_ex * w_ex;
        q.y[3] = q.y[3] + c.pscon_in * w_in;
    }
#pragma unroll
    for (int i = 0; i < NS; ++i) s[i] = q.y[i];
    s[NS] = static_cast<Real>(q.h);
    s[NS + 1] = Real(0);  // no current input on this path: I_stim <- 0
    return q.spiked;
}
template <typename Real, int MODEL>
__device__ bool cond_step(const PopCoef<Real> &c, Real *s, int &r, Real w_ex, Real w_in,
                          double dt, int *err, unsigned long long *rk_iters) {
    RkState<Real, MODEL> q;
    rk_begin<Real, MODEL>(q, s);
    while (!rk_done<Real, MODEL>(q, dt)) rk_substep<Real, MODEL>(c, q, r, dt);
    return rk_end<Real, MODEL>(c, q, s, r, w_ex, w_in, dt, err, rk_iters);
}

// iaf_psc_exp_multisynapse (_nest_neuron/iaf_psc_exp_multisynapse.py:716-790):
// exact membrane propagation summing every receptor's current, refractory
// countdown, receptor decay plus this step's weights, threshold and reset.
// s: V_m, i_const, i_syn[kMaxReceptors]; w: weight per receptor (pA).
template <typename Real>
__device__ __forceinline__ bool iaf_ms_step(const PopCoef<Real> &c, Real *s, int &r,
                                            const Real *w) {
    Real v = s[0] - c.E_L;
    if (r == 0) {
        Real syn = c.msP21[0] * s[2];
#pragma unroll
        for (int k = 1; k < kMaxReceptors; ++k)
            if (k < c.nrec) syn = syn + c.msP21[k] * s[2 + k];
        v = v * c.eP22 + (c.I_e + s[1]) * c.eP20 + syn;
    } else {
        r = r - 1;
    }
#pragma unroll
    for (int k = 0; k < kMaxReceptors; ++k)
        if (k < c.nrec) s[2 + k] = s[2 + k] * c.msP11[k] + w[k];
    const bool spike = v >= c.theta;
    if (spike) {
        r = c.ref_count;
        v = c.vreset;
    }
    s[0] = v + c.E_L;
    s[1] = Real(0);  // no current input on this path: i_const <- 0
    return spike;
}

// ------------------------------------------------------------- kernels

// The pieces of one neuron-step, shared by the per-step and the windowed
// engines.  Inputs of step n: the ring slot (read and cleared) plus the
// Poisson drives of the neuron's population.
template <typename Real>
__device__ __forceinline__ void step_inputs(const StepArgs<Real> &a, int g, int p,
                                            const PopCoef<Real> &c, int64_t n, Real (&in)[kMaxReceptors]) {
    const int slot = static_cast<int>(n % a.L);
    for (int ch = 0; ch < kMaxReceptors; ++ch) in[ch] = Real(0);
    for (int ch = 0; ch < a.R; ++ch) {
        Real *cell = a.ring + (static_cast<size_t>(slot) * a.R + ch) * a.N + g;
        in[ch] = *cell;
        *cell = Real(0);
    }
}
template <typename Real>
__device__ __forceinline__ void step_drives(const StepArgs<Real> &a, int g, int p,
                                            const PopCoef<Real> &c, int64_t n, Real (&in)[kMaxReceptors]) {
    for (int q = a.pop_drive_ptr[p]; q < a.pop_drive_ptr[p + 1]; ++q) {
        const DriveDev d = a.drives[a.pop_drive_list[q]];
        const int64_t se = n - d.lag;
        if (d.tmin < se && se <= d.tmax) {
            const uint64_t u = drive_draw(d, static_cast<uint32_t>(se),
                                          static_cast<uint32_t>(g - c.off));
            const int cnt = poisson_from_table(a.cdf + d.cdf_off, d.cdf_n, u);
            in[d.receptor < a.R ? d.receptor : 0] += static_cast<Real>(cnt) * static_cast<Real>(d.weight);
        }
    }
}
// the model's update of one step; returns the spike flag
template <typename Real, int MODEL>
__device__ __forceinline__ bool step_update(const StepArgs<Real> &a, const PopCoef<Real> &c, Real (&st)[8],
                                            int &r, Real (&in)[kMaxReceptors], double dt) {
    bool sp;
    if constexpr (MODEL == 0) {
        Real s6[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) s6[i] = st[i];
        sp = a.ports ? iaf_alpha_step_ports<Real>(c, s6, r, in[0], in[1])
                     : iaf_alpha_step<Real>(c, s6, r, in[0]);
#pragma unroll
        for (int i = 0; i < 6; ++i) st[i] = s6[i];
    } else if constexpr (MODEL == 1) {
        Real s6[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) s6[i] = st[i];
        sp = a.ports ? iaf_exp_step_ports<Real>(c, s6, r, in[0], in[1])
                     : iaf_exp_step<Real>(c, s6, r, in[0]);
#pragma unroll
        for (int i = 0; i < 6; ++i) st[i] = s6[i];
    } else if constexpr (MODEL == 5) {
        sp = iaf_ms_step<Real>(c, st, r, in);
    } else {
        sp = cond_step<Real, MODEL>(c, st, r, in[0], in[1], dt, a.err, a.rk_iters);
    }
    return sp;
}
// a spike of neuron g at step n into the recorder (when g is recorded)
template <typename Real>
__device__ __forceinline__ void step_record_spike(const StepArgs<Real> &a, int g, int64_t n) {
    if (a.spk_flag == nullptr || a.spk_flag[g]) {
        const unsigned long long at = atomicAdd(a.spk_count, 1ull);
        if (at < static_cast<unsigned long long>(a.spk_cap)) {
            a.spk_step[at] = n;
            a.spk_gid[at] = g;
        }
    }
}
template <typename Real>
__device__ __forceinline__ void step_record_v(const StepArgs<Real> &a, int g, int64_t n, Real v) {
    if (a.rec_slot) {
        const int rs = a.rec_slot[g];
        if (rs >= 0) a.v_out[static_cast<size_t>(n - a.run_step0) * a.n_rec + rs] = v;
    }
}

template <typename Real, int MODEL>
__global__ void __launch_bounds__(128) k_neuron_step(const StepArgs<Real> a, double dt) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.N) return;
    const int64_t n = *a.step_ptr;
    const int p = find_pop_t(a.coef, a.npop, g);
    const PopCoef<Real> c = a.coef[p];
    Real in[kMaxReceptors];
    step_inputs<Real>(a, g, p, c, n, in);
    step_drives<Real>(a, g, p, c, n, in);
    constexpr int kSlots = model_n_slots(MODEL);
    Real st[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) st[i] = i < kSlots ? a.s[i][g] : Real(0);
    int r = a.r[g];
    const bool sp = step_update<Real, MODEL>(a, c, st, r, in, dt);
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (i < kSlots) a.s[i][g] = st[i];
    a.r[g] = r;
    const int bit = static_cast<int>(n & 63);
    a.hist[g] = (a.hist[g] & ~(1ull << bit)) | (static_cast<uint64_t>(sp) << bit);
    if (sp) {
        const int pos = atomicAdd(a.step_nspk, 1);
        a.step_spk[pos] = static_cast<uint32_t>(g);
        step_record_spike<Real>(a, g, n);
    }
    step_record_v<Real>(a, g, n, st[0]);
}

// Static delivery of this step's spikes.  A work item is one chunk of
// kChunkEdges out-edges of one (spike, projection) pair, so a long row is
// spread over several warps; each lane loads its kEdgeU edge words and
// weights before the first atomic, which keeps kEdgeU loads in flight instead
// of one round trip per edge.
template <typename Real>
__global__ void __launch_bounds__(256) k_deliver_static(const StepArgs<Real> a) {
    const int64_t n = *a.step_ptr;
    const int nspk = *a.step_nspk;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int slot_n = static_cast<int>(n % a.L);
    const int C = a.static_chunks;
    const int64_t per_spike = static_cast<int64_t>(a.nproj) * C;
    for (int64_t item = warp; item < nspk * per_spike; item += nwarps) {
        const int i = static_cast<int>(item / per_spike);
        const int rem = static_cast<int>(item % per_spike);
        const int q = rem / C, chunk = rem % C;
        if (a.proj_plastic[q]) continue;
        const ProjDev<Real> &P = a.projs[q];
        const int g = static_cast<int>(a.step_spk[i]);
        const int pre_off = a.coef[P.pre_pop].off;
        if (g < pre_off || g >= pre_off + a.coef[P.pre_pop].n) continue;
        const int gl = g - pre_off;
        const int64_t beg = P.indptr[gl] + static_cast<int64_t>(chunk) * kChunkEdges;
        const int64_t end = P.indptr[gl + 1];
        if (beg >= end) continue;
        uint32_t ed[kEdgeU];
        Real w[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            const int64_t e = beg + u * 32 + lane;
            ed[u] = e < end ? __ldg(P.edges + e) : 0xFFFFFFFFu;
            w[u] = (e < end && !P.homogeneous) ? __ldg(P.w + e) : P.w0;
        }
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (ed[u] == 0xFFFFFFFFu) continue;
            const int slot = (slot_n + static_cast<int>(ed[u] >> kEdgeDelayShift)) % a.L;
            atomicAdd(a.ring + (static_cast<size_t>(slot) * a.R + P.receptor) * a.N + P.post_off +
                          (ed[u] & kEdgePostMask),
                      w[u]);
        }
    }
    // End of the step, by the last block to finish: zero the step's counters
    // (spike count, STDP list lengths; counter 1 is this arrival count) and
    // advance the device step.  Every block read the step and the spike
    // count before arriving here, and every other kernel of the step ran
    // before this one.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        int *ctr = a.step_nspk;
        if (atomicAdd(ctr + 1, 1) == static_cast<int>(gridDim.x) - 1) {
            __threadfence();
            for (int i = 0; i < a.n_counters; ++i) ctr[i] = 0;
            *a.step_ptr = n + 1;
        }
    }
}

// Weights of a plastic projection after the step that just closed
// (*step_ptr already advanced) into its row of the run's trajectory, the
// counterpart of the reference's per-step weight tap
// (_nest_network/simulator.py:1868-1880).
__global__ void k_weight_tap(const double *w, int64_t n_edges, double *wtrace,
                             const int64_t *step_ptr, int64_t run_step0) {
    const int64_t row = *step_ptr - 1 - run_step0;
    double *dst = wtrace + row * n_edges;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n_edges;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[e] = w[e];
}

// STDP 1: traces decay-then-add (event_plastic.py:390-420); lists of pres
// whose delayed spike arrives now and of posts that fired at n - 1.
__global__ void k_stdp_traces(StdpDev s, const uint64_t *hist, const int64_t *step_ptr) {
    const int64_t n = *step_ptr;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.n_pre) {
        const bool x = fired(hist, s.pre_off + i, n - s.lag);
        s.pre_trace[i] = s.pre_trace[i] * s.dec_pre + (x ? 1.0 : 0.0);
        if (s.rule == 1) s.pre_trace2[i] = s.pre_trace2[i] * s.dec_pre2 + (x ? 1.0 : 0.0);
        if (x) s.pre_list[atomicAdd(&s.counts[0], 1)] = i;
    }
    if (i < s.n_post) {
        const bool y = fired(hist, s.post_off + i, n - 1);
        s.post_trace[i] = s.post_trace[i] * s.dec_post + (y ? 1.0 : 0.0);
        if (s.rule == 1) s.post_trace2[i] = s.post_trace2[i] * s.dec_post2 + (y ? 1.0 : 0.0);
        if (y) s.post_list[atomicAdd(&s.counts[1], 1)] = i;
    }
}

// x^mu of the soft-bound terms: no pow for the additive rule (mu = 0, the
// reference kernel's fast path, _kernel/plasticity.py:548-556) or the
// multiplicative one (mu = 1, where x^1 is x)
__device__ __forceinline__ double stdp_pow(double x, double mu) {
    return mu == 1.0 ? x : (mu == 0.0 ? 1.0 : pow(x, mu));
}
// the normalised weight w / Wmax is taken as w * (1 / Wmax), the reciprocal
// formed once on the host in FP64
__device__ __forceinline__ double stdp_facilitate(const StdpDev &s, double w, double kplus) {
    const double wn = w * s.inv_Wmax;
    const double nw = wn + s.lambda_ * stdp_pow(1.0 - wn, s.mu_plus) * kplus;
    return nw < 1.0 ? nw * s.Wmax : s.Wmax;
}
__device__ __forceinline__ double stdp_depress(const StdpDev &s, double w, double kminus) {
    const double wn = w * s.inv_Wmax;
    const double nw = wn - s.alpha * s.lambda_ * stdp_pow(wn, s.mu_minus) * kminus;
    return nw > 0.0 ? nw * s.Wmax : 0.0;
}
// stdp_triplet_synapse.py:179-197: potentiation reads the fast pre trace r1
// weighted by the slow post trace o2, depression the fast post trace o1
// weighted by the slow pre trace r2 (each excluding this step's spike)
__device__ __forceinline__ double triplet_facilitate(const StdpDev &s, double w, double r1,
                                                     double o2) {
    const double nw = w + r1 * (s.a2p + s.a3p * o2);
    return nw < s.Wmax ? nw : s.Wmax;
}
__device__ __forceinline__ double triplet_depress(const StdpDev &s, double w, double o1,
                                                  double r2) {
    const double nw = w - o1 * (s.a2m + s.a3m * r2);
    return nw > 0.0 ? nw : 0.0;
}

// STDP 2: facilitation on the in-edges of posts that fired at n - 1
// (_nest_plasticity/stdp_synapse.py:163-165).  A work item is one chunk of
// kChunkEdges in-edges of one post; every lane gathers its kEdgeU pre ids,
// edge ids, pre traces and weights before the first store.  Each in-edge
// belongs to one post and each post is listed once, so no two lanes touch
// one weight.
__global__ void __launch_bounds__(256) k_stdp_facilitate(StdpDev s, const uint64_t *hist,
                                                         const int64_t *step_ptr) {
    const int64_t n = *step_ptr;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int C = s.in_chunks;
    const int64_t nitems = static_cast<int64_t>(s.counts[1]) * C;
    for (int64_t it = warp; it < nitems; it += nwarps) {
        const int j = s.post_list[it / C];
        const int64_t beg = s.cindptr[j] + (it % C) * kChunkEdges, end = s.cindptr[j + 1];
        if (beg >= end) continue;
        // the post fired at n - 1, so its own spike is 1 in every post trace
        const double o2 = s.rule == 1 ? s.post_trace2[j] - 1.0 : 0.0;
        int pre[kEdgeU];
        int64_t eid[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            const int64_t e = beg + u * 32 + lane;
            pre[u] = e < end ? static_cast<int>(s.cedges[e] & kEdgePostMask) : -1;
            eid[u] = e < end ? s.cperm[e] : 0;
        }
        double kplus[kEdgeU], w[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (pre[u] < 0) continue;
            const double x = fired(hist, s.pre_off + pre[u], n - s.lag) ? 1.0 : 0.0;
            kplus[u] = s.pre_trace[pre[u]] - x;
            w[u] = s.w[eid[u]];
        }
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (pre[u] < 0) continue;
            s.w[eid[u]] = s.rule == 1 ? triplet_facilitate(s, w[u], kplus[u], o2)
                                      : stdp_facilitate(s, w[u], kplus[u]);
        }
    }
}

// STDP 3: depression on the out-edges of pres whose delayed spike arrives
// now (stdp_synapse.py:167-169), then delivery of the updated weight into
// this step's ring slot (event_plastic.py:497-518).  Work items are chunks
// of kChunkEdges out-edges of one pre, with the loads of a lane's kEdgeU
// edges issued before its stores and atomics.
template <typename Real>
__global__ void __launch_bounds__(256) k_stdp_depress(StdpDev s, const StepArgs<Real> a) {
    const int64_t n = *a.step_ptr;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int C = s.out_chunks;
    const int64_t nitems = static_cast<int64_t>(s.counts[0]) * C;
    const int slot_n = static_cast<int>(n % a.L);
    Real *ring = a.ring + (static_cast<size_t>(slot_n) * a.R + s.receptor) * a.N + s.post_off;
    for (int64_t it = warp; it < nitems; it += nwarps) {
        const int i = s.pre_list[it / C];
        const int64_t beg = s.indptr[i] + (it % C) * kChunkEdges, end = s.indptr[i + 1];
        if (beg >= end) continue;
        // the pre's delayed spike arrives now: 1 in every pre trace
        const double r2 = s.rule == 1 ? s.pre_trace2[i] - 1.0 : 0.0;
        int post[kEdgeU];
        double w[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            const int64_t e = beg + u * 32 + lane;
            post[u] = e < end ? static_cast<int>(s.edges[e] & kEdgePostMask) : -1;
            w[u] = e < end ? s.w[e] : 0.0;
        }
        double kminus[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (post[u] < 0) continue;
            const double y = fired(a.hist, s.post_off + post[u], n - 1) ? 1.0 : 0.0;
            kminus[u] = s.post_trace[post[u]] - y;
        }
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (post[u] < 0) continue;
            const double nw = s.rule == 1 ? triplet_depress(s, w[u], kminus[u], r2)
                                          : stdp_depress(s, w[u], kminus[u]);
            s.w[beg + u * 32 + lane] = nw;
            atomicAdd(ring + post[u], static_cast<Real>(nw));
        }
    }
}

// ------------------------------------------------------ windowed engine
// A window covers the steps [n0, n0 + Wk), Wk <= W <= every lag, so a spike
// of the window arrives after it and the steps' inputs are known at its
// start, except the plastic weights, whose facilitation by the post's own
// spikes of the window must precede each arrival on the edge.  Per window:
//   pretrace: per pre of the plastic projection, the pre trace of every
//     step of the window without that step's arrival (kp, the K+ that a
//     facilitation at that step reads), and the pres whose spikes arrive;
//   arrivals: the out-edges of those pres into per-(step, post) lists;
//   neuron: each thread advances its neuron through the window; at step n
//     a plastic post updates its post trace, then for each edge arriving at
//     n applies the facilitations its own spikes of the window still owe
//     the edge (steps after the edge's last update, up to n) and the
//     depression, and adds the new weight to the step's input; the step's
//     static input comes from the ring as in the per-step engine;
//   deliver: the window's spikes into the ring slots n + lag;
//   facilitate: the facilitations owed by each post that fired in the
//     window on all its in-edges (those after each edge's last update); a
//     spike of the window's last step is facilitated in the next window, at
//     its first step, as the per-step form does.
// Every weight goes through the same operations in the same order as in
// the per-step engine (_nest_plasticity/stdp_synapse.py:163-169 per step).

__global__ void k_win_pretrace(WinDev w, const uint64_t *hist, int64_t n0, int Wk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.s.n_pre) return;
    double tr = w.s.pre_trace[i];
    uint32_t am = 0u;
    for (int k = 0; k < Wk; ++k) {
        const bool x = fired(hist, w.s.pre_off + i, n0 + k - w.s.lag);
        const double xv = x ? 1.0 : 0.0;
        const double t = tr * w.s.dec_pre + xv;
        w.kp[static_cast<size_t>(k) * w.s.n_pre + i] = t - xv;
        tr = t;
        am |= static_cast<uint32_t>(x) << k;
    }
    w.s.pre_trace[i] = tr;
    w.amask[i] = am;
    if (am) {
        const int q = atomicAdd(&w.ctr[1], 1);
        w.pre_list[q] = static_cast<uint32_t>(i);
        w.pre_list[w.s.n_pre + q] = am;
    }
}

__global__ void __launch_bounds__(256) k_win_arrivals(WinDev w) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int C = w.s.out_chunks, np = w.s.n_post;
    const int64_t nitems = static_cast<int64_t>(w.ctr[1]) * C;
    for (int64_t it = warp; it < nitems; it += nwarps) {
        const int q = static_cast<int>(it / C);
        const uint32_t i = w.pre_list[q], am = w.pre_list[w.s.n_pre + q];
        const int64_t beg = w.s.indptr[i] + (it % C) * kChunkEdges, end = w.s.indptr[i + 1];
        if (beg >= end) continue;
        int post[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            const int64_t e = beg + u * 32 + lane;
            post[u] = e < end ? static_cast<int>(w.s.edges[e] & kEdgePostMask) : -1;
        }
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (post[u] < 0) continue;
            const int64_t e = beg + u * 32 + lane;
            for (uint32_t m = am; m; m &= m - 1u) {
                const int k = __ffs(static_cast<int>(m)) - 1;
                const int pos = atomicAdd(&w.cnt[static_cast<size_t>(k) * np + post[u]], 1);
                if (pos < w.cap)
                {
                    WinArrival &en = w.arr[(static_cast<size_t>(k) * w.cap + pos) * np + post[u]];
                    en.e = static_cast<uint32_t>(e);
                    en.pre = i;
                }
                else
                    atomicExch(w.err, BSPK_DEV_ERR_OVERFLOW);
            }
        }
    }
}

// The plastic arrivals of window step k at post j (na of them), each edge
// brought up to date and stored: first the facilitations the post's spikes
// still owe it (bits of emask up to k: the spike at n0 - 1 + b is facilitated
// at n0 + b with K+ kp[b]; owed after fdone, the step of the edge's previous
// arrival in this window, or n0 - 1 when it has none, since the window before
// brought every edge there), then the depression with K- kminus; each new
// weight joins acc.  The arrivals of one step are distinct edges, so they go
// kWinArrU at a time: every load of a group is issued before its first store
// (the group's chains overlap).
template <typename Real>
__device__ __forceinline__ void win_arrivals_apply(const WinDev &w, int j, int k, int na,
                                                   uint64_t emask, double kminus, Real &acc) {
    const int np = w.s.n_post;
    const uint64_t kmask = emask & ((2ull << k) - 1ull);
    const WinArrival *ar = w.arr + static_cast<size_t>(k) * w.cap * np + j;
    for (int q0 = 0; q0 < na; q0 += kWinArrU) {
        uint32_t ee[kWinArrU], pr[kWinArrU];
#pragma unroll
        for (int u = 0; u < kWinArrU; ++u) {
            ee[u] = 0u;
            pr[u] = 0u;
            if (q0 + u < na) {
                const WinArrival en = ar[static_cast<size_t>(q0 + u) * np];
                ee[u] = en.e;
                pr[u] = en.pre;
            }
        }
        double wv[kWinArrU];
        uint64_t due[kWinArrU];
#pragma unroll
        for (int u = 0; u < kWinArrU; ++u) {
            wv[u] = 0.0;
            due[u] = 0ull;
            if (q0 + u < na) {
                wv[u] = w.s.w[ee[u]];
                // the edge's previous arrival in the window (its pre's last
                // bit below k) brought it up to date at that step
                const uint32_t prev = w.amask[pr[u]] & ((1u << k) - 1u);
                const int lo = prev ? 32 - __clz(static_cast<int>(prev)) : 0;
                due[u] = kmask & ~((1ull << lo) - 1ull);
            }
        }
        // K+ of each edge's first due facilitation, before any store
        double kp0[kWinArrU];
#pragma unroll
        for (int u = 0; u < kWinArrU; ++u) {
            kp0[u] = 0.0;
            if (due[u]) {
                const int b = __ffsll(static_cast<long long>(due[u])) - 1;
                kp0[u] = w.kp[static_cast<size_t>(b) * w.s.n_pre + pr[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kWinArrU; ++u) {
            if (q0 + u >= na) continue;
            double x = wv[u];
            uint64_t d = due[u];
            if (d) {
                x = stdp_facilitate(w.s, x, kp0[u]);
                for (d &= d - 1ull; d; d &= d - 1ull) {
                    const int b = __ffsll(static_cast<long long>(d)) - 1;
                    x = stdp_facilitate(w.s, x, w.kp[static_cast<size_t>(b) * w.s.n_pre + pr[u]]);
                }
            }
            x = stdp_depress(w.s, x, kminus);
            w.s.w[ee[u]] = x;
            acc += static_cast<Real>(x);
        }
    }
}

// Inputs of window step n = n0 + k of neuron g: the ring slot, then (a post
// of the plastic projection) the post trace of step n and the arrivals of
// step n (win_arrivals_apply), then the drives.
template <typename Real>
__device__ __forceinline__ void win_inputs(const StepArgs<Real> &a, const WinDev &w, int g, int p,
                                           const PopCoef<Real> &c, int64_t n0, int k, bool pp,
                                           int j, uint64_t prevbit, uint32_t spmask,
                                           double &post_tr, Real (&in)[kMaxReceptors]) {
    const int64_t n = n0 + k;
    step_inputs<Real>(a, g, p, c, n, in);
    if (pp) {
        const int np = w.s.n_post;
        // post trace of step n (decay, then the spike of n - 1) and the K- of
        // a depression at n (without that spike)
        const bool yb = k == 0 ? prevbit != 0 : ((spmask >> (k - 1)) & 1u) != 0;
        const double y = yb ? 1.0 : 0.0;
        const double t = post_tr * w.s.dec_post + y;
        const double kminus = t - y;
        post_tr = t;
        const size_t ci = static_cast<size_t>(k) * np + j;
        int na = w.cnt[ci];
        w.cnt[ci] = 0;  // cleared for the next window
        if (na > w.cap) na = w.cap;
        // the post's spikes at n0 - 1 + b (bit b)
        const uint64_t emask = (static_cast<uint64_t>(spmask) << 1) | prevbit;
        const int rec = w.s.receptor < a.R ? w.s.receptor : 0;
        win_arrivals_apply<Real>(w, j, k, na, emask, kminus, in[rec]);
    }
    step_drives<Real>(a, g, p, c, n, in);
}

// the bookkeeping after window step n0 + k of neuron g
template <typename Real>
__device__ __forceinline__ void win_after_step(const StepArgs<Real> &a, const WinDev &w, int g,
                                               int64_t n0, int k, bool sp, Real v,
                                               uint32_t &spmask, uint64_t &hw) {
    const int64_t n = n0 + k;
    spmask |= static_cast<uint32_t>(sp) << k;
    const int bit = static_cast<int>(n & 63);
    hw = (hw & ~(1ull << bit)) | (static_cast<uint64_t>(sp) << bit);
    if (sp) {
        const int pos = atomicAdd(&w.ctr[0], 1);
        w.spk[pos] = (static_cast<uint32_t>(g) << 5) | static_cast<uint32_t>(k);
        step_record_spike<Real>(a, g, n);
    }
    step_record_v<Real>(a, g, n, v);
}

// the end of a window for neuron g: its spike history, post trace and (a
// post that fired at n0 - 1 .. n0 + Wk - 2) its entry in the post list
template <typename Real>
__device__ __forceinline__ void win_close(const StepArgs<Real> &a, const WinDev &w, int g, bool pp, int j,
                                          int Wk, uint64_t prevbit, uint32_t spmask, uint64_t hw,
                                          double post_tr) {
    a.hist[g] = hw;
    if (pp) {
        w.s.post_trace[j] = post_tr;
        // the last step's spike is facilitated in the next window
        const uint32_t em = static_cast<uint32_t>(((static_cast<uint64_t>(spmask) << 1) | prevbit) &
                                                  ((1ull << Wk) - 1ull));
        if (em) {
            const int q = atomicAdd(&w.ctr[2], 1);
            w.post_list[q] = static_cast<uint32_t>(j);
            w.post_list[w.s.n_post + q] = em;
        }
    }
}

// Neuron pass of a window: one thread per neuron, the window's steps in order
// with all lanes of a warp at the same step (inputs, update, bookkeeping).
template <typename Real, int MODEL>
__global__ void __launch_bounds__(128) k_win_neuron(const StepArgs<Real> a, WinDev w, int64_t n0, int Wk,
                                                    double dt) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.N) return;
    const int p = find_pop_t(a.coef, a.npop, g);
    const PopCoef<Real> c = a.coef[p];
    constexpr int kSlots = model_n_slots(MODEL);
    Real st[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) st[i] = i < kSlots ? a.s[i][g] : Real(0);
    int r = a.r[g];
    const int j = g - w.s.post_off;
    const bool pp = w.on && j >= 0 && j < w.s.n_post;  // a post of the plastic projection
    double post_tr = pp ? w.s.post_trace[j] : 0.0;
    uint64_t hw = a.hist[g];
    // the spike of step n0 - 1, whose facilitation falls on step n0
    const uint64_t prevbit = (n0 >= 1 && ((hw >> ((n0 - 1) & 63)) & 1ull) != 0) ? 1ull : 0ull;
    uint32_t spmask = 0u;
    for (int k = 0; k < Wk; ++k) {
        Real in[kMaxReceptors];
        win_inputs<Real>(a, w, g, p, c, n0, k, pp, j, prevbit, spmask, post_tr, in);
        const bool sp = step_update<Real, MODEL>(a, c, st, r, in, dt);
        win_after_step<Real>(a, w, g, n0, k, sp, st[0], spmask, hw);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (i < kSlots) a.s[i][g] = st[i];
    a.r[g] = r;
    win_close<Real>(a, w, g, pp, j, Wk, prevbit, spmask, hw, post_tr);
}

// Static delivery of the window's spikes (as k_deliver_static, a spike of
// step n0 + k into the slots n0 + k + lag).
template <typename Real>
__global__ void __launch_bounds__(256) k_win_deliver(const StepArgs<Real> a, WinDev w, int64_t n0) {
    const int nspk = w.ctr[0];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int C = a.static_chunks;
    const int64_t per_spike = static_cast<int64_t>(a.nproj) * C;
    for (int64_t item = warp; item < nspk * per_spike; item += nwarps) {
        const int i = static_cast<int>(item / per_spike);
        const int rem = static_cast<int>(item % per_spike);
        const int q = rem / C, chunk = rem % C;
        if (a.proj_plastic[q]) continue;
        const ProjDev<Real> &P = a.projs[q];
        const uint32_t ent = w.spk[i];
        const int g = static_cast<int>(ent >> 5);
        const int pre_off = a.coef[P.pre_pop].off;
        if (g < pre_off || g >= pre_off + a.coef[P.pre_pop].n) continue;
        const int slot_n = static_cast<int>((n0 + static_cast<int64_t>(ent & 31u)) % a.L);
        const int gl = g - pre_off;
        const int64_t beg = P.indptr[gl] + static_cast<int64_t>(chunk) * kChunkEdges;
        const int64_t end = P.indptr[gl + 1];
        if (beg >= end) continue;
        uint32_t ed[kEdgeU];
        Real wv[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            const int64_t e = beg + u * 32 + lane;
            ed[u] = e < end ? __ldg(P.edges + e) : 0xFFFFFFFFu;
            wv[u] = (e < end && !P.homogeneous) ? __ldg(P.w + e) : P.w0;
        }
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (ed[u] == 0xFFFFFFFFu) continue;
            const int slot = (slot_n + static_cast<int>(ed[u] >> kEdgeDelayShift)) % a.L;
            atomicAdd(a.ring + (static_cast<size_t>(slot) * a.R + P.receptor) * a.N + P.post_off +
                          (ed[u] & kEdgePostMask),
                      wv[u]);
        }
    }
}

// The facilitations owed on all in-edges of the posts that fired at steps
// n0 - 1 .. n0 + Wk - 2: for a spike at n0 - 1 + b, the facilitation at step
// n0 + b (K+ kp[b]), unless an arrival of the edge at that step or later
// already covered it.  A spike of the window's last step is facilitated at the next
// window's first step, as in the per-step form.
__global__ void __launch_bounds__(256) k_win_facilitate(WinDev w) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int C = w.s.in_chunks, np = w.s.n_post;
    const int64_t nitems = static_cast<int64_t>(w.ctr[2]) * C;
    for (int64_t it = warp; it < nitems; it += nwarps) {
        const int q = static_cast<int>(it / C);
        const int j = static_cast<int>(w.post_list[q]);
        const uint64_t mask = w.post_list[np + q];
        const int64_t beg = w.s.cindptr[j] + (it % C) * kChunkEdges, end = w.s.cindptr[j + 1];
        if (beg >= end) continue;
        int pre[kEdgeU];
        int64_t eid[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            const int64_t cpos = beg + u * 32 + lane;
            pre[u] = cpos < end ? static_cast<int>(w.s.cedges[cpos] & kEdgePostMask) : -1;
            eid[u] = cpos < end ? w.s.cperm[cpos] : 0;
        }
        double wv[kEdgeU];
        uint32_t am[kEdgeU];
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (pre[u] < 0) continue;
            wv[u] = w.s.w[eid[u]];
            am[u] = w.amask[pre[u]];
        }
#pragma unroll
        for (int u = 0; u < kEdgeU; ++u) {
            if (pre[u] < 0) continue;
            // the edge's last arrival in the window brought it up to date
            const int lo = am[u] ? 32 - __clz(static_cast<int>(am[u])) : 0;
            uint64_t due = mask & ~((1ull << lo) - 1ull);
            double x = wv[u];
            for (; due; due &= due - 1ull) {
                const int b = __ffsll(static_cast<long long>(due)) - 1;
                x = stdp_facilitate(w.s, x, w.kp[static_cast<size_t>(b) * w.s.n_pre + pre[u]]);
            }
            w.s.w[eid[u]] = x;
        }
    }
}

// work items per row for rows of at most max_deg edges (at least one)
int chunks_of(int64_t max_deg) {
    const int64_t c = (max_deg + kChunkEdges - 1) / kChunkEdges;
    return c > 0 ? static_cast<int>(c) : 1;
}

template <typename Real>
StepArgs<Real> step_args(bspk_plan *p, int64_t *step_ptr) {
    StepArgs<Real> a{};
    a.N = p->N;
    a.npop = static_cast<int>(p->pops.size());
    a.nproj = static_cast<int>(p->projs.size());
    a.ndrive = static_cast<int>(p->drives.size());
    a.model = p->cfg.model;
    a.ports = p->ports_sep;
    a.R = plan_n_receptors(p);
    a.L = p->L;
    a.coef = static_cast<const PopCoef<Real> *>(p->d_coef);
    for (int i = 0; i < 8; ++i) a.s[i] = static_cast<Real *>(p->d_s[i]);
    a.r = p->d_r;
    a.ring = static_cast<Real *>(p->d_ring);
    a.projs = static_cast<const ProjDev<Real> *>(p->d_projs);
    a.proj_plastic = p->d_proj_plastic;
    a.drives = p->d_drives;
    a.pop_drive_ptr = p->d_pop_drive_ptr;
    a.pop_drive_list = p->d_pop_drive_list;
    a.cdf = p->d_cdf;
    a.hist = p->d_hist;
    a.step_spk = p->d_step_spk;
    a.step_nspk = p->d_step_counters;
    a.spk_step = p->d_spk_step;
    a.spk_gid = p->d_spk_gid;
    a.spk_count = p->d_spk_count;
    a.spk_cap = p->cfg.spike_capacity;
    a.spk_flag = p->has_spk_flag ? p->d_spk_flag : nullptr;
    a.rec_slot = p->rec_v.empty() ? nullptr : p->d_rec_slot;
    a.v_out = static_cast<Real *>(p->d_v);
    a.n_rec = static_cast<int>(p->rec_v.size());
    a.step_ptr = step_ptr;
    a.run_step0 = p->step;
    a.rk_iters = p->d_rk_iters;
    a.err = p->d_err;
    int64_t max_out = 0;
    for (const Proj &J : p->projs)
        if (!J.plastic && J.max_out > max_out) max_out = J.max_out;
    a.static_chunks = chunks_of(max_out);
    a.n_counters = p->n_step_counters;
    return a;
}

std::vector<StdpDev> stdp_descs(bspk_plan *p) {
    std::vector<StdpDev> v;
    int k = 0;
    for (auto &J : p->projs) {
        if (!J.plastic) continue;
        StdpDev s{};
        s.pre_off = p->pops[J.pre].off;
        s.post_off = p->pops[J.post].off;
        s.n_pre = p->pops[J.pre].n;
        s.n_post = p->pops[J.post].n;
        s.lag = (p->cfg.semantics == BSPK_LEGACY ? 1 : 0) + (J.delay.empty() ? 0 : J.delay[0]);
        s.receptor = J.receptor;
        s.tau_plus = J.stdp.tau_plus;
        s.tau_minus = J.stdp.tau_minus;
        s.lambda_ = J.stdp.lambda_;
        s.alpha = J.stdp.alpha;
        s.mu_plus = J.stdp.mu_plus;
        s.mu_minus = J.stdp.mu_minus;
        s.Wmax = J.stdp.Wmax;
        s.dec_pre = std::exp(-p->cfg.dt / J.stdp.tau_plus);
        s.dec_post = std::exp(-p->cfg.dt / J.stdp.tau_minus);
        s.rule = J.rule;
        s.out_chunks = chunks_of(J.max_out);
        s.in_chunks = chunks_of(J.max_in);
        if (J.rule == 1) {
            const bspk_stdp_triplet_params &t = J.trip;
            s.Wmax = t.Wmax;
            s.a2p = t.Aplus;
            s.a3p = t.Aplus_triplet;
            s.a2m = t.Aminus;
            s.a3m = t.Aminus_triplet;
            s.dec_pre = std::exp(-p->cfg.dt / t.tau_plus);
            s.dec_post = std::exp(-p->cfg.dt / t.tau_minus);
            s.dec_pre2 = std::exp(-p->cfg.dt / t.tau_plus_triplet);
            s.dec_post2 = std::exp(-p->cfg.dt / t.tau_minus_triplet);
        }
        s.inv_Wmax = 1.0 / s.Wmax;
        s.indptr = J.d_indptr;
        s.edges = J.d_edges;
        s.w = J.d_wplastic;
        s.cindptr = J.d_cindptr;
        s.cperm = J.d_cperm;
        s.cedges = J.d_cedges;
        s.pre_trace = static_cast<double *>(J.d_pre_trace);
        s.post_trace = static_cast<double *>(J.d_post_trace);
        s.pre_trace2 = J.rule == 1 ? s.pre_trace + s.n_pre : nullptr;
        s.post_trace2 = J.rule == 1 ? s.post_trace + s.n_post : nullptr;
        s.pre_list = J.d_pre_list;
        s.post_list = J.d_post_list;
        s.counts = p->d_step_counters + 2 + 2 * k;
        s.wtrace = J.rec_w ? J.d_wtrace : nullptr;
        s.n_edges = static_cast<int64_t>(J.post_local.size());
        s.run_step0 = p->step;
        v.push_back(s);
        ++k;
    }
    return v;
}

// One step: the STDP kernels of each plastic projection, the neuron update,
// then static delivery, whose last block also closes the step (counters and
// step counter), so a step is 2 + 3 n_plastic launches.
template <typename Real>
cudaError_t enqueue_step(bspk_plan *p, const StepArgs<Real> &a, const std::vector<StdpDev> &sd,
                         cudaStream_t st) {
    for (const StdpDev &s : sd) {
        const int nmax = s.n_pre > s.n_post ? s.n_pre : s.n_post;
        k_stdp_traces<<<(nmax + 255) / 256, 256, 0, st>>>(s, a.hist, a.step_ptr);
        k_stdp_facilitate<<<p->sm_count * 4, 256, 0, st>>>(s, a.hist, a.step_ptr);
        k_stdp_depress<Real><<<p->sm_count * 4, 256, 0, st>>>(s, a);
    }
    const int nb = (a.N + 127) / 128;
    const double dt = p->cfg.dt;
    if (a.model == 0) k_neuron_step<Real, 0><<<nb, 128, 0, st>>>(a, dt);
    else if (a.model == 1) k_neuron_step<Real, 1><<<nb, 128, 0, st>>>(a, dt);
    else if (a.model == 2) k_neuron_step<Real, 2><<<nb, 128, 0, st>>>(a, dt);
    else if (a.model == 3) k_neuron_step<Real, 3><<<nb, 128, 0, st>>>(a, dt);
    else if (a.model == 4) k_neuron_step<Real, 4><<<nb, 128, 0, st>>>(a, dt);
    else k_neuron_step<Real, 5><<<nb, 128, 0, st>>>(a, dt);
    k_deliver_static<Real><<<p->sm_count * 4, 256, 0, st>>>(a);
    for (const StdpDev &s : sd)
        if (s.wtrace && s.n_edges > 0)
            k_weight_tap<<<static_cast<int>(std::min<int64_t>(p->sm_count * 4, (s.n_edges + 255) / 256)),
                           256, 0, st>>>(s.w, s.n_edges, s.wtrace, a.step_ptr, s.run_step0);
    return cudaGetLastError();
}

template <typename Real>
int run_typed(bspk_plan *p, int64_t n_steps, cudaStream_t st) {
    BSPK_CUDA(cudaMemcpyAsync(p->d_step_ptr, &p->step, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    BSPK_CUDA(cudaMemsetAsync(p->d_step_counters, 0, sizeof(int) * p->n_step_counters, st));
    const StepArgs<Real> a = step_args<Real>(p, p->d_step_ptr);
    const std::vector<StdpDev> sd = stdp_descs(p);
    constexpr int64_t kChunk = 32;
    int taps = 0;
    for (const StdpDev &s : sd) taps += s.wtrace && s.n_edges > 0 ? 1 : 0;
    const int kernels_per_step = 2 + 3 * static_cast<int>(sd.size()) + taps;
    int64_t done = 0;
    if (n_steps >= kChunk) {
        // capture kChunk steps once per run (the arguments embed this run's
        // V-recording base), replay for every full chunk
        cudaGraph_t graph;
        cudaGraphExec_t exec;
        cudaStream_t cs;
        BSPK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        BSPK_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int64_t k = 0; k < kChunk && e == cudaSuccess; ++k) e = enqueue_step<Real>(p, a, sd, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            cudaStreamDestroy(cs);
            return fail(BSPK_ERR_CUDA, std::string("graph capture: ") +
                                           cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        BSPK_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        for (; done + kChunk <= n_steps; done += kChunk) BSPK_CUDA(cudaGraphLaunch(exec, st));
        BSPK_CUDA(cudaGraphExecDestroy(exec));
        BSPK_CUDA(cudaGraphDestroy(graph));
        BSPK_CUDA(cudaStreamDestroy(cs));
    }
    for (; done < n_steps; ++done) {
        cudaError_t e = enqueue_step<Real>(p, a, sd, st);
        if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
    }
    p->last_launches = n_steps * kernels_per_step;
    return BSPK_OK;
}

WinDev win_desc(bspk_plan *p, const std::vector<StdpDev> &sd) {
    WinDev w{};
    w.on = sd.empty() ? 0 : 1;
    if (w.on) w.s = sd[0];
    w.W = p->W;
    w.cap = p->win_cap;
    w.kp = p->d_win_kp;
    w.amask = p->d_win_amask;
    w.arr = p->d_win_arr;
    w.cnt = p->d_win_cnt;
    w.spk = p->d_win_spk;
    w.pre_list = p->d_win_pre;
    w.post_list = p->d_win_post;
    w.ctr = p->d_win_ctr;
    w.err = p->d_err;
    return w;
}

// The run in windows of W steps (the last one shorter), five launches each
// with a plastic projection, three without.
template <typename Real>
int run_windowed(bspk_plan *p, int64_t n_steps, cudaStream_t st) {
    const StepArgs<Real> a = step_args<Real>(p, p->d_step_ptr);
    const std::vector<StdpDev> sd = stdp_descs(p);
    const WinDev w = win_desc(p, sd);
    const double dt = p->cfg.dt;
    const int nb = (a.N + 127) / 128, eg = p->sm_count * 4;
    int64_t launches = 0;
    for (int64_t done = 0; done < n_steps;) {
        const int Wk = static_cast<int>(std::min<int64_t>(p->W, n_steps - done));
        const int64_t n0 = p->step + done;
        BSPK_CUDA(cudaMemsetAsync(w.ctr, 0, 4 * sizeof(int), st));
        if (w.on) {
            k_win_pretrace<<<(w.s.n_pre + 255) / 256, 256, 0, st>>>(w, a.hist, n0, Wk);
            k_win_arrivals<<<eg, 256, 0, st>>>(w);
            launches += 2;
        }
        switch (a.model) {
            case 0: k_win_neuron<Real, 0><<<nb, 128, 0, st>>>(a, w, n0, Wk, dt); break;
            case 1: k_win_neuron<Real, 1><<<nb, 128, 0, st>>>(a, w, n0, Wk, dt); break;
            case 2: k_win_neuron<Real, 2><<<nb, 128, 0, st>>>(a, w, n0, Wk, dt); break;
            case 3: k_win_neuron<Real, 3><<<nb, 128, 0, st>>>(a, w, n0, Wk, dt); break;
            case 4: k_win_neuron<Real, 4><<<nb, 128, 0, st>>>(a, w, n0, Wk, dt); break;
            default: k_win_neuron<Real, 5><<<nb, 128, 0, st>>>(a, w, n0, Wk, dt); break;
        }
        k_win_deliver<Real><<<eg, 256, 0, st>>>(a, w, n0);
        launches += 2;
        if (w.on) {
            k_win_facilitate<<<eg, 256, 0, st>>>(w);
            ++launches;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("window launch: ") + cudaGetErrorString(e));
        done += Wk;
    }
    p->last_launches = launches;
    return BSPK_OK;
}

}  // namespace

int run_per_step(bspk_plan *p, int64_t n_steps, cudaStream_t st) {
    // weight recording taps every step: the per-step form
    bool taps = false;
    for (const auto &J : p->projs) taps = taps || (J.plastic && J.rec_w);
    if (p->win && !taps)
        return p->cfg.precision == 64 ? run_windowed<double>(p, n_steps, st)
                                      : run_windowed<float>(p, n_steps, st);
    return p->cfg.precision == 64 ? run_typed<double>(p, n_steps, st)
                                  : run_typed<float>(p, n_steps, st);
}

}  // namespace bspk
