// adjoint.cu -- hand-written surrogate-gradient BPTT for a recurrent
// iaf_psc_exp network: forward with checkpoints every K steps, backward by
// segment recomputation + adjoint sweep.  Compiled with -fmad=false: every
// multiply and add is rounded separately, in the order of the float64
// restatement, so the FP64 build reproduces it bit for bit.
//
// Semantics (see the restatement for the derivation):
//   forward   NEST iaf_psc_exp step (_nest_neuron/iaf_psc_exp.py:552-682), the
//             summed input x sign-split into the two synaptic currents;
//             spikes allowed when not refractory at the start of the step;
//   backward  count_ste surrogate (_kernel/spiking.py:65-88) with the soft
//             reset path d_spike * (V_reset - V) (SpikeRule._jump,
//             _kernel/spiking.py:449-466) unless detach_reset; relaxed mode
//             (_check_relaxed, :422-447) emits the surrogate primitive;
//   surrogate fast sigmoid as a smooth step: s(m) = (1 + b m / (1 + b|m|)) / 2,
//             s'(m) = (b / 2) / (1 + b|m|)^2, m = V - V_th, b = slope (1/mV);
//   loss      mean over (trial, step, readout) of (z - y)^2 with the readout
//             rate z_t = alpha z_{t-1} + c s_t (rate_mse,
//             _kernel/learn/bptt.py:142-214), episodes as BPTT._episode
//             (_kernel/learn/bptt.py:437-491) with checkpoint-every-K.
//
// Layout: one CTA per trial, state and adjoint state in shared memory (one
// neuron per thread when N <= blockDim), W row-major over post neurons (CSR
// of in-edges) for the forward gather and the weight gradient, and its
// pre-major transpose (out-edges) for the adjoint of the recurrent input.
// Per-trial gradient buffers are summed over trials in trial order by a
// final kernel, so the result does not depend on scheduling.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "../../../include/bspk.h"
#include "plan_internal.h"
#include "umma.h"

namespace bspk {

namespace {

constexpr int kAdjUnroll = 8;   // edge loads in flight per thread

// Edges are kept in a padded column-major ("ELL") layout so that the
// threads of a warp, one post (or pre) neuron each, touch consecutive words:
// in-edge k of post i at [k][N] + i (k < deg_in[i]), out-edge k of pre p at
// [k][N] + p.  The weights of the caller's CSR are packed into it at every
// forward; per-trial weight gradients live in the same layout and are
// unpacked to CSR order by the final reduction.
template <typename Real>
struct AdjArgs {
    int N, NI, B, T, K, R, relaxed, detach, nseg, ref;
    Real eP22, eP21ex, eP21in, eP20, eP11ex, eP11in, I_e, theta, vr, alpha, cz, inv, beta, halfbeta;
    const int *deg_in, *deg_out;
    const int32_t *in_col;    // [din_max][N] pre of in-edge k of post i
    const int32_t *out_post;  // [dout_max][N] post of out-edge k of pre p
    const Real *w_ie;         // [din_max][N] packed weights, in-edge order
    const Real *w_oe;         // [dout_max][N] packed weights, out-edge order
    const Real *win_t;        // [NI][N] input weights, channel-major
    const uint8_t *inputs;  // [T][B][NI]
    const Real *targets;    // [T][B][R]
    // checkpoints [nseg][B][...]
    Real *ck_V, *ck_Ie, *ck_Ii, *ck_s, *ck_z;
    int *ck_r;
    // per-trial trace of one segment [B][K][N] (z: [B][K][R])
    Real *tr_x, *tr_vt, *tr_s, *tr_z;
    uint8_t *tr_a;
    Real *dwb, *dwib;        // per-trial gradients [B][din_max][N], [B][NI][N]
    double *loss_b;          // per-trial loss sums [B]
    unsigned long long *nspk;
    int64_t din_stride;      // din_max * N
    int split;               // CTAs per trial: 1, or 2 as a thread-block cluster
    // contraction mode (gemm = 1): the backward stores the input adjoint
    // gD[t][b][i] and the recompute the previous step's spikes
    // gS[t][b][p] = s_{t-1}[b][p] (row 0 stays zero); the weight gradients
    // are then two dense contractions over (t, b) instead of per-trial
    // read-modify-writes
    Real *gD, *gS;
    int gemm;
};

// A trial's CTA (1 or 2 per trial).  With split = 2 the two CTAs of a
// cluster own the neurons [lo, hi) and [hi, N) of one trial; each keeps the
// full spike and adjoint vectors in its shared memory and writes its half
// of each new vector into its peer's copy too, between two cluster barriers.
struct Part {
    int b, rank, lo, hi;
};
template <typename Real>
__device__ __forceinline__ Part part_of(const AdjArgs<Real> &a) {
    Part q;
    q.b = blockIdx.x / a.split;
    q.rank = blockIdx.x % a.split;
    q.lo = static_cast<int>(static_cast<int64_t>(a.N) * q.rank / a.split);
    q.hi = static_cast<int>(static_cast<int64_t>(a.N) * (q.rank + 1) / a.split);
    return q;
}
// barrier over the trial's CTAs
template <typename Real>
__device__ __forceinline__ void trial_sync(const AdjArgs<Real> &a) {
    if (a.split > 1) cooperative_groups::this_cluster().sync();
    else __syncthreads();
}
// dst[i] = src[i] for the part's neurons, in this CTA and (split = 2) in the
// peer's copy of dst; callers bracket it with trial_sync
template <typename Real>
__device__ __forceinline__ void publish(const AdjArgs<Real> &a, const Part &q, Real *dst,
                                        const Real *src) {
    Real *peer = dst;
    if (a.split > 1) peer = cooperative_groups::this_cluster().map_shared_rank(dst, q.rank ^ 1);
    for (int i = q.lo + threadIdx.x; i < q.hi; i += blockDim.x) {
        const Real v = src[i];
        dst[i] = v;
        if (a.split > 1) peer[i] = v;
    }
}

template <typename Real>
struct Smem {
    Real *V, *Ie, *Ii, *sp, *sc, *lV, *lIe, *lIi, *lxn, *lxc, *ls, *z, *g;
    int *r;
    double *acc;
    int *act;   // active inputs of the step, ascending
    int *u;     // their counts
};

template <typename Real>
__device__ Smem<Real> carve(unsigned char *raw, int N, int R, int NI) {
    Smem<Real> s;
    Real *p = reinterpret_cast<Real *>(raw);
    s.V = p; p += N;
    s.Ie = p; p += N;
    s.Ii = p; p += N;
    s.sp = p; p += N;
    s.sc = p; p += N;
    s.lV = p; p += N;
    s.lIe = p; p += N;
    s.lIi = p; p += N;
    s.lxn = p; p += N;
    s.lxc = p; p += N;
    s.ls = p; p += N;
    s.z = p; p += R;
    s.g = p; p += R;
    double *d = reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(p) + 7) & ~uintptr_t(7));
    s.acc = d; d += R;
    int *q = reinterpret_cast<int *>(d);
    s.r = q; q += N;
    s.act = q; q += NI + 1;
    s.u = q; q += NI;
    return s;
}

size_t adj_smem_bytes(int N, int R, int NI, size_t real) {
    return real * (11 * static_cast<size_t>(N) + 2 * R) + 8 + 8 * static_cast<size_t>(R) +
           4 * (static_cast<size_t>(N) + 2 * NI + 1) + 16;
}

// Active inputs of (t, b) in ascending channel order: s.act[0..n), s.act[NI] = n.
template <typename Real>
__device__ void gather_inputs(const AdjArgs<Real> &a, const Smem<Real> &s, int t, int b) {
    const uint8_t *u = a.inputs + (static_cast<size_t>(t) * a.B + b) * a.NI;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int n = 0;
        for (int k0 = 0; k0 < a.NI; k0 += 32) {
            const int k = k0 + lane;
            const int cnt = k < a.NI ? static_cast<int>(u[k]) : 0;
            const unsigned m = __ballot_sync(0xffffffffu, cnt != 0);
            if (cnt != 0) {
                const int pos = n + __popc(m & ((1u << lane) - 1u));
                s.act[pos] = k;
                s.u[pos] = cnt;
            }
            n += __popc(m);
        }
        if (lane == 0) s.act[a.NI] = n;
    }
}

// One forward step of trial b at step t from shared-memory state; spikes of
// step t - 1 in s.sp (has_prev), spikes of step t into s.sc.  With a trace
// pointer set, the step's x, V before the spike test, spike and the
// not-refractory flag are stored at trace row `row`.
template <typename Real>
__device__ void forward_step(const AdjArgs<Real> &a, const Smem<Real> &s, int t, const Part &q,
                             bool has_prev, bool trace, int row, unsigned &nsp) {
    const int N = a.N, NI = a.NI, b = q.b;
    const int nact = s.act[NI];
    for (int i = q.lo + threadIdx.x; i < q.hi; i += blockDim.x) {
        Real x = Real(0);
        if (has_prev) {
            // zero spikes add nothing: skipping them leaves every rounding unchanged
            const int d = a.deg_in[i];
            for (int k = 0; k < d; ++k) {
                const size_t o = static_cast<size_t>(k) * N + i;
                const Real sv = s.sp[__ldg(a.in_col + o)];
                if (sv != Real(0)) x = x + __ldg(a.w_ie + o) * sv;
            }
        }
        for (int q = 0; q < nact; ++q)
            x = x + __ldg(a.win_t + static_cast<size_t>(s.act[q]) * N + i) * static_cast<Real>(s.u[q]);
        const bool nr = s.r[i] == 0;
        Real Vt = s.V[i];
        if (nr) Vt = s.V[i] * a.eP22 + s.Ie[i] * a.eP21ex + s.Ii[i] * a.eP21in + a.I_e * a.eP20;
        else s.r[i] = s.r[i] - 1;
        const Real ie = s.Ie[i] * a.eP11ex, ii = s.Ii[i] * a.eP11in;
        const Real wex = x > Real(0) ? x : Real(0), win = x < Real(0) ? x : Real(0);
        s.Ie[i] = ie + wex;
        s.Ii[i] = ii + win;
        const bool hard = nr && Vt >= a.theta;
        Real sv;
        if (a.relaxed) {
            if (nr) {
                const Real m = Vt - a.theta;
                const Real q = Real(1) + a.beta * fabs(m);
                sv = Real(0.5) * (Real(1) + (a.beta * m) / q);
            } else {
                sv = Real(0);
            }
            s.V[i] = Vt + sv * (a.vr - Vt);
        } else {
            sv = hard ? Real(1) : Real(0);
            s.V[i] = hard ? a.vr : Vt;
        }
        if (hard) {
            s.r[i] = a.ref;
            ++nsp;
        }
        s.sc[i] = sv;
        if (trace && a.gemm && t + 1 < a.T) a.gS[(static_cast<size_t>(t + 1) * a.B + b) * N + i] = sv;
        if (trace) {
            const size_t o = (static_cast<size_t>(b) * a.K + row) * N + i;
            a.tr_x[o] = x;
            a.tr_vt[o] = Vt;
            a.tr_s[o] = sv;
            a.tr_a[o] = nr ? 1 : 0;
        }
    }
}

template <typename Real>
__device__ void load_checkpoint(const AdjArgs<Real> &a, const Smem<Real> &s, int seg, const Part &q) {
    const size_t o = (static_cast<size_t>(seg) * a.B + q.b) * a.N;
    for (int i = q.lo + threadIdx.x; i < q.hi; i += blockDim.x) {
        s.V[i] = a.ck_V[o + i];
        s.Ie[i] = a.ck_Ie[o + i];
        s.Ii[i] = a.ck_Ii[o + i];
        s.r[i] = a.ck_r[o + i];
    }
    // the whole spike vector: the recurrent gather reads every pre
    for (int i = threadIdx.x; i < a.N; i += blockDim.x) s.sp[i] = a.ck_s[o + i];
    const int b = q.b;
    const size_t oz = (static_cast<size_t>(seg) * a.B + b) * a.R;
    for (int j = threadIdx.x; j < a.R; j += blockDim.x) s.z[j] = a.ck_z[oz + j];
}

template <typename Real>
__device__ void store_checkpoint(const AdjArgs<Real> &a, const Smem<Real> &s, int seg, const Part &q) {
    const int b = q.b;
    const size_t o = (static_cast<size_t>(seg) * a.B + b) * a.N;
    for (int i = q.lo + threadIdx.x; i < q.hi; i += blockDim.x) {
        a.ck_V[o + i] = s.V[i];
        a.ck_Ie[o + i] = s.Ie[i];
        a.ck_Ii[o + i] = s.Ii[i];
        a.ck_r[o + i] = s.r[i];
        a.ck_s[o + i] = s.sp[i];
    }
    const size_t oz = (static_cast<size_t>(seg) * a.B + b) * a.R;
    if (q.rank == 0)  // the readouts (neurons 0..R-1) belong to the first part
        for (int j = threadIdx.x; j < a.R; j += blockDim.x) a.ck_z[oz + j] = s.z[j];
}

template <typename Real>
__global__ void __launch_bounds__(1024) k_adj_forward(const AdjArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char raw[];
    const Smem<Real> s = carve<Real>(raw, a.N, a.R, a.NI);
    const Part q = part_of(a);
    const int b = q.b;
    for (int i = threadIdx.x; i < a.N; i += blockDim.x) {
        s.V[i] = Real(0);
        s.Ie[i] = Real(0);
        s.Ii[i] = Real(0);
        s.r[i] = 0;
        s.sp[i] = Real(0);
    }
    for (int j = threadIdx.x; j < a.R; j += blockDim.x) {
        s.z[j] = Real(0);
        s.acc[j] = 0.0;
    }
    unsigned nsp = 0;
    trial_sync(a);
    for (int t = 0; t < a.T; ++t) {
        if (t % a.K == 0) store_checkpoint(a, s, t / a.K, q);
        gather_inputs(a, s, t, b);
        __syncthreads();
        forward_step(a, s, t, q, t > 0, false, 0, nsp);
        trial_sync(a);  // every read of step t - 1's spikes is done
        if (q.rank == 0) {
            const Real *y = a.targets + (static_cast<size_t>(t) * a.B + b) * a.R;
            for (int j = threadIdx.x; j < a.R; j += blockDim.x) {
                s.z[j] = s.z[j] * a.alpha + a.cz * s.sc[j];
                const double d = static_cast<double>(s.z[j] - y[j]);
                s.acc[j] = s.acc[j] + d * d;
            }
        }
        publish(a, q, s.sp, s.sc);
        trial_sync(a);
    }
    if (q.rank == 0 && threadIdx.x == 0) {
        double lb = 0.0;
        for (int j = 0; j < a.R; ++j) lb = lb + s.acc[j];
        a.loss_b[b] = lb;
    }
    if (a.nspk) {
        for (int o = 16; o > 0; o >>= 1) nsp += __shfl_xor_sync(0xffffffffu, nsp, o);
        if ((threadIdx.x & 31) == 0 && nsp) atomicAdd(a.nspk, static_cast<unsigned long long>(nsp));
    }
}

template <typename Real>
__global__ void __launch_bounds__(1024) k_adj_backward(const AdjArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char raw[];
    const Smem<Real> s = carve<Real>(raw, a.N, a.R, a.NI);
    const Part q = part_of(a);
    const int b = q.b, N = a.N, NI = a.NI;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        s.lV[i] = Real(0);
        s.lIe[i] = Real(0);
        s.lIi[i] = Real(0);
        s.lxn[i] = Real(0);
    }
    for (int j = threadIdx.x; j < a.R; j += blockDim.x) s.g[j] = Real(0);
    Real *dwb = a.dwb + static_cast<size_t>(b) * a.din_stride;
    Real *dwib = a.dwib + static_cast<size_t>(b) * N * NI;
    unsigned nsp_unused = 0;
    for (int seg = a.nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * a.K, t1 = min(a.T, t0 + a.K);
        // 1. recompute the segment from its checkpoint, keeping the trace
        trial_sync(a);
        load_checkpoint(a, s, seg, q);
        trial_sync(a);
        for (int t = t0; t < t1; ++t) {
            gather_inputs(a, s, t, b);
            __syncthreads();
            forward_step(a, s, t, q, t > 0, true, t - t0, nsp_unused);
            trial_sync(a);  // every read of step t - 1's spikes is done
            if (q.rank == 0) {
                const size_t oz = (static_cast<size_t>(b) * a.K + (t - t0)) * a.R;
                for (int j = threadIdx.x; j < a.R; j += blockDim.x) {
                    s.z[j] = s.z[j] * a.alpha + a.cz * s.sc[j];
                    a.tr_z[oz + j] = s.z[j];
                }
            }
            publish(a, q, s.sp, s.sc);
            trial_sync(a);  // the trace rows of both parts are written too
        }
        // 2. adjoint sweep over the segment, last step first
        for (int t = t1 - 1; t >= t0; --t) {
            const int row = t - t0;
            const Real *y = a.targets + (static_cast<size_t>(t) * a.B + b) * a.R;
            const size_t oz = (static_cast<size_t>(b) * a.K + row) * a.R;
            if (q.rank == 0)
                for (int j = threadIdx.x; j < a.R; j += blockDim.x)
                    s.g[j] = (a.tr_z[oz + j] - y[j]) * a.inv + a.alpha * s.g[j];
            gather_inputs(a, s, t, b);
            // spikes of step t - 1 (for the weight gradient) into s.sp
            if (t > 0) {
                const Real *src = row > 0 ? a.tr_s + (static_cast<size_t>(b) * a.K + row - 1) * N
                                          : a.ck_s + (static_cast<size_t>(seg) * a.B + b) * N;
                for (int i = threadIdx.x; i < N; i += blockDim.x) s.sp[i] = src[i];
            }
            __syncthreads();
            for (int p = q.lo + threadIdx.x; p < q.hi; p += blockDim.x) {
                Real l = p < a.R ? a.cz * s.g[p] : Real(0);
                const int d = a.deg_out[p];
                for (int k0 = 0; k0 < d; k0 += kAdjUnroll) {
                    int post[kAdjUnroll];
                    Real wv[kAdjUnroll];
#pragma unroll
                    for (int u = 0; u < kAdjUnroll; ++u) {
                        const int k = k0 + u;
                        const size_t o = static_cast<size_t>(k) * N + p;
                        post[u] = k < d ? __ldg(a.out_post + o) : -1;
                        wv[u] = k < d ? __ldg(a.w_oe + o) : Real(0);
                    }
#pragma unroll
                    for (int u = 0; u < kAdjUnroll; ++u)
                        if (post[u] >= 0) l = l + wv[u] * s.lxn[post[u]];
                }
                s.ls[p] = l;
            }
            __syncthreads();
            const int nact = s.act[NI];
            for (int i = q.lo + threadIdx.x; i < q.hi; i += blockDim.x) {
                const size_t o = (static_cast<size_t>(b) * a.K + row) * N + i;
                const bool nr = a.tr_a[o] != 0;
                const Real Vt = a.tr_vt[o], sv = a.tr_s[o];
                const Real m = Vt - a.theta;
                Real sg = Real(0);
                if (nr) {
                    const Real q = Real(1) + a.beta * fabs(m);
                    sg = a.halfbeta / (q * q);
                }
                const Real cross = a.detach ? Real(0) : s.lV[i] * (a.vr - Vt);
                const Real lVt = s.lV[i] * (Real(1) - sv) + (s.ls[i] + cross) * sg;
                const Real lx = a.tr_x[o] >= Real(0) ? s.lIe[i] : s.lIi[i];
                s.lIe[i] = s.lIe[i] * a.eP11ex + (nr ? lVt * a.eP21ex : Real(0));
                s.lIi[i] = s.lIi[i] * a.eP11in + (nr ? lVt * a.eP21in : Real(0));
                s.lV[i] = nr ? lVt * a.eP22 : lVt;
                s.lxc[i] = lx;
                if (a.gemm) {
                    a.gD[(static_cast<size_t>(t) * a.B + b) * N + i] = lx;
                } else if (t > 0) {
                    const int d = a.deg_in[i];
                    for (int k0 = 0; k0 < d; k0 += kAdjUnroll) {
                        int col[kAdjUnroll];
#pragma unroll
                        for (int u = 0; u < kAdjUnroll; ++u) {
                            const int k = k0 + u;
                            col[u] = k < d ? __ldg(a.in_col + static_cast<size_t>(k) * N + i) : -1;
                        }
                        // the read-modify-writes of one batch: all loads
                        // first, then all stores (one L2 round trip, not one
                        // per spiking pre); each edge still accumulates in
                        // time order
                        Real spre[kAdjUnroll], old[kAdjUnroll];
#pragma unroll
                        for (int u = 0; u < kAdjUnroll; ++u)
                            spre[u] = col[u] >= 0 ? s.sp[col[u]] : Real(0);
#pragma unroll
                        for (int u = 0; u < kAdjUnroll; ++u)
                            old[u] = spre[u] != Real(0) ? dwb[static_cast<size_t>(k0 + u) * N + i]
                                                        : Real(0);
#pragma unroll
                        for (int u = 0; u < kAdjUnroll; ++u)
                            if (spre[u] != Real(0))
                                dwb[static_cast<size_t>(k0 + u) * N + i] = old[u] + lx * spre[u];
                    }
                }
                for (int q0 = 0; q0 < (a.gemm ? 0 : nact); q0 += kAdjUnroll) {
                    Real old[kAdjUnroll];
#pragma unroll
                    for (int u = 0; u < kAdjUnroll; ++u)
                        old[u] = q0 + u < nact ? dwib[static_cast<size_t>(s.act[q0 + u]) * N + i]
                                               : Real(0);
#pragma unroll
                    for (int u = 0; u < kAdjUnroll; ++u)
                        if (q0 + u < nact)
                            dwib[static_cast<size_t>(s.act[q0 + u]) * N + i] =
                                old[u] + lx * static_cast<Real>(s.u[q0 + u]);
                }
            }
            trial_sync(a);  // every read of the previous lxn is done
            publish(a, q, s.lxn, s.lxc);
            trial_sync(a);
        }
    }
}

// Sum over trials in trial order (deterministic): out[e] = sum_b part[b][pos[e]].
template <typename Real>
__global__ void k_adj_reduce(const Real *part, int64_t stride, const int64_t *pos, int64_t n,
                             int B, Real *out) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t q = pos[e];
        Real acc = Real(0);
        for (int b = 0; b < B; ++b) acc = acc + part[static_cast<size_t>(b) * stride + q];
        out[e] = acc;
    }
}

// Input gradient: out[i * NI + k] = sum_b part[b][k][i].
template <typename Real>
__global__ void k_adj_reduce_in(const Real *part, int N, int NI, int B, Real *out) {
    const int64_t n = static_cast<int64_t>(N) * NI;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(e / NI), k = static_cast<int>(e - static_cast<int64_t>(i) * NI);
        Real acc = Real(0);
        for (int b = 0; b < B; ++b) acc = acc + part[(static_cast<size_t>(b) * NI + k) * N + i];
        out[e] = acc;
    }
}

// The FP32 weight-gradient contractions run on the tensor cores
// (umma_gemm.cu); these two kernels add their split-K partial sums in a fixed
// order.
// out[e] = sum over z in order of part[z][post(e)][pre(e)], the caller's CSR edges
__global__ void k_gemm_gather(const float *part, int S, int Nc, size_t MN, const int32_t *e_post,
                              const int32_t *e_pre, int64_t nnz, float *out) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < nnz;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const size_t q = static_cast<size_t>(e_post[e]) * Nc + e_pre[e];
        float acc = 0.f;
        for (int z = 0; z < S; ++z) acc = acc + part[z * MN + q];
        out[e] = acc;
    }
}

// out[q] = sum over z in order of part[z][q]
__global__ void k_gemm_sum(const float *part, int S, size_t n, float *out) {
    for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n;
         q += static_cast<size_t>(gridDim.x) * blockDim.x) {
        float acc = 0.f;
        for (int z = 0; z < S; ++z) acc = acc + part[z * n + q];
        out[q] = acc;
    }
}

// Pack the caller's CSR weights and input weights into the edge layout.
template <typename Real>
__global__ void k_adj_pack(const Real *w, const Real *w_in, const int64_t *ie_eid, int64_t n_ie,
                           const int64_t *oe_eid, int64_t n_oe, int N, int NI, Real *w_ie,
                           Real *w_oe, Real *win_t) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t t0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    for (int64_t q = t0; q < n_ie; q += stride) w_ie[q] = ie_eid[q] >= 0 ? w[ie_eid[q]] : Real(0);
    for (int64_t q = t0; q < n_oe; q += stride) w_oe[q] = oe_eid[q] >= 0 ? w[oe_eid[q]] : Real(0);
    const int64_t ni = static_cast<int64_t>(N) * NI;
    for (int64_t q = t0; q < ni; q += stride) {
        const int k = static_cast<int>(q / N), i = static_cast<int>(q - static_cast<int64_t>(k) * N);
        win_t[q] = w_in[static_cast<size_t>(i) * NI + k];
    }
}

__global__ void k_adj_loss(const double *loss_b, int B, double denom, double *loss) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double tot = 0.0;
        for (int b = 0; b < B; ++b) tot = tot + loss_b[b];
        *loss = tot / denom;
    }
}

}  // namespace

}  // namespace bspk

using namespace bspk;

struct bspk_adjoint {
    bspk_adjoint_config cfg{};
    int elt = 4, nseg = 0, threads = 0, din_max = 0, dout_max = 0;
    int split = 1;  // CTAs per trial (2: a thread-block cluster per trial)
    int64_t nnz = 0;
    size_t smem = 0;
    std::vector<void *> allocs;
    int *deg_in = nullptr, *deg_out = nullptr;
    int32_t *in_col = nullptr, *out_post = nullptr;
    int64_t *ie_eid = nullptr, *oe_eid = nullptr, *in_pos = nullptr;
    void *w_ie = nullptr, *w_oe = nullptr, *win_t = nullptr;
    void *ck_V = nullptr, *ck_Ie = nullptr, *ck_Ii = nullptr, *ck_s = nullptr, *ck_z = nullptr;
    int *ck_r = nullptr;
    void *tr_x = nullptr, *tr_vt = nullptr, *tr_s = nullptr, *tr_z = nullptr;
    uint8_t *tr_a = nullptr;
    void *dwb = nullptr, *dwib = nullptr;
    double *loss_b = nullptr;
    double *loss_dev = nullptr;  // the loss when the caller passes none
    unsigned long long *nspk = nullptr;
    double coef[16] = {};
    const void *targets = nullptr;  // operands of the last forward (borrowed)
    const uint8_t *inputs = nullptr;
    bool have_forward = false;
    // FP32 weight-gradient contraction: buffers allocated (can), selected (gemm)
    int can_gemm = 0, gemm = 0, sms = 0;
    void *gD = nullptr, *gS = nullptr;   // [n_steps][batch][n]
    float *gpart = nullptr;              // split-K partial sums
    int32_t *e_post = nullptr, *e_pre = nullptr;  // the CSR edges' (post, pre)
    __nv_bfloat16 *ux = nullptr, *uy = nullptr;   // packed bf16 operand parts
    int *d_err = nullptr;                         // device error flag (bounded waits)
};

extern "C" int bspk_adjoint_sizes(const bspk_adjoint *adj, int64_t *nnz, int64_t *n_w_in,
                                  int *precision) {
    if (!adj) return bspk::fail(BSPK_ERR_ARG, "null handle");
    if (nnz) *nnz = adj->nnz;
    if (n_w_in) *n_w_in = static_cast<int64_t>(adj->cfg.n) * adj->cfg.n_in;
    if (precision) *precision = adj->cfg.precision;
    return BSPK_OK;
}

namespace {

int aalloc(bspk_adjoint *h, void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    h->allocs.push_back(*p);
    return BSPK_OK;
}

int grid_of(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096))); }

template <typename Real>
AdjArgs<Real> make_args(const bspk_adjoint *h) {
    const bspk_adjoint_config &c = h->cfg;
    AdjArgs<Real> a{};
    a.N = c.n;
    a.NI = c.n_in;
    a.B = c.batch;
    a.T = c.n_steps;
    a.K = c.ckpt_every;
    a.R = c.n_readout;
    a.relaxed = c.relaxed;
    a.detach = c.detach_reset;
    a.nseg = h->nseg;
    a.ref = static_cast<int>(h->coef[15]);
    Real *cf[14] = {&a.eP22, &a.eP21ex, &a.eP21in, &a.eP20, &a.eP11ex, &a.eP11in, &a.I_e,
                    &a.theta, &a.vr, &a.alpha, &a.cz, &a.inv, &a.beta, &a.halfbeta};
    for (int i = 0; i < 14; ++i) *cf[i] = static_cast<Real>(h->coef[i]);
    a.deg_in = h->deg_in;
    a.deg_out = h->deg_out;
    a.in_col = h->in_col;
    a.out_post = h->out_post;
    a.w_ie = static_cast<const Real *>(h->w_ie);
    a.w_oe = static_cast<const Real *>(h->w_oe);
    a.win_t = static_cast<const Real *>(h->win_t);
    a.inputs = h->inputs;
    a.targets = static_cast<const Real *>(h->targets);
    a.ck_V = static_cast<Real *>(h->ck_V);
    a.ck_Ie = static_cast<Real *>(h->ck_Ie);
    a.ck_Ii = static_cast<Real *>(h->ck_Ii);
    a.ck_s = static_cast<Real *>(h->ck_s);
    a.ck_z = static_cast<Real *>(h->ck_z);
    a.ck_r = h->ck_r;
    a.tr_x = static_cast<Real *>(h->tr_x);
    a.tr_vt = static_cast<Real *>(h->tr_vt);
    a.tr_s = static_cast<Real *>(h->tr_s);
    a.tr_z = static_cast<Real *>(h->tr_z);
    a.tr_a = h->tr_a;
    a.dwb = static_cast<Real *>(h->dwb);
    a.dwib = static_cast<Real *>(h->dwib);
    a.loss_b = h->loss_b;
    a.nspk = h->nspk;
    a.din_stride = static_cast<int64_t>(h->din_max) * c.n;
    a.split = h->split;
    a.gD = static_cast<Real *>(h->gD);
    a.gS = static_cast<Real *>(h->gS);
    a.gemm = h->gemm;
    return a;
}

// One CTA per trial, or (split = 2) a cluster of two CTAs per trial.
template <typename Real>
cudaError_t launch_trials(void (*kernel)(AdjArgs<Real>), const AdjArgs<Real> &a,
                          const bspk_adjoint *h, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(h->cfg.batch * h->split));
    cfg.blockDim = dim3(static_cast<unsigned>(h->threads));
    cfg.dynamicSmemBytes = h->smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(h->split);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, a);
}

template <typename Real>
int set_smem(bspk_adjoint *h) {
    BSPK_CUDA(cudaFuncSetAttribute(k_adj_forward<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(h->smem)));
    BSPK_CUDA(cudaFuncSetAttribute(k_adj_backward<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(h->smem)));
    return BSPK_OK;
}

template <typename Real>
int run_forward(bspk_adjoint *h, const void *w, const void *w_in, double *loss, int64_t *n_spikes,
                cudaStream_t st) {
    const bspk_adjoint_config &c = h->cfg;
    const int64_t n_ie = static_cast<int64_t>(h->din_max) * c.n;
    const int64_t n_oe = static_cast<int64_t>(h->dout_max) * c.n;
    const int64_t ni = static_cast<int64_t>(c.n) * c.n_in;
    k_adj_pack<Real><<<grid_of(std::max(std::max(n_ie, n_oe), ni)), 256, 0, st>>>(
        static_cast<const Real *>(w), static_cast<const Real *>(w_in), h->ie_eid, n_ie, h->oe_eid,
        n_oe, c.n, c.n_in, static_cast<Real *>(h->w_ie), static_cast<Real *>(h->w_oe),
        static_cast<Real *>(h->win_t));
    BSPK_CUDA(cudaGetLastError());
    const AdjArgs<Real> a = make_args<Real>(h);
    BSPK_CUDA(cudaMemsetAsync(h->nspk, 0, sizeof(unsigned long long), st));
    BSPK_CUDA(launch_trials<Real>(k_adj_forward<Real>, a, h, st));
    const double denom = static_cast<double>(c.batch) * c.n_steps * c.n_readout;
    k_adj_loss<<<1, 32, 0, st>>>(h->loss_b, c.batch, denom, loss);
    BSPK_CUDA(cudaGetLastError());
    if (n_spikes)
        BSPK_CUDA(cudaMemcpyAsync(n_spikes, h->nspk, sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    return BSPK_OK;
}

// dL/dw and dL/dw_in of an FP32 handle by contraction over (step, trial) on
// the tensor cores: the adjoints split into 3 bf16 parts, the spikes into 1
// (0/1 values, exact) or 2 (the relaxed forward's surrogate values), the
// input counts into 1 (exact)
int run_contractions(bspk_adjoint *h, float *dw, float *dw_in, cudaStream_t st) {
    const bspk_adjoint_config &c = h->cfg;
    const int N = c.n, NI = c.n_in;
    const int64_t K = static_cast<int64_t>(c.n_steps) * c.batch;
    BSPK_CUDA(umma_pack_f32(static_cast<const float *>(h->gD), N, K, 3, h->ux, st));
    if (h->nnz > 0) {
        const int ny = c.relaxed ? 2 : 1;
        BSPK_CUDA(umma_pack_f32(static_cast<const float *>(h->gS), N, K, ny, h->uy, st));
        const int S = umma_splits(h->sms, N, N, K);
        BSPK_CUDA(umma_gemm(h->ux, N, h->uy, ny, N, K, S, h->gpart, h->d_err, st));
        k_gemm_gather<<<grid_of(h->nnz), 256, 0, st>>>(h->gpart, S, N, static_cast<size_t>(N) * N,
                                                       h->e_post, h->e_pre, h->nnz, dw);
    }
    if (NI > 0 && dw_in) {
        BSPK_CUDA(umma_pack_u8(h->inputs, NI, K, h->uy, st));
        const int S = umma_splits(h->sms, N, NI, K);
        BSPK_CUDA(umma_gemm(h->ux, N, h->uy, 1, NI, K, S, h->gpart, h->d_err, st));
        const size_t n = static_cast<size_t>(N) * NI;
        k_gemm_sum<<<grid_of(static_cast<int64_t>(n)), 256, 0, st>>>(h->gpart, S, n, dw_in);
    }
    BSPK_CUDA(cudaGetLastError());
    return BSPK_OK;
}

template <typename Real>
int run_backward(bspk_adjoint *h, void *dw, void *dw_in, cudaStream_t st) {
    const AdjArgs<Real> a = make_args<Real>(h);
    const bspk_adjoint_config &c = h->cfg;
    if (a.gemm) {
        // step 0's row of the shifted spikes stays zero
        BSPK_CUDA(cudaMemsetAsync(h->gS, 0, sizeof(Real) * static_cast<size_t>(c.batch) * c.n, st));
        BSPK_CUDA(launch_trials<Real>(k_adj_backward<Real>, a, h, st));
        if constexpr (std::is_same<Real, float>::value)
            return run_contractions(h, static_cast<float *>(dw), static_cast<float *>(dw_in), st);
        return fail(BSPK_ERR_UNSUPPORTED, "contraction mode is FP32 only");
    }
    const size_t nw = static_cast<size_t>(c.batch) * a.din_stride;
    const size_t nwi = static_cast<size_t>(c.batch) * c.n * c.n_in;
    BSPK_CUDA(cudaMemsetAsync(h->dwb, 0, sizeof(Real) * std::max<size_t>(nw, 1), st));
    BSPK_CUDA(cudaMemsetAsync(h->dwib, 0, sizeof(Real) * std::max<size_t>(nwi, 1), st));
    BSPK_CUDA(launch_trials<Real>(k_adj_backward<Real>, a, h, st));
    if (h->nnz > 0)
        k_adj_reduce<Real><<<grid_of(h->nnz), 256, 0, st>>>(static_cast<const Real *>(h->dwb),
                                                           a.din_stride, h->in_pos, h->nnz, c.batch,
                                                           static_cast<Real *>(dw));
    const int64_t ni = static_cast<int64_t>(c.n) * c.n_in;
    if (ni > 0 && dw_in)
        k_adj_reduce_in<Real><<<grid_of(ni), 256, 0, st>>>(static_cast<const Real *>(h->dwib), c.n,
                                                          c.n_in, c.batch, static_cast<Real *>(dw_in));
    BSPK_CUDA(cudaGetLastError());
    return BSPK_OK;
}

}  // namespace

extern "C" {

int bspk_adjoint_ctas_per_trial(const bspk_adjoint *h) { return h ? h->split : 0; }

int bspk_adjoint_set_contraction(bspk_adjoint *h, int on) {
    if (!h) return fail(BSPK_ERR_ARG, "null handle");
    if (on && !h->can_gemm)
        return fail(BSPK_ERR_UNSUPPORTED, "weight-gradient contraction needs an FP32 handle with its buffers");
    h->gemm = on ? 1 : 0;
    return BSPK_OK;
}

int bspk_adjoint_contraction(const bspk_adjoint *h) { return h ? h->gemm : 0; }

int bspk_adjoint_status(bspk_adjoint *h) {
    if (!h) return fail(BSPK_ERR_ARG, "null handle");
    BSPK_CUDA(cudaSetDevice(h->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    int e = 0;
    BSPK_CUDA(cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        BSPK_CUDA(cudaMemset(h->d_err, 0, sizeof(int)));
        return fail(BSPK_ERR_TIMEOUT, "a bounded wait of the gradient contraction ran out");
    }
    return BSPK_OK;
}

int bspk_adjoint_create(const bspk_adjoint_config *cfg, const int64_t *row_ptr, const int32_t *col,
                        int64_t nnz, bspk_adjoint **out) {
    if (!cfg || !out || !row_ptr || (nnz > 0 && !col)) return fail(BSPK_ERR_ARG, "null argument");
    const bspk_adjoint_config &c = *cfg;
    if (!(c.dt > 0)) return fail(BSPK_ERR_ARG, "dt must be > 0");
    if (c.precision != 32 && c.precision != 64) return fail(BSPK_ERR_ARG, "precision must be 32 or 64");
    if (c.n <= 0 || c.n_in < 0 || c.batch <= 0 || c.n_steps <= 0 || c.ckpt_every <= 0)
        return fail(BSPK_ERR_ARG, "sizes must be positive");
    if (c.n_readout < 0 || c.n_readout > c.n) return fail(BSPK_ERR_ARG, "n_readout must be in [0, n]");
    if (!(c.readout_tau > 0) || !(c.slope > 0)) return fail(BSPK_ERR_ARG, "readout_tau and slope must be > 0");
    if (row_ptr[0] != 0 || row_ptr[c.n] != nnz) return fail(BSPK_ERR_ARG, "row_ptr does not span the edges");
    for (int i = 0; i < c.n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return fail(BSPK_ERR_ARG, "row_ptr must be non-decreasing");
    for (int64_t e = 0; e < nnz; ++e)
        if (col[e] < 0 || col[e] >= c.n) return fail(BSPK_ERR_ARG, "pre index out of range");
    std::vector<double> P(c.params, c.params + 9);
    PopCoef<double> pc;
    int rc = host_make_coef(BSPK_IAF_PSC_EXP, P, c.dt, &pc);
    if (rc) return rc;
    bspk_adjoint *h = new bspk_adjoint();
    h->cfg = c;
    h->elt = c.precision == 64 ? 8 : 4;
    h->nnz = nnz;
    h->nseg = (c.n_steps + c.ckpt_every - 1) / c.ckpt_every;
    const double alpha = std::exp(-c.dt / c.readout_tau);
    const double denom = static_cast<double>(c.batch) * c.n_steps * c.n_readout;
    const double coef[16] = {pc.eP22, pc.eP21ex, pc.eP21in, pc.eP20, pc.eP11ex, pc.eP11in,
                             c.params[8], c.params[4] - c.params[0], c.params[5] - c.params[0],
                             alpha, (1.0 - alpha) * 1000.0 / c.dt,
                             c.n_readout > 0 ? 2.0 / denom : 0.0, c.slope, 0.5 * c.slope, 0.0,
                             static_cast<double>(pc.ref_count)};
    for (int i = 0; i < 16; ++i) h->coef[i] = coef[i];
    // Two CTAs per trial (a cluster sharing its spike and adjoint vectors
    // through distributed shared memory) while the batch leaves every trial
    // a pair of SMs; the readouts must lie in the first half.
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device) != cudaSuccess)
            sms = 0;
        h->split = (2 * c.batch <= sms && c.n >= 64 && c.n_readout <= c.n / 2) ? 2 : 1;
        h->sms = sms;
    }
    const int per_cta = (c.n + h->split - 1) / h->split;
    h->threads = std::min(1024, std::max(32, (per_cta + 31) / 32 * 32));
    h->smem = adj_smem_bytes(c.n, c.n_readout, c.n_in, h->elt);
    if (h->smem > 220 * 1024) {
        delete h;
        return fail(BSPK_ERR_UNSUPPORTED, "network too large for the per-trial shared-memory state");
    }
    // edge layout: in-edges of post i in row order, out-edges of pre p in
    // (post, row position) order, both column-major padded
    const int N = c.n;
    std::vector<int> din(N), dout(N, 0);
    for (int i = 0; i < N; ++i) din[i] = static_cast<int>(row_ptr[i + 1] - row_ptr[i]);
    for (int64_t e = 0; e < nnz; ++e) dout[col[e]]++;
    h->din_max = std::max(1, *std::max_element(din.begin(), din.end()));
    h->dout_max = std::max(1, *std::max_element(dout.begin(), dout.end()));
    const size_t n_ie = static_cast<size_t>(h->din_max) * N, n_oe = static_cast<size_t>(h->dout_max) * N;
    std::vector<int32_t> in_col(n_ie, 0), out_post(n_oe, 0);
    std::vector<int64_t> ie_eid(n_ie, -1), oe_eid(n_oe, -1), in_pos(std::max<int64_t>(nnz, 1));
    std::vector<int> ofill(N, 0);
    for (int i = 0; i < N; ++i)
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            const int k = static_cast<int>(e - row_ptr[i]);
            const size_t o = static_cast<size_t>(k) * N + i;
            in_col[o] = col[e];
            ie_eid[o] = e;
            in_pos[e] = static_cast<int64_t>(o);
            const int p = col[e];
            const size_t oo = static_cast<size_t>(ofill[p]++) * N + p;
            out_post[oo] = i;
            oe_eid[oo] = e;
        }
    int dev0 = 0;
    cudaGetDevice(&dev0);
    auto bail = [&](int code) {
        for (void *p : h->allocs) cudaFree(p);
        delete h;
        cudaSetDevice(dev0);
        return code;
    };
    if (cudaSetDevice(c.device) != cudaSuccess) return bail(fail(BSPK_ERR_CUDA, "cudaSetDevice failed"));
    const size_t B = c.batch, S = h->nseg, K = c.ckpt_every, R = c.n_readout, NN = N;
    const size_t el = h->elt, NI = std::max(c.n_in, 1);
    struct Buf { void **p; size_t bytes; };
    const Buf bufs[] = {
        {reinterpret_cast<void **>(&h->deg_in), 4 * NN},
        {reinterpret_cast<void **>(&h->deg_out), 4 * NN},
        {reinterpret_cast<void **>(&h->in_col), 4 * n_ie},
        {reinterpret_cast<void **>(&h->out_post), 4 * n_oe},
        {reinterpret_cast<void **>(&h->ie_eid), 8 * n_ie},
        {reinterpret_cast<void **>(&h->oe_eid), 8 * n_oe},
        {reinterpret_cast<void **>(&h->in_pos), 8 * static_cast<size_t>(std::max<int64_t>(nnz, 1))},
        {&h->w_ie, el * n_ie}, {&h->w_oe, el * n_oe}, {&h->win_t, el * NN * NI},
        {&h->ck_V, el * S * B * NN}, {&h->ck_Ie, el * S * B * NN}, {&h->ck_Ii, el * S * B * NN},
        {&h->ck_s, el * S * B * NN}, {&h->ck_z, el * S * B * std::max<size_t>(R, 1)},
        {reinterpret_cast<void **>(&h->ck_r), 4 * S * B * NN},
        {&h->tr_x, el * B * K * NN}, {&h->tr_vt, el * B * K * NN}, {&h->tr_s, el * B * K * NN},
        {&h->tr_z, el * B * K * std::max<size_t>(R, 1)},
        {reinterpret_cast<void **>(&h->tr_a), B * K * NN},
        {&h->dwb, el * B * n_ie},
        {&h->dwib, el * B * NN * NI},
        {reinterpret_cast<void **>(&h->loss_b), 8 * B},
        {reinterpret_cast<void **>(&h->loss_dev), 8},
        {reinterpret_cast<void **>(&h->nspk), 8},
        {reinterpret_cast<void **>(&h->d_err), 4},
    };
    for (const Buf &bf : bufs) {
        rc = aalloc(h, bf.p, bf.bytes);
        if (rc) return bail(rc);
    }
    if (cudaMemcpy(h->deg_in, din.data(), 4 * NN, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->deg_out, dout.data(), 4 * NN, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->in_col, in_col.data(), 4 * n_ie, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->out_post, out_post.data(), 4 * n_oe, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->ie_eid, ie_eid.data(), 8 * n_ie, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->oe_eid, oe_eid.data(), 8 * n_oe, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->in_pos, in_pos.data(), 8 * in_pos.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(BSPK_ERR_CUDA, "upload of the structure failed"));
    // FP32: the buffers of the weight-gradient contraction, when they fit in
    // 16 GB (otherwise the read-modify-write mode only)
    if (c.precision == 32) {
        const int64_t Kr = static_cast<int64_t>(c.n_steps) * c.batch;
        const size_t S1 = umma_splits(h->sms, N, N, Kr), S2 = umma_splits(h->sms, N, c.n_in, Kr);
        const size_t part = std::max(S1 * NN * NN, S2 * NN * static_cast<size_t>(c.n_in));
        const size_t op = 4 * static_cast<size_t>(Kr) * NN;
        const size_t ne = static_cast<size_t>(std::max<int64_t>(nnz, 1));
        // bf16 parts of the operands: 3 of the adjoints, 2 of the spikes (or
        // 1 of the input counts)
        const size_t xb = 2 * 3 * umma_part_elems(N, Kr);
        const size_t yb = 2 * std::max(2 * umma_part_elems(N, Kr), umma_part_elems(std::max(c.n_in, 1), Kr));
        if (2 * op + 4 * part + 8 * ne + xb + yb <= (size_t(16) << 30)) {
            void *p[7] = {};
            const size_t by[7] = {op, op, 4 * std::max<size_t>(part, 1), 4 * ne, 4 * ne, xb, yb};
            bool ok = true;
            for (int k = 0; k < 7 && ok; ++k) {
                ok = cudaMalloc(&p[k], by[k]) == cudaSuccess;
                if (ok) h->allocs.push_back(p[k]);
            }
            if (ok) {
                std::vector<int32_t> ep(ne, 0);
                for (int i = 0; i < N; ++i)
                    for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) ep[e] = i;
                ok = cudaMemcpy(p[3], ep.data(), 4 * ne, cudaMemcpyHostToDevice) == cudaSuccess &&
                     (nnz == 0 || cudaMemcpy(p[4], col, 4 * static_cast<size_t>(nnz),
                                             cudaMemcpyHostToDevice) == cudaSuccess);
                if (!ok) return bail(fail(BSPK_ERR_CUDA, "upload of the edge list failed"));
                h->gD = p[0];
                h->gS = p[1];
                h->gpart = static_cast<float *>(p[2]);
                h->e_post = static_cast<int32_t *>(p[3]);
                h->e_pre = static_cast<int32_t *>(p[4]);
                h->ux = static_cast<__nv_bfloat16 *>(p[5]);
                h->uy = static_cast<__nv_bfloat16 *>(p[6]);
                h->can_gemm = h->gemm = 1;
            } else {
                cudaGetLastError();  // an allocation that failed leaves the mode off
            }
        }
    }
    if (cudaMemset(h->d_err, 0, sizeof(int)) != cudaSuccess) return bail(fail(BSPK_ERR_CUDA, "memset failed"));
    rc = h->elt == 8 ? set_smem<double>(h) : set_smem<float>(h);
    if (rc) return bail(rc);
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(BSPK_ERR_CUDA, "upload failed"));
    cudaSetDevice(dev0);
    *out = h;
    return BSPK_OK;
}

int bspk_adjoint_destroy(bspk_adjoint *h) {
    if (!h) return BSPK_OK;
    int dev0 = 0;
    cudaGetDevice(&dev0);
    cudaSetDevice(h->cfg.device);
    for (void *p : h->allocs) cudaFree(p);
    cudaSetDevice(dev0);
    delete h;
    return BSPK_OK;
}

int bspk_adjoint_forward(bspk_adjoint *h, const void *w, const void *w_in, const uint8_t *inputs,
                         const void *targets, double *loss, int64_t *n_spikes, void *stream) {
    if (!h || (!w && h->nnz > 0) || (!w_in && h->cfg.n_in > 0) || !inputs ||
        (!targets && h->cfg.n_readout > 0))
        return fail(BSPK_ERR_ARG, "null argument");
    BSPK_CUDA(cudaSetDevice(h->cfg.device));
    if (!loss) loss = h->loss_dev;
    h->inputs = inputs;
    h->targets = targets;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = h->elt == 8 ? run_forward<double>(h, w, w_in, loss, n_spikes, st)
                         : run_forward<float>(h, w, w_in, loss, n_spikes, st);
    if (rc) return rc;
    h->have_forward = true;
    return BSPK_OK;
}

int bspk_adjoint_backward(bspk_adjoint *h, void *dw, void *dw_in, void *stream) {
    if (!h || (!dw && h->nnz > 0)) return fail(BSPK_ERR_ARG, "null argument");
    if (!h->have_forward) return fail(BSPK_ERR_STATE, "backward needs a forward on this handle first");
    BSPK_CUDA(cudaSetDevice(h->cfg.device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return h->elt == 8 ? run_backward<double>(h, dw, dw_in, st) : run_backward<float>(h, dw, dw_in, st);
}

}  // extern "C"
