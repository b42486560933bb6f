// aeif_args.h -- per-step engine: aeif_cond_alpha (adaptive RKF45) and
// networks with plastic (stdp_synapse) projections.  One step is a short
// sequence of kernels, replayed through a CUDA graph; the step index lives
// in device memory (advanced by the last kernel of the step), so the same
// graph serves every chunk of steps.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device_types.h"

struct bspk_plan;

namespace bspk {

template <typename Real>
struct StepArgs {
    int N, npop, nproj, ndrive, model, R, L;
    int ports;  // iaf models: 1 = receptor ports 0 / 1 kept apart (no sign split)
    const PopCoef<Real> *coef;
    Real *s[8];
    int *r;
    Real *ring;  // [L][R][N]
    const ProjDev<Real> *projs;
    const int *proj_plastic;  // 1 for plastic projections (delivered by the STDP kernels)
    const DriveDev *drives;
    const int *pop_drive_ptr, *pop_drive_list;
    const uint64_t *cdf;
    uint64_t *hist;       // spike history word per neuron (bit m & 63)
    uint32_t *step_spk;   // spikes of the current step (gids)
    int *step_nspk;
    int64_t *spk_step;
    int32_t *spk_gid;
    unsigned long long *spk_count;
    int64_t spk_cap;
    const uint8_t *spk_flag;
    const int32_t *rec_slot;
    Real *v_out;
    int n_rec;
    int64_t *step_ptr;    // device step counter
    int64_t run_step0;
    unsigned long long *rk_iters;
    int *err;
    int static_chunks;  // edge work items per row of the widest static projection
    int n_counters;     // per-step counters at step_nspk (zeroed at the end of each step)
};

// One plastic projection (pair STDP, eager substrate).
struct StdpDev {
    int pre_off, post_off, n_pre, n_post, lag;  // lag: arrival lag of the pre spike
    int receptor;
    double tau_plus, tau_minus, lambda_, alpha, mu_plus, mu_minus, Wmax, dec_pre, dec_post;
    int rule;  // 0: pair stdp_synapse, 1: stdp_triplet_synapse
    double a2p, a3p, a2m, a3m, dec_pre2, dec_post2;  // triplet amplitudes, slow-trace decays
    double inv_Wmax;
    int out_chunks, in_chunks;  // edge work items per pre row / post column
    const int64_t *indptr;   // CSR over pre
    const uint32_t *edges;   // post_local | lag << 24
    double *w;               // FP64 weights, CSR order
    const int64_t *cindptr;  // CSC over post
    const int64_t *cperm;    // CSC position -> CSR edge id
    const uint32_t *cedges;  // pre_local | lag << 24
    double *pre_trace, *post_trace;    // fast traces
    double *pre_trace2, *post_trace2;  // slow traces (triplet rule)
    int *pre_list, *post_list, *counts;  // counts[0] pres, counts[1] posts of this step
    // weight trajectory: after every step, row (step - run_step0 - 1) of
    // wtrace[n_steps][n_edges] receives the weights (nullptr: not recorded)
    double *wtrace;
    int64_t n_edges, run_step0;
};

// Windowed engine: the neuron kernel advances W steps per launch (all lags
// >= W, so no spike of a window arrives inside it) and the plastic
// projection's weights are brought up to date per edge at each arrival.
struct WinDev {
    int on;                // a plastic pair-rule projection is handled (s)
    StdpDev s;
    int W, cap;            // window; arrivals held per (step, post)
    double *kp;            // [W][n_pre] pre trace at step n0 + k without that step's arrival
    uint32_t *amask;       // [n_pre] window steps at which each pre's spikes arrive
                           // (bit k: step n0 + k); an edge's arrivals in the window
                           // are exactly its pre's bits, so the last step that
                           // brought it up to date follows from them
    WinArrival *arr;       // [W][cap][n_post] arrivals at n0 + k
    int *cnt;              // [W][n_post] arrivals per (step, post), cleared by their reader
    uint32_t *spk;         // spikes of the window: gid << 5 | step in window
    uint32_t *pre_list;    // pres with arrivals in the window, then their step masks
    uint32_t *post_list;   // plastic posts that fired in the window, then their masks
    int *ctr;              // [0] window spikes, [1] arriving pres, [2] posts that fired
    int *err;
};

int run_per_step(bspk_plan *p, int64_t n_steps, cudaStream_t st);

}  // namespace bspk
