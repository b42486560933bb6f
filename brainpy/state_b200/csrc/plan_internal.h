// plan_internal.h -- the plan object behind the C ABI (host only).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/bspk.h"
#include "device_types.h"

namespace bspk {

int fail(int code, const std::string &msg);

#define BSPK_CUDA(call)                                                                 \
    do {                                                                                \
        cudaError_t e__ = (call);                                                       \
        if (e__ != cudaSuccess)                                                         \
            return ::bspk::fail(BSPK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)

struct Pop {
    int n = 0, off = 0;
    std::vector<double> p;
    PopCoef<double> c{};
};

struct Proj {
    int pre = 0, post = 0, receptor = 0;
    std::vector<int64_t> indptr;
    std::vector<int32_t> post_local, delay;
    std::vector<double> w;
    bool homogeneous = false;
    double w0 = 0.0;
    bool plastic = false;
    bspk_stdp_params stdp{};
    int rule = 0;  // 0: pair stdp_synapse, 1: stdp_triplet_synapse
    bspk_stdp_triplet_params trip{};
    int trace_cols() const { return rule == 1 ? 2 : 1; }  // traces per side
    int input_order = 0;
    int64_t max_out = 0, max_in = 0;  // largest row / column of the CSR (set at upload)
    // device
    int64_t *d_indptr = nullptr;
    uint32_t *d_edges = nullptr;
    void *d_w = nullptr;
    int64_t *d_cindptr = nullptr;
    uint32_t *d_cedges = nullptr;
    double *d_cw = nullptr;
    double *d_wplastic = nullptr;   // FP64 plastic weights (CSR order)
    int64_t *d_cperm = nullptr;     // CSC position -> CSR edge id
    void *d_pre_trace = nullptr, *d_post_trace = nullptr;  // [trace_cols][n]
    int *d_pre_list = nullptr, *d_post_list = nullptr;  // per-step STDP work lists
    // weight trajectory of the last run (bspk_record_weights): [steps][E]
    bool rec_w = false;
    double *d_wtrace = nullptr;
    int64_t wtrace_cap = 0, wtrace_steps = 0;
};

struct Drive {
    int post = 0, lag = 0, receptor = 0, delay = 0;
    double rate = 0, weight = 0;
    uint32_t seed = 0;
    int64_t tmin = 0, tmax = 0;
    std::vector<double> cdf;       // kind 0: the CDF in float64
    int input_order = 0;
    int kind = 0;                  // 1: the reference kernel path's stream
    uint32_t key0 = 0, key1 = 0;   // kind 1: the device population's object key
    int64_t unit_off = 0;          // kind 1: unit of the population's first neuron
    std::vector<uint64_t> thr;     // kind 1: integer thresholds (jax_rng.h)
};

}  // namespace bspk

struct bspk_plan {
    bspk_config cfg{};
    std::vector<bspk::Pop> pops;
    std::vector<bspk::Proj> projs;
    std::vector<bspk::Drive> drives;
    std::vector<int> input_kind;  // creation order: >= 0 proj id, < 0 drive -(id+1)
    std::vector<int32_t> rec_v;
    std::vector<uint8_t> spk_flag;
    bool has_spk_flag = false;
    int N = 0;
    bool uploaded = false;
    int64_t step = 0;
    // derived
    int W = 1, L = 1, max_lag = 0;
    int elt = 4;  // bytes per Real
    // device buffers
    std::vector<void *> allocs;
    void *d_s[9] = {};
    int *d_r = nullptr;
    void *d_ring = nullptr;
    uint64_t *d_hist = nullptr;
    void *d_coef = nullptr;
    void *d_projs = nullptr;
    bspk::DriveDev *d_drives = nullptr;
    uint64_t *d_cdf = nullptr;
    int cdf_total = 0;
    int *d_pop_out_ptr = nullptr, *d_pop_out_list = nullptr;
    int *d_pop_in_ptr = nullptr, *d_pop_in_list = nullptr;
    int *d_pop_drive_ptr = nullptr, *d_pop_drive_list = nullptr;
    int64_t *d_spk_step = nullptr;
    int32_t *d_spk_gid = nullptr;
    unsigned long long *d_spk_count = nullptr;
    uint8_t *d_spk_flag = nullptr;
    int32_t *d_rec_slot = nullptr;
    void *d_v = nullptr;
    int64_t v_steps_cap = 0;
    int64_t last_run_steps = 0;
    unsigned int *d_barrier = nullptr;
    int *d_err = nullptr;
    // per-step engine (aeif / plastic)
    uint32_t *d_step_spk = nullptr;  // spikes of the current step (gids)
    int *d_step_nspk = nullptr;
    unsigned long long *d_rk_iters = nullptr;
    int *d_proj_plastic = nullptr;    // 1 per plastic projection
    int *d_step_counters = nullptr;   // [0] spikes of the step, then 2 per plastic projection
    int n_step_counters = 0;
    int64_t *d_step_ptr = nullptr;    // device step counter of the per-step engine
    // windowed form of the per-step engine (WinDev): the neuron kernel
    // advances W steps per launch when every lag is >= W >= 2 and at most one
    // projection is plastic (pair rule, one lag); weight recording runs the
    // per-step form
    bool win = false, win_ok = false;  // selected, possible
    double *d_win_kp = nullptr;
    uint32_t *d_win_amask = nullptr;
    bspk::WinArrival *d_win_arr = nullptr;
    int *d_win_cnt = nullptr;
    int win_cap = 0;
    uint32_t trial = 0;  // trial index of the keyed drives' step keys
    uint32_t *d_win_spk = nullptr;
    uint32_t *d_win_pre = nullptr;
    uint32_t *d_win_post = nullptr;
    int *d_win_ctr = nullptr;
    // timing
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    int grid = 0, block = 0, tile = 0;
    int sm_count = 0;
    // tiled (target-partitioned) fast path
    bool tiled = false;
    int *d_tptr = nullptr;
    uint32_t *d_tedges = nullptr;
    void *d_tw = nullptr;          // per-edge fixed-point weights (int32 / int64), or null
    void *d_twproj = nullptr;      // per-projection fixed-point weights
    double tinv_scale = 1.0;       // 2^-k of the fixed-point ring
    uint32_t *d_tlist = nullptr;   // spike records [kRecBufs][G][kRecWords]
    uint32_t *d_tovf = nullptr;    // record overflow [kRecBufs][G][list_cap]
    long long *d_trec = nullptr;   // per-CTA spike-record counts
    int list_cap = 0;
    bool smem_ptr = false;
    int hold_cta = -1, hold_win = -1;  // test hook of the next run (tiled path)
    void *h_stage = nullptr;  // pinned host staging of read-backs (V_m traces), grown on demand
    size_t h_stage_bytes = 0;
    // iaf models with receptor ports kept apart (0 = 'ex', 1 = 'in_', signs
    // kept), stepped by the per-step engine; 0 = one summed input split by sign
    int ports_sep = 0;
    // set at upload: a separate-port plan that the tiled kernel runs (two
    // rings in shared memory) instead of the per-step engine
    int ports_tiled = 0;
    int tW = 1;                    // tiled window (half the smallest lag when pipelined)
    int tpipe = 0;                 // 1: window j - 1 is delivered after window j's update
    void *d_tdrive = nullptr;      // Poisson drive of one launch, [steps][N]
    int64_t *d_cspk_step = nullptr;  // compacted spike list of the last run (tiled)
    int32_t *d_cspk_gid = nullptr;
    unsigned long long *d_cspk_n = nullptr;
    bool cspk_valid = false;
    int64_t cspk_n = 0;
    int64_t tdrive_steps = 0;      // its capacity in steps
    // Drive double buffer.  Beside each persistent launch, the drive pass of
    // the steps that follow it (the next launch of the run, or the same
    // number of steps after the run) runs on a side stream into the other
    // buffer; a run that starts where the prefill starts uses it as is.
    void *d_tdrive2 = nullptr;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_side = nullptr, ev_main = nullptr;
    int64_t pref_step0 = -1, pref_n = 0;  // prefilled steps [pref_step0, +pref_n)
    int pref_buf = 0;                     // in buffer 0 (d_tdrive) or 1 (d_tdrive2)
    // the step a checkpoint restore rewound the plan to (-1: none since the
    // last run that started elsewhere): a run from there is taken for a
    // rerun, and the prefill after it targets that step again
    int64_t restart_step = -1;
    bool drive_overlap = true;
    int rec_rep = 1;                      // copies of every spike record (tiled kernel)
    int poll_pause = 400;                 // ns before a window's first record poll
    int drive_chunk = 0;                  // steps per persistent launch (0: drive budget)
    int rec_stride = 16;                  // words per record slot (kRecWords or more)
    size_t tlist_words = 0;               // allocated words of d_tlist
};

namespace bspk {
int dalloc_bytes(bspk_plan *p, void **ptr, size_t bytes);
// float64 coefficients of a population (propagators, thresholds) and the
// Poisson CDF of rate*dt as 53-bit integer thresholds
int host_make_coef(int model, const std::vector<double> &params, double h, PopCoef<double> *c);
std::vector<uint64_t> host_poisson_thresholds(double lam);
int sync_and_check(bspk_plan *p);
// Grow the plan's pinned staging buffer to at least `bytes`.
int plan_stage(bspk_plan *p, size_t bytes);
// Input channels of the plan's ring (receptor ports) and whether the
// per-step engine steps it.
inline int plan_n_receptors(const bspk_plan *p) {
    return p->ports_sep ? 2 : model_n_receptors(p->cfg.model);
}
inline bool plan_per_step(const bspk_plan *p) {
    return model_per_step(p->cfg.model) || (p->ports_sep != 0 && !p->ports_tiled);
}
}  // namespace bspk
