// batch_args.h -- many independent iaf networks ("instances") of uneven
// sizes in one persistent launch.
//
// Every instance is cut into tiles of at most T neurons (T = blockDim.x);
// the host assigns tiles to CTAs (longest-processing-time first over a cost
// model that a pilot run calibrates) and each CTA advances its tiles window
// by window.  An instance's recurrent edges share one arrival lag, and its
// window is that lag: what a window emits arrives exactly in the next
// window, so the arrivals of a tile-window are delivered into a transient
// shared-memory accumulator acc[W][T] right before the window's updates and
// nothing but state and spike records persists between windows.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device_types.h"
#include "lif_args.h"

namespace bspk {

constexpr int kBatchMaxPops = 8;     // populations per instance
constexpr int kBatchMaxDrives = 8;   // Poisson drives per instance
constexpr int kBatchMaxProj = 16;    // projections per instance
constexpr int kBatchMaxWindow = 64;  // arrival lag in steps
constexpr int kBatchCdfCap = 1024;   // CDF entries per instance (shared memory)
constexpr int kBatchStepBits = 6;    // record payload: pre << 6 | step in window

struct BatchInstDev {
    int n;                  // neurons
    int W;                  // window = arrival lag of every recurrent edge
    int tile0, ntiles;      // the instance's tiles
    int npop;
    int pop_off[kBatchMaxPops + 1];
    int coef0;              // first PopCoef of the instance
    int ndrive, drive0;     // drives; DriveDev.pop is the instance-local pop
    int cdf_n;              // CDF entries of all its drives (DriveDev.cdf_off local)
    int64_t cdf0;
    int proj0;              // fixed-point projection weights proj_w[proj0 + slot]
    double inv_scale;       // 2^-k of the instance's fixed-point accumulator
    int rec_cap;            // entries per tile record
    int record;             // keep the spike train (step, neuron) of this instance
    int64_t rec0;           // records of tile t, parity p: rec0 + (2 t + p) * (1 + rec_cap)
    int64_t g0;             // first neuron in the global state arrays
    int64_t ptr0;           // tile CSR bounds: ptr[ptr0 + tile * n + pre] (+1)
    int64_t edge0;          // first edge of the instance
};

struct BatchTileDev {
    int inst;
    int tloc;               // tile index within the instance
    int first, n;           // instance-local neurons [first, first + n)
};

template <typename Real>
struct BatchArgs {
    int n_tiles, n_inst, T, Wmax;
    const BatchInstDev *inst;
    const BatchTileDev *tiles;
    const int *cta_ptr, *cta_tiles;  // CTA c runs cta_tiles[cta_ptr[c] .. cta_ptr[c + 1])
    const PopCoef<Real> *coef;
    const DriveDev *drives;
    const uint64_t *cdf;
    // fixed point (int32 for FP32, int64 for FP64): arrivals are accumulated
    // as integers, w_fix = rint(w 2^k) with k per instance such that no
    // accumulator slot can overflow
    const typename FixOf<Real>::type *proj_w;
    Real *s[6];
    int *r;
    const int *ptr;                  // int32 bounds relative to the instance's edge0
    const uint32_t *edges;           // post_in_tile | projection slot << 16
    unsigned long long *recs;        // tagged words: (window + 1) << 32 | payload
    int *part;                       // per tile: entries already written in a split window
    unsigned int *spk_cnt;           // spikes per neuron since upload
    int64_t *spk_step;               // recorded spikes, per-CTA regions of spk_cap
    int32_t *spk_id;                 // instance-local neuron
    int32_t *spk_inst;
    long long *rec_count;            // per CTA
    int64_t spk_cap;
    int64_t step0, n_steps;
    int64_t n_total;                 // neurons of all instances
    const Real *drive;               // Poisson drive drive[(step - drive_step0) * n_total + g]
    int64_t drive_step0;
    int *err;
};

size_t lif_batch_smem(int T, int Wmax, int dbl);
template <typename Real>
cudaError_t launch_lif_batch(const BatchArgs<Real> &a, int model, int grid, cudaStream_t st);
template <typename Real>
int lif_batch_max_ctas_per_sm(int model, int T, int Wmax);
// Poisson drive of every neuron of every instance for steps [m0, m0 + n).
template <typename Real>
cudaError_t launch_batch_drive_fill(const BatchArgs<Real> &a, int64_t m0, int n, Real *out,
                                    cudaStream_t st);

}  // namespace bspk
