// lif_args.h -- launch arguments of the windowed iaf kernels.
#pragma once
#include <cuda_runtime.h>

#include "device_types.h"

namespace bspk {

template <typename Real>
struct LifArgs {
    int N, npop, nproj, ndrive;
    const PopCoef<Real> *coef;
    Real *s[6];
    int *r;
    Real *ring;
    int L;
    const ProjDev<Real> *projs;
    const int *pop_out_ptr, *pop_out_list;      // outgoing projections per pre pop
    const int *pop_in_ptr, *pop_in_list;        // inputs per post pop, creation order
                                                // (>= 0 projection, < 0 drive -(id+1))
    const DriveDev *drives;
    const int *pop_drive_ptr, *pop_drive_list;  // drives per post pop
    const uint64_t *cdf;  // Poisson CDF thresholds floor(F * 2^53)
    int cdf_total;
    int64_t step0, n_steps, run_step0;
    int W;
    int pipe;   // tiled kernel: 1 = window j-1 is delivered after window j's update
    int tile;
    int model;
    int64_t *spk_step;
    int32_t *spk_gid;
    unsigned long long *spk_count;
    int64_t spk_cap;
    const uint8_t *spk_flag;
    const int32_t *rec_slot;
    Real *v_out;
    int n_rec;
    uint64_t *hist;  // exact mode spike history (bit m & 63 of neuron g)
    unsigned int *barrier;
    int *err;
};

// Target-partitioned delivery structures of the tiled kernel: for every CTA
// c a CSR over all pre neurons of the edges that target c's tile,
// ptr[c * (N + 1) + pre] .. ptr[c * (N + 1) + pre + 1] into `edges` (edge
// word = post_in_tile | lag << 16 | projection << 24); per-window spike
// records list[kRecBufs][rec_rep][G][rec_stride] (tagged count word + kRecInline
// tagged entries) with an overflow area ovf[kRecBufs][G][list_cap];
// (with separate receptor ports, bit 15 of the edge word is the port);
// per-CTA spike-record counts rec_count[G] (running across the launches of
// one run); the Poisson drive of every (step, neuron) of the launch, drawn
// by a separate kernel, drive[(step - drive_step0) * N + neuron].
constexpr int kRecWords = 16;
constexpr int kRecInline = kRecWords - 1;
constexpr int kRecBufs = 4;
constexpr int kRecRepMax = 16;

// The tiled kernel accumulates arrivals in fixed point: weights are
// rint(w * 2^k) in int32 (FP32 plans) or int64 (FP64 plans), k chosen per plan
// so that no ring slot can overflow (|sum| <= max over neurons of the sum of
// |w| over their in-edges, since an edge contributes at most once per arrival
// step).  Integer shared-memory atomics are several times faster than
// floating-point ones here, and integer sums do not depend on the order of
// the additions.
template <typename Real>
struct FixOf;
template <>
struct FixOf<float> {
    using type = int32_t;
};
template <>
struct FixOf<double> {
    using type = long long;
};

template <typename Real>
struct TiledArgs {
    using Fix = typename FixOf<Real>::type;
    const int *ptr;
    const uint32_t *edges;
    const Fix *wfix;   // per-edge fixed-point weights, or nullptr when every projection is homogeneous
    const Fix *wproj;  // per-projection fixed-point weight (homogeneous projections)
    Real inv_scale;    // 2^-k
    uint32_t *list;
    uint32_t *ovf;
    long long *rec_count;
    int list_cap;
    int smem_ptr;   // 1: the tile's CSR bounds are staged in shared memory
    const Real *drive;
    int64_t drive_step0;
    // test hook: CTA hold_cta does not publish the header of its record of
    // window hold_win (-1: none), so every bounded wait for it runs out
    int hold_cta, hold_win;
    // 1: the receptor ports 'ex' and 'in_' have rings of their own (edge
    // word bit 15 = port; drives feed 'ex'); 0: one ring, sum split by sign
    int ports;
    // copies of every record (1..kRecRepMax): CTA c polls copy c % rec_rep,
    // so each record line is read by G / rec_rep CTAs instead of all G
    int rec_rep;
    // words from one CTA's record to the next (>= kRecWords): records on
    // separate lines, or spread further over L2
    int rec_stride;
    // pause (ns) before the first poll of a window's records, about one
    // write latency: a poll issued right after this CTA's own publish mostly
    // finds the other records not yet written
    int poll_pause;
};

struct TiledLayout {
    size_t coef, proj, ring, drv, spk, ptr, total;
};
// drv: double-buffered drive of one window, [2][W][tile]
__host__ __device__ inline TiledLayout tiled_layout(size_t coef_sz, size_t proj_sz, size_t real_sz,
                                                    int npop, int nproj, int tile, int L, int W,
                                                    int n_ptr) {
    auto al = [](size_t x) { return (x + 15) & ~size_t(15); };
    TiledLayout l;
    l.coef = 0;
    l.proj = al(l.coef + coef_sz * npop);
    l.ring = al(l.proj + proj_sz * nproj);
    l.drv = al(l.ring + real_sz * static_cast<size_t>(L) * tile);
    l.spk = al(l.drv + real_sz * 2 * static_cast<size_t>(W) * tile);
    l.ptr = al(l.spk + sizeof(uint32_t) * static_cast<size_t>(tile) * W);
    l.total = al(l.ptr + sizeof(int) * static_cast<size_t>(n_ptr));
    return l;
}

template <typename Real>
cudaError_t launch_lif_tiled(const LifArgs<Real> &a, const TiledArgs<Real> &t2, int grid,
                             cudaStream_t st);
// Poisson drive of steps [m0, m0 + n) for every neuron into out[(m - m0) * N + g];
// `beside`: blocks of 128 threads sized to run next to the persistent kernel.
template <typename Real>
cudaError_t launch_drive_fill(const LifArgs<Real> &a, int64_t m0, int n, Real *out,
                              cudaStream_t st, bool beside = false);
// ports: two rings ('ex', 'in_') instead of one
size_t lif_tiled_smem(int tile, int L, int W, int N, int npop, int nproj, bool dbl, bool smem_ptr,
                      bool ports = false);
// Recorded spikes of the tiled kernel's per-CTA regions into one list.
cudaError_t launch_compact_spikes(int G, int64_t region, const long long *rec_count,
                                  const int64_t *in_step, const int32_t *in_gid, int64_t *out_step,
                                  int32_t *out_gid, unsigned long long *out_n, cudaStream_t st);

// Launchers (cooperative, persistent).  Return the cudaError_t of the launch.
template <typename Real>
cudaError_t launch_lif_fast(const LifArgs<Real> &a, int grid, int block, cudaStream_t st);
cudaError_t launch_lif_exact(const LifArgs<double> &a, int grid, int block, cudaStream_t st);

size_t lif_fast_smem(int tile, int W, int npop, int ndrive, int nproj, int cdf_total, bool dbl);

// Shared-memory layout of the windowed kernels (16-byte aligned sections).
struct SmemLayout {
    size_t coef, drive, proj, cdf, spk, total;
};
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline SmemLayout smem_layout(size_t coef_sz, size_t proj_sz, int npop,
                                                  int ndrive, int nproj, int cdf_total,
                                                  int spk_rows, int spk_cols) {
    SmemLayout l;
    l.coef = 0;
    l.drive = align16(l.coef + coef_sz * npop);
    l.proj = align16(l.drive + sizeof(DriveDev) * ndrive);
    l.cdf = align16(l.proj + proj_sz * nproj);
    l.spk = align16(l.cdf + sizeof(double) * cdf_total);
    l.total = align16(l.spk + sizeof(uint32_t) * static_cast<size_t>(spk_rows) * spk_cols);
    return l;
}
size_t lif_exact_smem(int block, int npop, int ndrive, int nproj, int cdf_total);

}  // namespace bspk
