// lif_fast.cu -- persistent windowed kernel for iaf_psc_alpha / iaf_psc_exp
// networks (FP32 or FP64, atomics-order delivery).
//
// One cooperative launch runs a whole bspk_run, one CTA per SM.  Time is cut
// into windows of W = d_min steps (the smallest arrival lag of any edge): no
// spike emitted inside a window can arrive inside it, so every neuron
// advances W steps without hearing from any other CTA.  Per window:
//   A. each CTA updates its tile of neurons for W steps: ring slots are read
//      with L2-only loads and cleared, the Poisson drive is drawn in-register
//      (threefry counter RNG + CDF table in shared memory), spikes go to a
//      shared-memory list;
//   B. the CTA expands its spikes' CSR rows into 128-edge chunks (block scan
//      in shared memory) and its warps scatter the chunks in parallel with
//      red.add into ring slot (n + lag) mod L, so every row's loads are in
//      flight at once instead of one dependent chain per row;
//   C. one bounded grid barrier.
// L >= W + max_lag, so B of window k never aliases a slot A of window k reads.
#include "common.cuh"
#include "lif_args.h"

namespace bspk {

namespace {

constexpr int kChunk = 128;      // edges per delivery chunk (4 per lane)
constexpr int kItemCap = 1024;   // (spike, projection) rows expanded per batch
constexpr int kTabCap = 256;     // adjacency-table entries kept in shared memory

// In-place exclusive scan of s[0..n) by the whole block; returns the total.
__device__ int block_exclusive_scan(int *s, int n, int *s_warp) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    int carry = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + tid;
        const int v = i < n ? s[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_warp[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < nw) s_warp[lane] = t;  // inclusive warp totals
        }
        __syncthreads();
        const int warp_off = wid > 0 ? s_warp[wid - 1] : 0;
        const int total = s_warp[nw - 1];
        if (i < n) s[i] = carry + warp_off + x - v;
        carry += total;
        __syncthreads();
    }
    return carry;
}

__device__ __forceinline__ int find_pop(const int *s_off, int npop, int g) {
    int p = 0;
    while (p + 1 < npop && s_off[p + 1] <= g) ++p;
    return p;
}

}  // namespace

template <typename Real, int MODEL>
__global__ void __launch_bounds__(512) k_lif_fast(const LifArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemLayout lay = smem_layout(sizeof(PopCoef<Real>), sizeof(ProjDev<Real>), a.npop,
                                       a.ndrive, a.nproj, a.cdf_total, a.tile, a.W);
    PopCoef<Real> *s_coef = reinterpret_cast<PopCoef<Real> *>(smem_raw + lay.coef);
    DriveDev *s_drive = reinterpret_cast<DriveDev *>(smem_raw + lay.drive);
    ProjDev<Real> *s_proj = reinterpret_cast<ProjDev<Real> *>(smem_raw + lay.proj);
    uint64_t *s_cdf = reinterpret_cast<uint64_t *>(smem_raw + lay.cdf);
    uint32_t *s_spk = reinterpret_cast<uint32_t *>(smem_raw + lay.spk);
    __shared__ int s_off[kMaxPops + 1];
    __shared__ int s_out_ptr[kMaxPops + 1], s_drv_ptr[kMaxPops + 1];
    __shared__ int s_out_list[kTabCap], s_drv_list[kTabCap];
    __shared__ int s_item_beg[kItemCap];        // first edge of the row
    __shared__ int s_item_end[kItemCap];
    __shared__ int s_item_nch[kItemCap];        // chunks, then exclusive offsets
    __shared__ uint32_t s_item_meta[kItemCap];  // proj << 16 | slot of the spike step
    __shared__ int s_warp[32];
    __shared__ int s_nsp;
    __shared__ unsigned long long s_base;

    const int tid = threadIdx.x, B = blockDim.x;
    for (int i = tid; i < a.npop; i += B) {
        s_coef[i] = a.coef[i];
        s_off[i] = a.coef[i].off;
    }
    for (int i = tid; i <= a.npop; i += B) {
        s_out_ptr[i] = a.pop_out_ptr[i];
        s_drv_ptr[i] = a.pop_drive_ptr[i];
    }
    for (int i = tid; i < a.ndrive; i += B) s_drive[i] = a.drives[i];
    for (int i = tid; i < a.nproj; i += B) s_proj[i] = a.projs[i];
    for (int i = tid; i < a.cdf_total; i += B) s_cdf[i] = a.cdf[i];
    __syncthreads();
    for (int i = tid; i < s_out_ptr[a.npop] && i < kTabCap; i += B) s_out_list[i] = a.pop_out_list[i];
    for (int i = tid; i < s_drv_ptr[a.npop] && i < kTabCap; i += B) s_drv_list[i] = a.pop_drive_list[i];
    int max_out = 0;
    for (int p = 0; p < a.npop; ++p) max_out = max(max_out, s_out_ptr[p + 1] - s_out_ptr[p]);
    __syncthreads();

    const int N = a.N, L = a.L;
    const int cta0 = blockIdx.x * a.tile;
    const int cta1 = min(cta0 + a.tile, N);
    const int64_t n_end = a.step0 + a.n_steps;
    const int lane = tid & 31, wid = tid >> 5, nw = B >> 5;
    int epoch = 0;

    for (int64_t n0 = a.step0; n0 < n_end; n0 += a.W) {
        const int Wk = static_cast<int>((n_end - n0) < a.W ? (n_end - n0) : a.W);
        if (tid == 0) s_nsp = 0;
        __syncthreads();
        const int slot0 = static_cast<int>(n0 % L);

        // ---- A: neuron updates for Wk steps
        for (int g = cta0 + tid; g < cta1; g += B) {
            const int p = find_pop(s_off, a.npop, g);
            const PopCoef<Real> &c = s_coef[p];
            Real st[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) st[i] = a.s[i][g];
            int r = a.r[g];
            const int rslot = a.rec_slot ? a.rec_slot[g] : -1;
            Real in[kMaxWindow];
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k) {
                if (k < Wk) {
                    int slot = slot0 + k;
                    if (slot >= L) slot -= L;
                    Real *cell = a.ring + static_cast<size_t>(slot) * N + g;
                    in[k] = __ldcg(cell);
                    __stcg(cell, Real(0));
                }
            }
            for (int q = s_drv_ptr[p]; q < s_drv_ptr[p + 1]; ++q) {
                const DriveDev &d = s_drive[s_drv_list[q]];
                const uint32_t idx = static_cast<uint32_t>(g - c.off);
                const Real w = static_cast<Real>(d.weight);
#pragma unroll
                for (int k = 0; k < kMaxWindow; ++k) {
                    if (k < Wk) {
                        const int64_t se = n0 + k - d.lag;
                        if (d.tmin < se && se <= d.tmax) {
                            const uint64_t u = drive_draw(d, static_cast<uint32_t>(se), idx);
                            const int cnt = poisson_from_table(s_cdf + d.cdf_off, d.cdf_n, u);
                            in[k] += static_cast<Real>(cnt) * w;
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k) {
                if (k < Wk) {
                    bool sp;
                    if (MODEL == 0) sp = iaf_alpha_step<Real>(c, st, r, in[k]);
                    else sp = iaf_exp_step<Real>(c, st, r, in[k]);
                    if (sp) {
                        const int pos = atomicAdd(&s_nsp, 1);
                        s_spk[pos] = (static_cast<uint32_t>(g - cta0) << 5) | static_cast<uint32_t>(k);
                    }
                    if (rslot >= 0)
                        a.v_out[static_cast<size_t>(n0 + k - a.run_step0) * a.n_rec + rslot] = st[0];
                }
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) a.s[i][g] = st[i];
            a.r[g] = r;
        }
        __syncthreads();
        const int nsp = s_nsp;

        // ---- spike record
        if (nsp > 0) {
            if (tid == 0) s_base = atomicAdd(a.spk_count, static_cast<unsigned long long>(nsp));
            __syncthreads();
            for (int i = tid; i < nsp; i += B) {
                const uint32_t e = s_spk[i];
                const int g = cta0 + static_cast<int>(e >> 5);
                const unsigned long long at = s_base + i;
                if (at < static_cast<unsigned long long>(a.spk_cap)) {
                    const bool keep = a.spk_flag == nullptr || a.spk_flag[g] != 0;
                    a.spk_step[at] = n0 + (e & 31u);
                    a.spk_gid[at] = keep ? g : -1;  // unrecorded neuron: hole
                }
            }
        }

        // ---- B: chunked scatter of this CTA's spikes
        if (max_out > 0) {
            const int spk_per_batch = kItemCap / max_out;
            for (int i0 = 0; i0 < nsp; i0 += spk_per_batch) {
                const int ns = min(spk_per_batch, nsp - i0);
                const int M = ns * max_out;
                for (int m = tid; m < M; m += B) {
                    const int i = i0 + m / max_out, qq = m % max_out;
                    const uint32_t e = s_spk[i];
                    const int g = cta0 + static_cast<int>(e >> 5);
                    const int p = find_pop(s_off, a.npop, g);
                    int nch = 0;
                    if (qq < s_out_ptr[p + 1] - s_out_ptr[p]) {
                        const int pj = s_out_list[s_out_ptr[p] + qq];
                        const int gl = g - s_off[p];
                        const int64_t beg = __ldg(s_proj[pj].indptr + gl);
                        const int64_t end = __ldg(s_proj[pj].indptr + gl + 1);
                        int nmod = slot0 + static_cast<int>(e & 31u);
                        if (nmod >= L) nmod -= L;
                        s_item_beg[m] = static_cast<int>(beg);
                        s_item_end[m] = static_cast<int>(end);
                        s_item_meta[m] = (static_cast<uint32_t>(pj) << 16) | static_cast<uint32_t>(nmod);
                        nch = static_cast<int>((end - beg + kChunk - 1) / kChunk);
                    }
                    s_item_nch[m] = nch;
                }
                __syncthreads();
                const int C = block_exclusive_scan(s_item_nch, M, s_warp);
                // warps take chunks; a binary search finds each chunk's row
                for (int c = wid; c < C; c += nw) {
                    int lo = 0, hi = M - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (s_item_nch[mid] <= c) lo = mid; else hi = mid - 1;
                    }
                    const uint32_t meta = s_item_meta[lo];
                    const ProjDev<Real> &P = s_proj[meta >> 16];
                    const int nmod = static_cast<int>(meta & 0xFFFFu);
                    const int j0 = s_item_beg[lo] + (c - s_item_nch[lo]) * kChunk;
                    const int jend = s_item_end[lo];
                    Real *base = a.ring + P.post_off;
                    uint32_t ed[kChunk / 32];
                    Real w[kChunk / 32];
#pragma unroll
                    for (int u = 0; u < kChunk / 32; ++u) {
                        const int j = j0 + u * 32 + lane;
                        if (j < jend) {
                            ed[u] = __ldg(P.edges + j);
                            w[u] = P.homogeneous ? P.w0 : __ldg(P.w + j);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kChunk / 32; ++u) {
                        const int j = j0 + u * 32 + lane;
                        if (j < jend) {
                            int slot = nmod + static_cast<int>(ed[u] >> kEdgeDelayShift);
                            if (slot >= L) slot -= L;
                            atomicAdd(base + static_cast<size_t>(slot) * N + (ed[u] & kEdgePostMask),
                                      w[u]);
                        }
                    }
                }
                __syncthreads();
            }
        }

        // ---- C: grid barrier (none needed after the last window)
        if (n0 + a.W < n_end) {
            ++epoch;
            if (!grid_barrier(a.barrier, static_cast<unsigned int>(epoch), a.err)) return;
        }
    }
}

size_t lif_fast_smem(int tile, int W, int npop, int ndrive, int nproj, int cdf_total, bool dbl) {
    const SmemLayout lay =
        smem_layout(dbl ? sizeof(PopCoef<double>) : sizeof(PopCoef<float>),
                    dbl ? sizeof(ProjDev<double>) : sizeof(ProjDev<float>), npop, ndrive, nproj,
                    cdf_total, tile, W);
    return lay.total;
}

template <typename Real>
cudaError_t launch_lif_fast(const LifArgs<Real> &a, int grid, int block, cudaStream_t st) {
    const size_t smem = lif_fast_smem(a.tile, a.W, a.npop, a.ndrive, a.nproj, a.cdf_total,
                                      sizeof(Real) == 8);
    void *args[] = {const_cast<LifArgs<Real> *>(&a)};
    const void *fn = a.model == 0 ? reinterpret_cast<const void *>(&k_lif_fast<Real, 0>)
                                  : reinterpret_cast<const void *>(&k_lif_fast<Real, 1>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem, st);
}

template cudaError_t launch_lif_fast<float>(const LifArgs<float> &, int, int, cudaStream_t);
template cudaError_t launch_lif_fast<double>(const LifArgs<double> &, int, int, cudaStream_t);

}  // namespace bspk
