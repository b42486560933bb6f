// lif_fast.cu -- persistent windowed kernel for iaf_psc_alpha / iaf_psc_exp
// networks (FP32 or FP64, atomics-order delivery).
//
// One cooperative launch runs a whole bspk_run.  Time is cut into windows of
// W = d_min steps (the smallest arrival lag of any edge): no spike emitted
// inside a window can arrive inside it, so every neuron advances W steps
// without hearing from any other CTA.  Per window:
//   A. each CTA updates its tile of neurons for W steps: ring slots are read
//      with L2-only loads and cleared, the Poisson drive is drawn in-register
//      (threefry counter RNG + CDF table in shared memory), spikes go to a
//      shared-memory list;
//   B. the CTA scatters its own spikes over their CSR rows with red.add into
//      ring slot (n + lag) mod L (all threads of the CTA stride over a row);
//   C. one bounded grid barrier.
// L >= W + max_lag, so B of window k never aliases a slot A of window k reads.
#include <cooperative_groups.h>

#include "common.cuh"
#include "lif_args.h"

namespace bspk {

template <typename Real, int MODEL>
__global__ void __launch_bounds__(512) k_lif_fast(const LifArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemLayout lay = smem_layout(sizeof(PopCoef<Real>), sizeof(ProjDev<Real>), a.npop,
                                       a.ndrive, a.nproj, a.cdf_total, a.tile, a.W);
    PopCoef<Real> *s_coef = reinterpret_cast<PopCoef<Real> *>(smem_raw + lay.coef);
    DriveDev *s_drive = reinterpret_cast<DriveDev *>(smem_raw + lay.drive);
    ProjDev<Real> *s_proj = reinterpret_cast<ProjDev<Real> *>(smem_raw + lay.proj);
    double *s_cdf = reinterpret_cast<double *>(smem_raw + lay.cdf);
    uint32_t *s_spk = reinterpret_cast<uint32_t *>(smem_raw + lay.spk);
    __shared__ int s_nsp;
    __shared__ unsigned long long s_base;

    const int tid = threadIdx.x;
    for (int i = tid; i < a.npop; i += blockDim.x) s_coef[i] = a.coef[i];
    for (int i = tid; i < a.ndrive; i += blockDim.x) s_drive[i] = a.drives[i];
    for (int i = tid; i < a.nproj; i += blockDim.x) s_proj[i] = a.projs[i];
    for (int i = tid; i < a.cdf_total; i += blockDim.x) s_cdf[i] = a.cdf[i];
    __syncthreads();

    const int N = a.N, L = a.L;
    const int cta0 = blockIdx.x * a.tile;
    const int cta1 = min(cta0 + a.tile, N);
    const int64_t n_end = a.step0 + a.n_steps;
    int epoch = 0;

    for (int64_t n0 = a.step0; n0 < n_end; n0 += a.W) {
        const int Wk = static_cast<int>((n_end - n0) < a.W ? (n_end - n0) : a.W);
        if (tid == 0) s_nsp = 0;
        __syncthreads();
        const int slot0 = static_cast<int>(n0 % L);

        // ---- A: neuron updates for Wk steps
        for (int g = cta0 + tid; g < cta1; g += blockDim.x) {
            int p = 0;
            while (p + 1 < a.npop && s_coef[p + 1].off <= g) ++p;
            const PopCoef<Real> &c = s_coef[p];
            Real st[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) st[i] = a.s[i][g];
            int r = a.r[g];
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
            for (int q = a.pop_drive_ptr[p]; q < a.pop_drive_ptr[p + 1]; ++q) {
                const DriveDev &d = s_drive[a.pop_drive_list[q]];
                const uint32_t idx = static_cast<uint32_t>(g - c.off);
                const Real w = static_cast<Real>(d.weight);
#pragma unroll
                for (int k = 0; k < kMaxWindow; ++k) {
                    if (k < Wk) {
                        const int64_t se = n0 + k - d.lag;
                        if (d.tmin < se && se <= d.tmax) {
                            const double u = uniform01(d.seed, 0u, static_cast<uint32_t>(se), idx);
                            const int cnt = poisson_from_table(s_cdf + d.cdf_off, d.cdf_n, u);
                            in[k] += static_cast<Real>(cnt) * w;
                        }
                    }
                }
            }
            const int rslot = a.rec_slot ? a.rec_slot[g] : -1;
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

        // ---- spike record (all spikes of flagged neurons)
        if (nsp > 0) {
            if (tid == 0) s_base = atomicAdd(a.spk_count, static_cast<unsigned long long>(nsp));
            __syncthreads();
            for (int i = tid; i < nsp; i += blockDim.x) {
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

        // ---- B: scatter own spikes, whole CTA strides over each row
        for (int i = 0; i < nsp; ++i) {
            const uint32_t e = s_spk[i];
            const int g = cta0 + static_cast<int>(e >> 5);
            const int k = static_cast<int>(e & 31u);
            int p = 0;
            while (p + 1 < a.npop && s_coef[p + 1].off <= g) ++p;
            const int gl = g - s_coef[p].off;
            int nmod = slot0 + k;
            if (nmod >= L) nmod -= L;
            for (int q = a.pop_out_ptr[p]; q < a.pop_out_ptr[p + 1]; ++q) {
                const ProjDev<Real> &P = s_proj[a.pop_out_list[q]];
                const int64_t beg = __ldg(P.indptr + gl), end = __ldg(P.indptr + gl + 1);
                Real *base = a.ring + P.post_off;
                for (int64_t j = beg + tid; j < end; j += blockDim.x) {
                    const uint32_t ed = __ldg(P.edges + j);
                    int slot = nmod + static_cast<int>(ed >> kEdgeDelayShift);
                    if (slot >= L) slot -= L;
                    const Real w = P.homogeneous ? P.w0 : __ldg(P.w + j);
                    atomicAdd(base + static_cast<size_t>(slot) * N + (ed & kEdgePostMask), w);
                }
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
