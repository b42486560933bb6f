// lif_exact.cu -- deterministic FP64 kernel for iaf networks with the
// reference Simulator's timing (compiled with -fmad=false: every multiply and
// add is rounded separately, as in the reference's float64 arithmetic).
//
// Delivery is a pull over in-edges instead of atomics, so the summation order
// is fixed: for every post neuron and step, each projection's contributions
// are summed in ascending pre order (the order of a serial CSR scatter,
// _nest_network/projections.py:56-59), and the projections' vectors are added
// to the input in creation order (sum_delta_inputs, _base.py:312-382).  The
// pre spike trains come from a 64-step history word per neuron, so a window of
// W steps reads each in-edge once.  Requires max_lag + W <= 64.
#include <mutex>
#include <vector>

#include "common.cuh"
#include "lif_args.h"
#include "plan_internal.h"

namespace bspk {

__device__ __forceinline__ uint64_t rotr64(uint64_t x, int s) {
    s &= 63;
    return s == 0 ? x : (x >> s) | (x << (64 - s));
}

template <int MODEL>
__global__ void __launch_bounds__(256) k_lif_exact(const LifArgs<double> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemLayout lay = smem_layout(sizeof(PopCoef<double>), sizeof(ProjDev<double>), a.npop,
                                       a.ndrive, a.nproj, a.cdf_total, 0, 0);
    PopCoef<double> *s_coef = reinterpret_cast<PopCoef<double> *>(smem_raw + lay.coef);
    DriveDev *s_drive = reinterpret_cast<DriveDev *>(smem_raw + lay.drive);
    ProjDev<double> *s_proj = reinterpret_cast<ProjDev<double> *>(smem_raw + lay.proj);
    uint64_t *s_cdf = reinterpret_cast<uint64_t *>(smem_raw + lay.cdf);
    double *ybuf = reinterpret_cast<double *>(smem_raw + lay.total);  // [kMaxWindow][block]

    const int tid = threadIdx.x, B = blockDim.x;
    for (int i = tid; i < a.npop; i += B) s_coef[i] = a.coef[i];
    for (int i = tid; i < a.ndrive; i += B) s_drive[i] = a.drives[i];
    for (int i = tid; i < a.nproj; i += B) s_proj[i] = a.projs[i];
    for (int i = tid; i < a.cdf_total; i += B) s_cdf[i] = a.cdf[i];
    for (int k = 0; k < kMaxWindow; ++k) ybuf[k * B + tid] = 0.0;
    __syncthreads();

    const int N = a.N;
    const int cta0 = blockIdx.x * a.tile;
    const int cta1 = min(cta0 + a.tile, N);
    const int64_t n_end = a.step0 + a.n_steps;
    int epoch = 0;

    for (int64_t n0 = a.step0; n0 < n_end; n0 += a.W) {
        const int Wk = static_cast<int>((n_end - n0) < a.W ? (n_end - n0) : a.W);
        const uint64_t wmask = Wk >= 64 ? ~0ull : ((1ull << Wk) - 1ull);
        for (int g = cta0 + tid; g < cta1; g += B) {
            int p = 0;
            while (p + 1 < a.npop && s_coef[p + 1].off <= g) ++p;
            const PopCoef<double> &c = s_coef[p];
            const int gl = g - c.off;
            double tot[kMaxWindow];
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k) tot[k] = 0.0;
            for (int q = a.pop_in_ptr[p]; q < a.pop_in_ptr[p + 1]; ++q) {
                const int id = a.pop_in_list[q];
                if (id < 0) {  // Poisson drive: y = count * weight
                    const DriveDev &d = s_drive[-id - 1];
#pragma unroll
                    for (int k = 0; k < kMaxWindow; ++k) {
                        if (k < Wk) {
                            const int64_t se = n0 + k - d.lag;
                            double y = 0.0;
                            if (d.tmin < se && se <= d.tmax) {
                                const uint64_t u = bits53(d.seed, 0u, static_cast<uint32_t>(se),
                                                           static_cast<uint32_t>(gl));
                                const int cnt = poisson_from_table(s_cdf + d.cdf_off, d.cdf_n, u);
                                y = static_cast<double>(cnt) * d.weight;
                            }
                            tot[k] = tot[k] + y;
                        }
                    }
                    continue;
                }
                const ProjDev<double> &P = s_proj[id];
                const int pre_off = s_coef[P.pre_pop].off;
                const int64_t beg = P.cindptr[gl], end = P.cindptr[gl + 1];
                for (int64_t e = beg; e < end; ++e) {
                    const uint32_t ed = __ldg(P.cedges + e);
                    const int pre = static_cast<int>(ed & kEdgePostMask);
                    const int lag = static_cast<int>(ed >> kEdgeDelayShift);
                    const int64_t m0 = n0 - lag;  // step whose spike arrives at n0
                    uint64_t bits = rotr64(__ldcg(a.hist + pre_off + pre),
                                           static_cast<int>(((m0 % 64) + 64) % 64)) & wmask;
                    if (m0 < 0) bits &= m0 <= -64 ? 0ull : ~((1ull << (-m0)) - 1ull);
                    if (!bits) continue;
                    const double w = P.homogeneous ? P.w0 : __ldg(P.cw + e);
                    while (bits) {
                        const int k = __ffsll(static_cast<long long>(bits)) - 1;
                        bits &= bits - 1ull;
                        ybuf[k * B + tid] = ybuf[k * B + tid] + w;
                    }
                }
#pragma unroll
                for (int k = 0; k < kMaxWindow; ++k) {
                    if (k < Wk) {
                        tot[k] = tot[k] + ybuf[k * B + tid];
                        ybuf[k * B + tid] = 0.0;
                    }
                }
            }
            double st[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) st[i] = a.s[i][g];
            int r = a.r[g];
            uint64_t h = a.hist[g];
            const int rslot = a.rec_slot ? a.rec_slot[g] : -1;
            const bool keep = a.spk_flag == nullptr || a.spk_flag[g] != 0;
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k) {
                if (k < Wk) {
                    bool sp;
                    if (MODEL == 0) sp = iaf_alpha_step<double>(c, st, r, tot[k]);
                    else sp = iaf_exp_step<double>(c, st, r, tot[k]);
                    const int bit = static_cast<int>((n0 + k) & 63);
                    h = (h & ~(1ull << bit)) | (static_cast<uint64_t>(sp) << bit);
                    if (sp && keep) {
                        const unsigned long long at = atomicAdd(a.spk_count, 1ull);
                        if (at < static_cast<unsigned long long>(a.spk_cap)) {
                            a.spk_step[at] = n0 + k;
                            a.spk_gid[at] = g;
                        }
                    }
                    if (rslot >= 0)
                        a.v_out[static_cast<size_t>(n0 + k - a.run_step0) * a.n_rec + rslot] = st[0];
                }
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) a.s[i][g] = st[i];
            a.r[g] = r;
            a.hist[g] = h;
        }
        if (n0 + a.W < n_end) {
            ++epoch;
            if (!grid_barrier(a.barrier, static_cast<unsigned int>(epoch), a.err)) return;
        }
    }
}

size_t lif_exact_smem(int block, int npop, int ndrive, int nproj, int cdf_total) {
    const SmemLayout lay = smem_layout(sizeof(PopCoef<double>), sizeof(ProjDev<double>), npop,
                                       ndrive, nproj, cdf_total, 0, 0);
    return lay.total + sizeof(double) * kMaxWindow * static_cast<size_t>(block);
}

cudaError_t launch_lif_exact(const LifArgs<double> &a, int grid, int block, cudaStream_t st) {
    const size_t smem = lif_exact_smem(block, a.npop, a.ndrive, a.nproj, a.cdf_total);
    void *args[] = {const_cast<LifArgs<double> *>(&a)};
    const void *fn = a.model == 0 ? reinterpret_cast<const void *>(&k_lif_exact<0>)
                                  : reinterpret_cast<const void *>(&k_lif_exact<1>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem, st);
}

}  // namespace bspk
