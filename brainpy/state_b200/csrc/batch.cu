// batch.cu -- persistent kernel for a batch of independent iaf networks of
// uneven sizes (instances), one cooperative launch for the whole batch.
//
// CTA c owns a list of tiles (up to T = blockDim.x neurons of one instance
// each, one neuron per thread) and advances them round by round; round r
// moves every tile through window k = floor(step0 / W) + r of its instance
// (W = the instance's arrival lag, so windows of different instances need
// not line up).  One tile-window:
//   1. wait until every tile of the instance published window k - 1
//      (tagged count word with a "complete" bit; bounded poll), gather the
//      entries whose arrival falls into the steps processed now;
//   2. deliver: per gathered spike the bucket of edges that target this
//      tile (CSR over the instance's pre neurons), flattened across threads,
//      shared-memory atomics into the transient accumulator acc[W][T];
//   3. update: each thread advances its neuron through the window's steps
//      (state loaded from HBM at the start, stored at the end), adding the
//      counter-based Poisson drive; spikes become tagged 64-bit record
//      entries ((window + 1) << 32 | pre << 6 | step in window).
// A tile rewrites its parity-p record for window k + 2 only after all tiles
// of the instance completed window k + 1, which each of them does only after
// reading window k, so two record buffers suffice.  Dependencies point to
// the previous window only and every CTA processes windows in order, so the
// co-resident grid cannot deadlock; every poll still gives up after 2 s.
#include <cuda_pipeline.h>

#include <algorithm>

#include "batch_args.h"
#include "common.cuh"

namespace bspk {

namespace {
constexpr int kBListCap = 1024;   // gathered spikes per delivery chunk
constexpr int kBEdgeUnroll = 8;   // edge loads in flight per thread
constexpr uint64_t kBPollNs = 2000000000ull;
constexpr uint32_t kCompleteBit = 0x80000000u;

__device__ __forceinline__ uint64_t gclock() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fix_add(int32_t *p, int32_t v) { atomicAdd(p, v); }
__device__ __forceinline__ void fix_add(long long *p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

// Exclusive scan of s[0..n) by the whole block; returns the total.
__device__ int block_scan_excl(int *s, int n, int *s_warp) {
    const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = T >> 5;
    const int per = (n + T - 1) / T;
    const int b0 = tid * per, b1 = min(n, b0 + per);
    int run = 0;
    for (int i = b0; i < b1; ++i) run += s[i];
    int x = run;
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
        if (lane < nw) s_warp[lane] = t;
    }
    __syncthreads();
    int acc = (wid > 0 ? s_warp[wid - 1] : 0) + x - run;
    const int total = s_warp[nw - 1];
    for (int i = b0; i < b1; ++i) {
        const int v = s[i];
        s[i] = acc;
        acc += v;
    }
    __syncthreads();
    return total;
}
}  // namespace

// FP32: 80 registers per thread let three 256-neuron tiles (CTAs) share an
// SM, whose independent tile-window chains overlap (514 against 548 ms per
// simulated second for the 256-instance sweep with 128 registers, where
// one 512-neuron tile per SM was the best shape); FP64 keeps 128 (80 spills).
template <typename Real>
constexpr int batch_regs() {
    return sizeof(Real) == 4 ? 80 : 128;
}

template <typename Real, int MODEL>
__global__ void __maxnreg__(batch_regs<Real>()) k_lif_batch(const BatchArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using Fix = typename FixOf<Real>::type;
    Fix *acc = reinterpret_cast<Fix *>(smem_raw);  // [Wmax][T], fixed point
    Real *drv_s = reinterpret_cast<Real *>(smem_raw + sizeof(Fix) * a.Wmax * blockDim.x);  // [Wmax][T]
    __shared__ BatchInstDev s_inst;
    __shared__ BatchTileDev s_tile;
    __shared__ Fix s_w[kBatchMaxProj];
    __shared__ uint32_t s_list[kBListCap];  // pre << 6 | arrival step relative to the pass
    __shared__ int s_ibeg[kBListCap], s_ioff[kBListCap + 1];
    __shared__ int s_cnt[kBListCap + 1];    // entries per source tile (then their scan)
    __shared__ int s_warp[32];
    __shared__ int s_nlist, s_nsp, s_nrec, s_base, s_abort;

    const int T = blockDim.x, tid = threadIdx.x, c = blockIdx.x;
    const int tb = a.cta_ptr[c], te = a.cta_ptr[c + 1];
    const int64_t n_end = a.step0 + a.n_steps;
    int64_t rec_n = a.rec_count ? a.rec_count[c] : 0;  // recorded spikes (uniform), across launches
    int loaded = -1;    // instance whose drives/CDF/weights sit in shared memory
    if (tid == 0) s_abort = 0;

    for (int round = 0;; ++round) {
        int any = 0;
        for (int q = tb; q < te; ++q) {
            const int ti = a.cta_tiles[q];
            __syncthreads();
            if (tid == 0) {
                s_tile = a.tiles[ti];
                s_inst = a.inst[s_tile.inst];
            }
            __syncthreads();
            const int W = s_inst.W;
            const int64_t k = a.step0 / W + round;
            const int64_t wa = k * W;
            const int64_t sa = a.step0 > wa ? a.step0 : wa;
            const int64_t sb = n_end < wa + W ? n_end : wa + W;
            if (sa >= sb) continue;  // uniform: every thread read the same words
            any = 1;
            const BatchTileDev tl = s_tile;
            const int n_inst = s_inst.n;
            const int off = static_cast<int>(sa - wa), Wk = static_cast<int>(sb - sa);
            if (tl.inst != loaded) {
                for (int i = tid; i < kBatchMaxProj; i += T) s_w[i] = a.proj_w[s_inst.proj0 + i];
                loaded = tl.inst;
            }
            // this thread's neuron: state in registers for the window
            const bool own = tid < tl.n;
            const int li = tl.first + tid;
            const int64_t g = s_inst.g0 + li;
            Real st[6] = {Real(0), Real(0), Real(0), Real(0), Real(0), Real(0)};
            int r = 0, pop = 0;
            PopCoef<Real> cf{};
            if (own) {
#pragma unroll
                for (int i = 0; i < 6; ++i) st[i] = a.s[i][g];
                r = a.r[g];
                while (pop + 1 < s_inst.npop && s_inst.pop_off[pop + 1] <= li) ++pop;
                cf = a.coef[s_inst.coef0 + pop];
                // this window's drive, staged while the window's arrivals are gathered
                const Real *src = a.drive + (sa - a.drive_step0) * a.n_total + g;
                for (int j = 0; j < Wk; ++j)
                    __pipeline_memcpy_async(drv_s + j * T + tid, src + static_cast<int64_t>(j) * a.n_total,
                                            sizeof(Real));
            }
            __pipeline_commit();
            for (int i = tid; i < Wk * T; i += T) acc[i] = Fix(0);
            if (tid == 0) {
                s_nsp = 0;
                s_nrec = 0;
                s_base = sa > wa ? a.part[ti] : 0;
            }
            __syncthreads();

            // ---- 1 + 2: gather window k - 1 of the instance and deliver
            if (k >= 1) {
                const int P = s_inst.ntiles, cap = s_inst.rec_cap;
                const uint32_t tagp = static_cast<uint32_t>(k);  // (k - 1) + 1
                const int par = static_cast<int>((k - 1) & 1);
                const unsigned long long *rbase = a.recs + s_inst.rec0;
                for (int j = tid; j < P; j += T) {
                    const unsigned long long *cw = rbase + static_cast<int64_t>(2 * j + par) * (1 + cap);
                    unsigned long long w = ld_relaxed(cw);
                    const uint64_t t0 = gclock();
                    while (static_cast<uint32_t>(w >> 32) != tagp || !(static_cast<uint32_t>(w) & kCompleteBit)) {
                        if (gclock() - t0 > kBPollNs || *(volatile int *)a.err) {
                            atomicCAS(a.err, 0, BSPK_DEV_ERR_TIMEOUT);
                            s_abort = 1;
                            break;
                        }
                        w = ld_relaxed(cw);
                    }
                    s_cnt[j] = static_cast<int>(static_cast<uint32_t>(w) & ~kCompleteBit);
                }
                __syncthreads();
                if (s_abort) return;
                const int total = block_scan_excl(s_cnt, P, s_warp);
                if (tid == 0) s_cnt[P] = total;
                for (int q0 = 0; q0 < total; q0 += kBListCap) {
                    const int qn = min(kBListCap, total - q0);
                    if (tid == 0) s_nlist = 0;
                    __syncthreads();
                    for (int i = tid; i < qn; i += T) {
                        const int qq = q0 + i;
                        int lo = 0, hi = P - 1;  // last source tile with s_cnt[j] <= qq
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s_cnt[mid] <= qq) lo = mid; else hi = mid - 1;
                        }
                        const unsigned long long *ew =
                            rbase + static_cast<int64_t>(2 * lo + par) * (1 + cap) + 1 + (qq - s_cnt[lo]);
                        unsigned long long w = ld_relaxed(ew);
                        const uint64_t t0 = gclock();
                        bool ok = true;
                        while (static_cast<uint32_t>(w >> 32) != tagp) {
                            if (gclock() - t0 > kBPollNs || *(volatile int *)a.err) {
                                atomicCAS(a.err, 0, BSPK_DEV_ERR_TIMEOUT);
                                s_abort = 1;
                                ok = false;
                                break;
                            }
                            w = ld_relaxed(ew);
                        }
                        const uint32_t pay = static_cast<uint32_t>(w);
                        const int stp = static_cast<int>(pay & ((1u << kBatchStepBits) - 1u));
                        if (ok && stp >= off && stp < off + Wk) {
                            const int pos = atomicAdd(&s_nlist, 1);
                            s_list[pos] = (pay & ~((1u << kBatchStepBits) - 1u)) | static_cast<uint32_t>(stp - off);
                        }
                    }
                    __syncthreads();
                    if (s_abort) return;
                    const int S = s_nlist;
                    const int *tptr = a.ptr + s_inst.ptr0 + static_cast<int64_t>(tl.tloc) * n_inst;
                    for (int i = tid; i < S; i += T) {
                        const int pre = static_cast<int>(s_list[i] >> kBatchStepBits);
                        const int b0 = __ldg(tptr + pre), b1 = __ldg(tptr + pre + 1);
                        s_ibeg[i] = b0;
                        s_ioff[i] = b1 - b0;
                    }
                    __syncthreads();
                    const int Tot = block_scan_excl(s_ioff, S, s_warp);
                    if (tid == 0) s_ioff[S] = Tot;
                    __syncthreads();
                    const uint32_t *edges = a.edges + s_inst.edge0;
                    const int per = (Tot + T - 1) / T;
                    const int e_beg = tid * per, e_end = min(Tot, e_beg + per);
                    if (e_beg < e_end) {
                        int it = 0, hi = S - 1;
                        while (it < hi) {
                            const int mid = (it + hi + 1) >> 1;
                            if (s_ioff[mid] <= e_beg) it = mid; else hi = mid - 1;
                        }
                        int it_end = s_ioff[it + 1];
                        for (int e0 = e_beg; e0 < e_end; e0 += kBEdgeUnroll) {
                            int jj[kBEdgeUnroll], sl[kBEdgeUnroll];
#pragma unroll
                            for (int u = 0; u < kBEdgeUnroll; ++u) {
                                const int e = e0 + u;
                                jj[u] = -1;
                                sl[u] = 0;
                                if (e < e_end) {
                                    while (e >= it_end) it_end = s_ioff[++it + 1];
                                    jj[u] = s_ibeg[it] + (e - s_ioff[it]);
                                    sl[u] = static_cast<int>(s_list[it] & ((1u << kBatchStepBits) - 1u));
                                }
                            }
                            uint32_t ed[kBEdgeUnroll];
#pragma unroll
                            for (int u = 0; u < kBEdgeUnroll; ++u)
                                if (jj[u] >= 0) ed[u] = __ldg(edges + jj[u]);
#pragma unroll
                            for (int u = 0; u < kBEdgeUnroll; ++u)
                                if (jj[u] >= 0)
                                    fix_add(acc + sl[u] * T + static_cast<int>(ed[u] & 0xFFFFu),
                                            s_w[ed[u] >> 16]);
                        }
                    }
                    __syncthreads();
                }
            }

            // ---- 3: updates of the processed steps
            const int cap = s_inst.rec_cap;
            unsigned long long *own_rec =
                a.recs + s_inst.rec0 + static_cast<int64_t>(2 * tl.tloc + (k & 1)) * (1 + cap);
            const unsigned long long tag = static_cast<unsigned long long>(k + 1) << 32;
            int nsp_local = 0;
            __pipeline_wait_prior(0);
            if (own) {
                for (int j = 0; j < Wk; ++j) {
                    const int64_t n = sa + j;
                    const Real x = static_cast<Real>(acc[j * T + tid]) * static_cast<Real>(s_inst.inv_scale) +
                                   drv_s[j * T + tid];
                    bool sp;
                    if (MODEL == 0) sp = iaf_alpha_step<Real>(cf, st, r, x);
                    else sp = iaf_exp_step<Real>(cf, st, r, x);
                    if (sp) {
                        ++nsp_local;
                        const int at = s_base + atomicAdd(&s_nsp, 1);
                        if (at < cap)
                            own_rec[1 + at] = tag | (static_cast<uint32_t>(li) << kBatchStepBits) |
                                              static_cast<uint32_t>(off + j);
                        if (s_inst.record) {
                            const int64_t rp = rec_n + atomicAdd(&s_nrec, 1);
                            if (rp < a.spk_cap) {
                                const int64_t o = static_cast<int64_t>(c) * a.spk_cap + rp;
                                a.spk_step[o] = n;
                                a.spk_id[o] = li;
                                a.spk_inst[o] = tl.inst;
                            }
                        }
                    }
                }
#pragma unroll
                for (int i = 0; i < 6; ++i) a.s[i][g] = st[i];
                a.r[g] = r;
                if (nsp_local) a.spk_cnt[g] += static_cast<unsigned int>(nsp_local);
            }
            __syncthreads();
            if (tid == 0) {
                const int tot = s_base + s_nsp;
                if (tot > cap) {
                    atomicCAS(a.err, 0, BSPK_DEV_ERR_OVERFLOW);
                    s_abort = 1;
                }
                const bool complete = sb == wa + W;
                own_rec[0] = tag | (complete ? kCompleteBit : 0u) | static_cast<uint32_t>(min(tot, cap));
                if (!complete) a.part[ti] = min(tot, cap);
            }
            rec_n += s_nrec;
            __syncthreads();
            if (s_abort) return;
        }
        if (!any) break;
    }
    if (tid == 0 && a.rec_count) a.rec_count[c] = rec_n;
}

size_t lif_batch_smem(int T, int Wmax, int dbl) {
    return static_cast<size_t>(T) * Wmax * (dbl ? 16 : 8);  // fixed-point arrivals + drive
}

// Drive pass: thread per neuron over a run of steps.  out[(m - m0) N + g] =
// sum over the drives of g's population (creation order) of count * weight,
// count by CDF inversion of threefry((seed, 0), (m - lag, index in pop)).
template <typename Real>
__global__ void __launch_bounds__(256) k_batch_drive_fill(const BatchArgs<Real> a, int64_t m0, int n,
                                                          int spb, Real *out) {
    const int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (g >= a.n_total) return;
    int lo = 0, hi = a.n_inst - 1;  // instance of g: last with g0 <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.inst[mid].g0 <= g) lo = mid; else hi = mid - 1;
    }
    const BatchInstDev &I = a.inst[lo];
    const int li = static_cast<int>(g - I.g0);
    int pop = 0;
    while (pop + 1 < I.npop && I.pop_off[pop + 1] <= li) ++pop;
    const uint32_t idx = static_cast<uint32_t>(li - I.pop_off[pop]);
    const int k0 = blockIdx.y * spb, k1 = min(n, k0 + spb);
    int nmatch = 0, dsel = 0;
    for (int d = 0; d < I.ndrive; ++d)
        if (a.drives[I.drive0 + d].pop == pop) {
            ++nmatch;
            dsel = d;
        }
    if (nmatch == 1) {
        // one drive for this population (the sweep's case): descriptor and
        // first CDF thresholds in registers, counts as in the general path
        const DriveDev D = a.drives[I.drive0 + dsel];
        const uint64_t *T = a.cdf + I.cdf0 + D.cdf_off;
        constexpr uint64_t kNone = ~0ull;  // no threshold: never below a 53-bit draw
        const uint64_t T0 = D.cdf_n > 0 ? T[0] : kNone, T1 = D.cdf_n > 1 ? T[1] : kNone,
                       T2 = D.cdf_n > 2 ? T[2] : kNone, T3 = D.cdf_n > 3 ? T[3] : kNone;
        const Real wd = static_cast<Real>(D.weight);
        for (int k = k0; k < k1; ++k) {
            const int64_t se = m0 + k - D.lag;
            Real add = Real(0);
            if (D.tmin < se && se <= D.tmax) {
                const uint64_t u = bits53(D.seed, 0u, static_cast<uint32_t>(se), idx);
                int cnt;
                if (u > T3) {
                    cnt = 4;
                    while (cnt < D.cdf_n && u > T[cnt]) ++cnt;
                } else {
                    cnt = (u > T0) + (u > T1) + (u > T2);
                }
                add += static_cast<Real>(cnt) * wd;
            }
            out[static_cast<int64_t>(k) * a.n_total + g] = add;
        }
        return;
    }
    for (int k = k0; k < k1; ++k) {
        const int64_t m = m0 + k;
        Real add = Real(0);
        for (int d = 0; d < I.ndrive; ++d) {
            const DriveDev &D = a.drives[I.drive0 + d];
            const int64_t se = m - D.lag;
            if (D.pop == pop && D.tmin < se && se <= D.tmax) {
                const uint64_t u = bits53(D.seed, 0u, static_cast<uint32_t>(se), idx);
                const int cnt = poisson_from_table(a.cdf + I.cdf0 + D.cdf_off, D.cdf_n, u);
                add += static_cast<Real>(cnt) * static_cast<Real>(D.weight);
            }
        }
        out[static_cast<int64_t>(k) * a.n_total + g] = add;
    }
}

template <typename Real>
cudaError_t launch_batch_drive_fill(const BatchArgs<Real> &a, int64_t m0, int n, Real *out,
                                    cudaStream_t st) {
    if (n <= 0 || a.n_total <= 0) return cudaSuccess;
    const int64_t gx = (a.n_total + 255) / 256;
    if (gx > 2147483647) return cudaErrorInvalidValue;
    const int gy = static_cast<int>(std::min<int64_t>(std::max<int64_t>(1, (148 * 16 + gx - 1) / gx),
                                                      std::min(n, 65535)));
    const int spb = (n + gy - 1) / gy;
    k_batch_drive_fill<Real><<<dim3(static_cast<unsigned>(gx), (n + spb - 1) / spb), 256, 0, st>>>(
        a, m0, n, spb, out);
    return cudaGetLastError();
}

template cudaError_t launch_batch_drive_fill<float>(const BatchArgs<float> &, int64_t, int, float *,
                                                    cudaStream_t);
template cudaError_t launch_batch_drive_fill<double>(const BatchArgs<double> &, int64_t, int,
                                                     double *, cudaStream_t);

template <typename Real>
cudaError_t launch_lif_batch(const BatchArgs<Real> &a, int model, int grid, cudaStream_t st) {
    const size_t smem = lif_batch_smem(a.T, a.Wmax, sizeof(Real) == 8);
    void *args[] = {const_cast<BatchArgs<Real> *>(&a)};
    const void *fn = model == 0 ? reinterpret_cast<const void *>(&k_lif_batch<Real, 0>)
                                : reinterpret_cast<const void *>(&k_lif_batch<Real, 1>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(a.T), args, smem, st);
}

template <typename Real>
int lif_batch_max_ctas_per_sm(int model, int T, int Wmax) {
    const size_t smem = lif_batch_smem(T, Wmax, sizeof(Real) == 8);
    const void *fn = model == 0 ? reinterpret_cast<const void *>(&k_lif_batch<Real, 0>)
                                : reinterpret_cast<const void *>(&k_lif_batch<Real, 1>);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, T, smem) != cudaSuccess) return 0;
    return nb;
}

template cudaError_t launch_lif_batch<float>(const BatchArgs<float> &, int, int, cudaStream_t);
template cudaError_t launch_lif_batch<double>(const BatchArgs<double> &, int, int, cudaStream_t);
template int lif_batch_max_ctas_per_sm<float>(int, int, int);
template int lif_batch_max_ctas_per_sm<double>(int, int, int);

}  // namespace bspk
