// lif_tiled.cu -- persistent windowed kernel for iaf networks with
// target-partitioned delivery and record-based synchronisation (FP32/FP64).
//
// One cooperative launch runs a whole bspk_run, one 256-thread CTA per SM.
// CTA c owns the neurons [c*tile, (c+1)*tile): their state lives in
// registers for the whole run, their arrival ring in shared memory
// (ring_s[slot][t], L = W + max_lag + 1 slots), and so does the CSR index of
// every edge that targets them (rows = all pre neurons).  Time advances in
// windows of W = d_min steps: nothing emitted in a window arrives inside it.
// Per window:
//   A. thread t advances neuron t for W steps from ring_s + the drive buffer;
//      each spike is written, tagged with the window's epoch, into this CTA's
//      64-byte record (count word + 15 entries, overflow area beyond);
//   B. delivery warps read all CTAs' records in one coalesced pass and spin
//      until every word they need carries the current tag (a dataflow
//      barrier: no separate grid barrier, no fences: each 32-bit word is
//      validated by its own tag), then pull each spike's edge segment for
//      this tile (bucket bounds from shared memory, one L2 round trip for
//      all edges) and accumulate with shared-memory atomics; meanwhile the
//      remaining warps draw the next window's Poisson drive.
// Records are double-buffered by window parity: CTA x rewrites its parity-p
// record for window e+2 only after reading every record of window e+1, which
// each CTA writes only after it finished reading window e.  Every poll is
// bounded (2 s of globaltimer), after which the error flag is raised and all
// threads of every CTA leave.
#include "common.cuh"
#include "lif_args.h"

namespace bspk {

namespace {
constexpr int kTabCap2 = 256;
constexpr int kDelivWarps = 5;
constexpr int kDeliv = 32 * kDelivWarps;      // threads that deliver
constexpr int kRecPerHalf = 16;               // records per half-warp: G <= 2*5*16 = 160
constexpr int kListCap = 2048;                // spikes gathered per window and CTA
constexpr int kEdgeUnroll = 16;               // edge loads in flight per thread

__device__ __forceinline__ void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Exclusive scan of s[0..n) by the first nth threads (named barrier `bar`):
// thread t scans a run of ceil(n / nth) consecutive elements, the runs' sums
// are scanned across warps; three barriers whatever n is.  Returns the total.
__device__ int scan_named(int *s, int n, int *s_warp, int nth, int bar) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = nth >> 5;
    const int per = (n + nth - 1) / nth;
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
    named_sync(bar, nth);
    if (wid == 0) {
        int t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) s_warp[lane] = t;
    }
    named_sync(bar, nth);
    int acc = (wid > 0 ? s_warp[wid - 1] : 0) + x - run;
    const int total = s_warp[nw - 1];
    for (int i = b0; i < b1; ++i) {
        const int v = s[i];
        s[i] = acc;
        acc += v;
    }
    named_sync(bar, nth);
    return total;
}

__device__ __forceinline__ int find_pop2(const int *s_off, int npop, int g) {
    int p = 0;
    while (p + 1 < npop && s_off[p + 1] <= g) ++p;
    return p;
}

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint32_t kTagMask = 0xFF000000u;
constexpr uint64_t kPollLimitNs = 2000000000ull;  // 2 s
}  // namespace

template <typename Real, int MODEL>
__global__ void __launch_bounds__(256) k_lif_tiled(const LifArgs<Real> a, const TiledArgs<Real> t2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TiledLayout lay = tiled_layout(sizeof(PopCoef<Real>), sizeof(ProjDev<Real>), sizeof(Real),
                                         a.npop, a.ndrive, a.nproj, a.cdf_total, a.tile, a.L,
                                         gridDim.x, t2.smem_ptr ? a.N + 1 : 0);
    PopCoef<Real> *s_coef = reinterpret_cast<PopCoef<Real> *>(smem_raw + lay.coef);
    DriveDev *s_drive = reinterpret_cast<DriveDev *>(smem_raw + lay.drive);
    ProjDev<Real> *s_proj = reinterpret_cast<ProjDev<Real> *>(smem_raw + lay.proj);
    uint64_t *s_cdf = reinterpret_cast<uint64_t *>(smem_raw + lay.cdf);
    Real *ring_s = reinterpret_cast<Real *>(smem_raw + lay.ring);
    Real *drv_s = reinterpret_cast<Real *>(smem_raw + lay.drv);  // [kMaxWindow][tile]
    uint32_t *s_spk = reinterpret_cast<uint32_t *>(smem_raw + lay.spk);
    int *s_ptr = reinterpret_cast<int *>(smem_raw + lay.ptr);   // this tile's CSR bounds
    __shared__ int s_off[kMaxPops + 1];
    __shared__ int s_drv_ptr[kMaxPops + 1];
    __shared__ int s_drv_list[kTabCap2];
    __shared__ int s_warp[32];
    __shared__ uint32_t s_list[kListCap];  // gathered spikes: pre gid << 5 | step in window
    __shared__ int s_ibeg[kListCap], s_ioff[kListCap + 1];
    __shared__ int s_nsp, s_nlist, s_abort;

    const int tid = threadIdx.x, B = blockDim.x;
    const int G = gridDim.x, c = blockIdx.x;
    const int N = a.N, L = a.L, tile = a.tile;
    const int cta0 = c * tile;
    const int nloc = max(0, min(tile, N - cta0));
    const int *gptr = t2.ptr + static_cast<size_t>(c) * (N + 1);  // this tile's bounds in HBM

    for (int i = tid; i < a.npop; i += B) {
        s_coef[i] = a.coef[i];
        s_off[i] = a.coef[i].off;
    }
    for (int i = tid; i <= a.npop; i += B) s_drv_ptr[i] = a.pop_drive_ptr[i];
    for (int i = tid; i < a.ndrive; i += B) s_drive[i] = a.drives[i];
    for (int i = tid; i < a.nproj; i += B) s_proj[i] = a.projs[i];
    for (int i = tid; i < a.cdf_total; i += B) s_cdf[i] = a.cdf[i];
    if (t2.smem_ptr)
        for (int i = tid; i <= N; i += B) s_ptr[i] = gptr[i];
    // arrival ring of this tile: global [L][N] -> shared [L][tile]
    for (int i = tid; i < L * tile; i += B) {
        const int slot = i / tile, tt = i % tile;
        ring_s[i] = tt < nloc ? a.ring[static_cast<size_t>(slot) * N + cta0 + tt] : Real(0);
    }
    if (tid == 0) s_abort = 0;
    __syncthreads();
    for (int i = tid; i < s_drv_ptr[a.npop] && i < kTabCap2; i += B) s_drv_list[i] = a.pop_drive_list[i];

    // neuron t of this tile lives in thread t's registers for the whole run
    const bool own = tid < nloc;
    const int g = cta0 + tid;
    Real st[6] = {Real(0), Real(0), Real(0), Real(0), Real(0), Real(0)};
    int r = 0, rslot = -1;
    PopCoef<Real> cf{};  // by value: registers, no aliasing with ring_s stores
    if (own) {
        cf = s_coef[find_pop2(s_off, a.npop, g)];
#pragma unroll
        for (int i = 0; i < 6; ++i) st[i] = a.s[i][g];
        r = a.r[g];
        rslot = a.rec_slot ? a.rec_slot[g] : -1;
    }
    // this CTA's region of the spike record (no global atomic on the hot path)
    const int64_t rec_cap = a.spk_cap / G;
    int64_t *my_spk_step = a.spk_step + static_cast<size_t>(c) * rec_cap;
    int32_t *my_spk_gid = a.spk_gid + static_cast<size_t>(c) * rec_cap;
    int64_t rec_n = 0;  // uniform across the CTA
    __syncthreads();

    const int64_t n_end = a.step0 + a.n_steps;
    // Poisson drive of every (step, neuron) pair of the window starting at
    // m0 into drv_s[k][t], four independent threefry chains per thread.
    auto fill_drive = [&](int64_t m0, int Wm, int t0, int nth) {
        const int npairs = Wm * nloc;
        for (int base = 0; base < npairs; base += 4 * nth) {
            int kk[4], tt[4], pp[4];
            Real add[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int idx = base + j * nth + t0;
                kk[j] = idx / (nloc > 0 ? nloc : 1);
                tt[j] = idx - kk[j] * nloc;
                pp[j] = idx < npairs ? find_pop2(s_off, a.npop, cta0 + tt[j]) : -1;
                add[j] = Real(0);
            }
            const int qmax = pp[0] >= 0 ? s_drv_ptr[a.npop] : 0;
            for (int q = 0; q < qmax; ++q) {
                const DriveDev &d = s_drive[s_drv_list[q]];
                uint64_t u[4];
                bool on[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t se = m0 + kk[j] - d.lag;
                    on[j] = pp[j] >= 0 && d.pop == pp[j] && d.tmin < se && se <= d.tmax;
                    u[j] = on[j] ? bits53(d.seed, 0u, static_cast<uint32_t>(se),
                                          static_cast<uint32_t>(cta0 + tt[j] - s_off[pp[j]]))
                                 : 0ull;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (on[j]) {
                        const int cnt = poisson_from_table(s_cdf + d.cdf_off, d.cdf_n, u[j]);
                        add[j] += static_cast<Real>(cnt) * static_cast<Real>(d.weight);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (pp[j] >= 0) drv_s[kk[j] * tile + tt[j]] = add[j];
        }
    };
    fill_drive(a.step0, static_cast<int>((n_end - a.step0) < a.W ? (n_end - a.step0) : a.W), tid, B);
    __syncthreads();

    uint32_t epoch = 0;
    for (int64_t n0 = a.step0; n0 < n_end; n0 += a.W, ++epoch) {
        const int Wk = static_cast<int>((n_end - n0) < a.W ? (n_end - n0) : a.W);
        const int slot0 = static_cast<int>(n0 % L);
        const int par = epoch & 1;
        // tag = (epoch + 1) mod 256 in the top byte: zeroed memory never
        // matches, and the stale record of the same parity (epoch - 2) differs
        const uint32_t tag = ((epoch + 1u) & 0xFFu) << 24;
        uint32_t *rec = t2.list + (static_cast<size_t>(par) * G + c) * kRecWords;
        uint32_t *ovf = t2.ovf + (static_cast<size_t>(par) * G + c) * t2.list_cap;
        if (tid == 0) {
            s_nsp = 0;
            s_nlist = 0;
        }
        __syncthreads();

        // ---- A: neuron updates (rolled loop over the window)
        if (own) {
            int slot = slot0;
            for (int k = 0; k < Wk; ++k) {
                const Real x = ring_s[slot * tile + tid] + drv_s[k * tile + tid];
                ring_s[slot * tile + tid] = Real(0);
                bool sp;
                if (MODEL == 0) sp = iaf_alpha_step<Real>(cf, st, r, x);
                else sp = iaf_exp_step<Real>(cf, st, r, x);
                if (sp) {
                    const int pos = atomicAdd(&s_nsp, 1);
                    const uint32_t ent = (static_cast<uint32_t>(tid) << 5) | static_cast<uint32_t>(k);
                    s_spk[pos] = ent;
                    if (pos < kRecInline) rec[1 + pos] = tag | ent;
                    else ovf[pos - kRecInline] = tag | ent;
                }
                if (rslot >= 0)
                    a.v_out[static_cast<size_t>(n0 + k - a.run_step0) * a.n_rec + rslot] = st[0];
                if (++slot == L) slot = 0;
            }
        }
        __syncthreads();
        const int nsp = s_nsp;
        if (tid == 0) rec[0] = tag | static_cast<uint32_t>(nsp);

        // ---- spike record into this CTA's region (holes for unrecorded neurons)
        for (int i = tid; i < nsp; i += B) {
            const uint32_t e = s_spk[i];
            const int gg = cta0 + static_cast<int>(e >> 5);
            const int64_t at = rec_n + i;
            if (at < rec_cap) {
                const bool kp = a.spk_flag == nullptr || a.spk_flag[gg] != 0;
                my_spk_step[at] = n0 + (e & 31u);
                my_spk_gid[at] = kp ? gg : -1;
            }
        }
        rec_n += nsp;

        // ---- B (delivery warps) || next window's drive (the other warps)
        if (tid < kDeliv) {
            const int lane = tid & 31, wid = tid >> 5;
            const int half = lane >> 4, w = lane & 15;
            // 1. gather: half-warp h of warp v reads records (v + 5 i) * 2 + h,
            //    lane w word w; every polling round issues all of the lane's
            //    loads at once, then validates each record (count word and the
            //    entries it announces must carry the tag); a record's entries
            //    go to s_list once, on the round it validates.
            const uint32_t *recs = t2.list + static_cast<size_t>(par) * G * kRecWords;
            unsigned pend = 0;  // bit i: record of slot i still pending (uniform per half)
#pragma unroll
            for (int i = 0; i < kRecPerHalf; ++i)
                if ((wid + kDelivWarps * i) * 2 + half < G) pend |= 1u << i;
            const uint64_t t_start = gtimer();
            while (__any_sync(0xffffffffu, pend != 0u)) {
                uint32_t word[kRecPerHalf];
#pragma unroll
                for (int i = 0; i < kRecPerHalf; ++i) {
                    const int j = (wid + kDelivWarps * i) * 2 + half;
                    word[i] = (pend >> i) & 1u ? __ldcg(recs + j * kRecWords + w) : 0u;
                }
#pragma unroll
                for (int i = 0; i < kRecPerHalf; ++i) {
                    const int j = (wid + kDelivWarps * i) * 2 + half;
                    const bool pending = (pend >> i) & 1u;
                    const uint32_t head = __shfl_sync(0xffffffffu, word[i], lane & 16);
                    const int cnt = (head & kTagMask) == tag ? static_cast<int>(head & 0xFFFFFFu) : -1;
                    const bool ok = !pending || (cnt >= 0 && (w == 0 || w > cnt ||
                                                              (word[i] & kTagMask) == tag));
                    const unsigned bal = __ballot_sync(0xffffffffu, ok);
                    const bool half_ok = (half ? (bal >> 16) : (bal & 0xFFFFu)) == 0xFFFFu;
                    if (pending && half_ok) {
                        if (w >= 1 && w <= cnt) {
                            const int pos = atomicAdd(&s_nlist, 1);
                            if (pos < kListCap)
                                s_list[pos] = ((static_cast<uint32_t>(j * tile) +
                                                ((word[i] & 0xFFFFFFu) >> 5)) << 5) | (word[i] & 31u);
                        }
                        if (w == 0 && cnt > kRecInline) {  // overflow entries
                            const uint32_t *src =
                                t2.ovf + (static_cast<size_t>(par) * G + j) * t2.list_cap;
                            for (int q = 0; q < cnt - kRecInline; ++q) {
                                uint32_t ow = __ldcg(src + q);
                                const uint64_t tq = gtimer();
                                while ((ow & kTagMask) != tag) {
                                    if (gtimer() - tq > kPollLimitNs) {
                                        atomicExch(a.err, BSPK_DEV_ERR_TIMEOUT);
                                        s_abort = 1;
                                        break;
                                    }
                                    ow = __ldcg(src + q);
                                }
                                const int pos = atomicAdd(&s_nlist, 1);
                                if (pos < kListCap)
                                    s_list[pos] = ((static_cast<uint32_t>(j * tile) +
                                                    ((ow & 0xFFFFFFu) >> 5)) << 5) | (ow & 31u);
                            }
                        }
                        pend &= ~(1u << i);
                    }
                }
                if (__any_sync(0xffffffffu, pend != 0u && gtimer() - t_start > kPollLimitNs)) {
                    if (lane == 0) {
                        atomicExch(a.err, BSPK_DEV_ERR_TIMEOUT);
                        s_abort = 1;
                    }
                    break;
                }
            }
            named_sync(1, kDeliv);
            const int S = min(s_nlist, kListCap);
            if (s_nlist > kListCap && tid == 0) {
                atomicExch(a.err, BSPK_DEV_ERR_OVERFLOW);
                s_abort = 1;
            }
            // 2. bucket bounds of every gathered spike (shared memory when the
            //    tile's CSR index fits there)
            for (int i = tid; i < S; i += kDeliv) {
                const int pre = static_cast<int>(s_list[i] >> 5);
                const int b0 = t2.smem_ptr ? s_ptr[pre] : __ldg(gptr + pre);
                const int b1 = t2.smem_ptr ? s_ptr[pre + 1] : __ldg(gptr + pre + 1);
                s_ibeg[i] = b0;
                s_ioff[i] = b1 - b0;
            }
            named_sync(1, kDeliv);
            const int T = scan_named(s_ioff, S, s_warp, kDeliv, 1);
            if (tid == 0) s_ioff[S] = T;
            named_sync(1, kDeliv);
            // 3. every edge of the window: thread t takes the contiguous slice
            //    [t K, (t+1) K) of the flattened edges, finds its first spike
            //    once, walks forward, and keeps kEdgeUnroll loads in flight
            const int K = (T + kDeliv - 1) / kDeliv;
            const int e_beg = tid * K, e_end = min(T, e_beg + K);
            if (e_beg < e_end) {
                int it = 0, hi = S - 1;
                while (it < hi) {
                    const int mid = (it + hi + 1) >> 1;
                    if (s_ioff[mid] <= e_beg) it = mid; else hi = mid - 1;
                }
                int it_end = s_ioff[it + 1];
                for (int e0 = e_beg; e0 < e_end; e0 += kEdgeUnroll) {
                    int jj[kEdgeUnroll], nm[kEdgeUnroll];
#pragma unroll
                    for (int u = 0; u < kEdgeUnroll; ++u) {
                        const int e = e0 + u;
                        jj[u] = -1;
                        if (e < e_end) {
                            while (e >= it_end) it_end = s_ioff[++it + 1];
                            jj[u] = s_ibeg[it] + (e - s_ioff[it]);
                            const int m = slot0 + static_cast<int>(s_list[it] & 31u);
                            nm[u] = m >= L ? m - L : m;
                        }
                    }
                    uint32_t ed[kEdgeUnroll];
                    Real wv[kEdgeUnroll];
#pragma unroll
                    for (int u = 0; u < kEdgeUnroll; ++u) {
                        if (jj[u] >= 0) {
                            ed[u] = __ldg(t2.edges + jj[u]);
                            wv[u] = t2.w ? __ldg(t2.w + jj[u]) : Real(0);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kEdgeUnroll; ++u) {
                        if (jj[u] >= 0) {
                            if (!t2.w) wv[u] = s_proj[ed[u] >> 24].w0;
                            int slot = nm[u] + static_cast<int>((ed[u] >> 16) & 0xFFu);
                            if (slot >= L) slot -= L;
                            atomicAdd(ring_s + slot * tile + (ed[u] & 0xFFFFu), wv[u]);
                        }
                    }
                }
            }
        } else if (n0 + a.W < n_end) {
            const int64_t m0 = n0 + a.W;
            fill_drive(m0, static_cast<int>((n_end - m0) < a.W ? (n_end - m0) : a.W),
                       tid - kDeliv, B - kDeliv);
        }
        __syncthreads();
        if (s_abort) return;
    }

    // ---- persist state, the tile's ring and this CTA's record count
    if (own) {
#pragma unroll
        for (int i = 0; i < 6; ++i) a.s[i][g] = st[i];
        a.r[g] = r;
    }
    for (int i = tid; i < L * nloc; i += B) {
        const int slot = i / nloc, tt = i % nloc;
        a.ring[static_cast<size_t>(slot) * N + cta0 + tt] = ring_s[slot * tile + tt];
    }
    if (tid == 0) t2.rec_count[c] = rec_n;
}

size_t lif_tiled_smem(int tile, int L, int G, int N, int npop, int ndrive, int nproj,
                      int cdf_total, bool dbl, bool smem_ptr) {
    return tiled_layout(dbl ? sizeof(PopCoef<double>) : sizeof(PopCoef<float>),
                        dbl ? sizeof(ProjDev<double>) : sizeof(ProjDev<float>), dbl ? 8 : 4, npop,
                        ndrive, nproj, cdf_total, tile, L, G, smem_ptr ? N + 1 : 0)
        .total;
}

template <typename Real>
cudaError_t launch_lif_tiled(const LifArgs<Real> &a, const TiledArgs<Real> &t2, int grid,
                             cudaStream_t st) {
    const size_t smem = lif_tiled_smem(a.tile, a.L, grid, a.N, a.npop, a.ndrive, a.nproj,
                                       a.cdf_total, sizeof(Real) == 8, t2.smem_ptr != 0);
    void *args[] = {const_cast<LifArgs<Real> *>(&a), const_cast<TiledArgs<Real> *>(&t2)};
    const void *fn = a.model == 0 ? reinterpret_cast<const void *>(&k_lif_tiled<Real, 0>)
                                  : reinterpret_cast<const void *>(&k_lif_tiled<Real, 1>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, smem, st);
}

template cudaError_t launch_lif_tiled<float>(const LifArgs<float> &, const TiledArgs<float> &, int,
                                             cudaStream_t);
template cudaError_t launch_lif_tiled<double>(const LifArgs<double> &, const TiledArgs<double> &,
                                              int, cudaStream_t);

}  // namespace bspk
