// lif_tiled.cu -- persistent windowed kernel for iaf networks with
// target-partitioned delivery and record-based synchronisation (FP32/FP64).
//
// One cooperative launch runs a stretch of steps, one 512-thread CTA per SM.
// CTA c owns the neurons [c*tile, (c+1)*tile): their state lives in
// registers for the whole launch, their arrival ring in shared memory
// (ring_s[slot][t], L slots), and so does the CSR index of every edge that
// targets them (rows = all pre neurons).  The Poisson drive of the launch is
// drawn beforehand by k_drive_fill (a full-GPU pass over (step, neuron)) and
// streamed into shared memory one window ahead with cp.async.
//
// Time advances in windows of W steps.  When the smallest arrival lag is at
// least 2 W ("pipelined"), a window's spikes are delivered one window late:
// iteration j updates window j, publishes its spikes, then delivers window
// j - 1, whose arrivals all fall in window j + 1 or later.  The records of
// window j - 1 were published by every CTA a whole iteration earlier, so the
// poll rarely waits and its first loads are issued before the update.
// Otherwise (lag < 2) iteration j delivers window j itself.
// Per window:
//   update: thread t advances neuron t through the window's steps from
//      ring_s + the drive; each spike becomes a tagged entry of this CTA's
//      64-byte record (count word + 15 entries, overflow area beyond), and the
//      unused entries are rewritten with the window's tag too;
//   deliver: all warps read all CTAs' records of the window in one coalesced
//      pass and spin until every word they need carries the window's tag
//      (each 32-bit word is validated by its own 18-bit tag: no grid barrier,
//      no fences), then pull each spike's edge segment for this tile (bounds
//      from shared memory, one L2 round trip for all edges) and accumulate
//      with shared-memory atomics.
// Records rotate over 4 buffers: CTA x writes the buffer of window j + 4
// only after its own delivery of window j + 2, which waited for every CTA to
// publish window j + 2, which each does only after finishing its delivery of
// window j.  Every poll is bounded (2 s of globaltimer), after which the
// error flag is raised and all threads of every CTA leave.
#include <cuda_pipeline.h>

#include <algorithm>

#include "common.cuh"
#include "lif_args.h"

namespace bspk {

namespace {
constexpr int kMaxCtas = 160;                 // G <= 160 CTAs, one per SM
constexpr int kListCap = 2048;                // spikes gathered per window and CTA
constexpr int kEdgeUnroll = 8;                // edge loads in flight per thread
constexpr int kUpd = 2;                       // window steps whose inputs sit in registers
constexpr int kEdgeCap = 4096;                // flattened edges mapped per pass
constexpr int kTagShift = 14;                 // word = tag (18 bits) << 14 | payload
constexpr uint32_t kPayMask = (1u << kTagShift) - 1u;
constexpr uint32_t kTagMask = ~kPayMask;
constexpr uint64_t kPollLimitNs = 2000000000ull;  // 2 s

// Exclusive scan of s[0..n) by the whole block that also writes s[n] = total
// and, for the flattened edges below `cap`, the spike of each edge into espk.
// Returns the total.
__device__ int block_scan_map(int *s, int n, int *s_warp, uint16_t *espk, int cap) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    const int per = (n + blockDim.x - 1) / blockDim.x;
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
        for (int q = acc; q < min(acc + v, cap); ++q) espk[q] = static_cast<uint16_t>(i);
        acc += v;
    }
    if (tid == 0) s[n] = total;
    __syncthreads();
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

__device__ __forceinline__ void fix_add(int32_t *p, int32_t v) { atomicAdd(p, v); }
__device__ __forceinline__ void fix_add(long long *p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

__device__ __forceinline__ uint32_t tag_of(int64_t window) {
    return (static_cast<uint32_t>(window + 1) & 0x3FFFFu) << kTagShift;
}
}  // namespace

// Poisson drive of steps [m0, m0 + n): out[(m - m0) * N + g] = sum over the
// drives of g's population (creation order) of count * weight, the count
// drawn by CDF inversion of threefry((seed, 0), (m - lag, index in pop)).
// Block (x, y) covers neurons [256 x, 256 x + 256) over the steps
// [y spb, (y + 1) spb): one thread per neuron, its population and drives
// looked up once, stores coalesced along neurons.
template <typename Real>
__global__ void __launch_bounds__(256) k_drive_fill(const LifArgs<Real> a, int64_t m0, int n, int spb,
                                                    Real *out) {
    __shared__ int s_off[kMaxPops + 1];
    for (int i = threadIdx.x; i < a.npop; i += blockDim.x) s_off[i] = a.coef[i].off;
    if (threadIdx.x == 0) s_off[a.npop] = a.N;
    __syncthreads();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = g < a.N;
    const int gc = valid ? g : a.N - 1;  // a lane beyond the network looks up the last neuron
    const int k0 = blockIdx.y * spb, k1 = min(n, k0 + spb);
    const int p = find_pop2(s_off, a.npop, gc);
    const uint32_t idx = static_cast<uint32_t>(gc - s_off[p]);
    const int q0 = a.pop_drive_ptr[p], q1 = a.pop_drive_ptr[p + 1];
    {
        // The reference kernel path's stream (kind 1) draws a step's numbers
        // for a block of 1024 units from one step key, fold(fold(block key,
        // step), trial): two threefry rounds that every lane of a warp would
        // repeat.  When all 32 lanes have one such drive with the same block
        // key, lag and window, lane l derives the step key of step kc + l and
        // the warp shares the 32 keys by shuffles: one threefry per draw.
        constexpr unsigned kFull = 0xffffffffu;
        const bool one = q1 - q0 == 1;
        DriveDev d{};
        if (one) d = a.drives[a.pop_drive_list[q0]];
        const uint64_t unit = static_cast<uint64_t>(d.unit_off) + idx;
        uint32_t kb0 = d.key0, kb1 = d.key1;
        const bool keyed = one && d.kind == 1;
        if (keyed) fold_key(kb0, kb1, static_cast<uint32_t>(unit >> 10));
        const uint32_t r0 = __shfl_sync(kFull, kb0, 0), r1 = __shfl_sync(kFull, kb1, 0);
        const int lag0 = __shfl_sync(kFull, d.lag, 0);
        const long long tmin0 = __shfl_sync(kFull, static_cast<long long>(d.tmin), 0);
        const long long tmax0 = __shfl_sync(kFull, static_cast<long long>(d.tmax), 0);
        if (__all_sync(kFull, keyed && kb0 == r0 && kb1 == r1 && d.lag == lag0 &&
                                  d.tmin == tmin0 && d.tmax == tmax0)) {
            const int lane = threadIdx.x & 31;
            const uint64_t *T = a.cdf + d.cdf_off;
            constexpr uint64_t kNone = ~0ull;
            const uint64_t T0 = d.cdf_n > 0 ? T[0] : kNone, T1 = d.cdf_n > 1 ? T[1] : kNone,
                           T2 = d.cdf_n > 2 ? T[2] : kNone, T3 = d.cdf_n > 3 ? T[3] : kNone;
            const Real wd = static_cast<Real>(d.weight);
            const uint32_t ln = static_cast<uint32_t>(unit & 1023u);
            for (int kc = k0; kc < k1; kc += 32) {
                uint32_t s0 = kb0, s1 = kb1;
                fold_key(s0, s1, static_cast<uint32_t>(m0 + kc + lane - lag0));
                fold_key(s0, s1, d.trial);
                const int kend = min(32, k1 - kc);
                for (int j = 0; j < kend; ++j) {
                    const uint32_t t0 = __shfl_sync(kFull, s0, j), t1 = __shfl_sync(kFull, s1, j);
                    const int64_t se = m0 + kc + j - lag0;
                    Real add = Real(0);
                    if (tmin0 < se && se <= tmax0) {
                        uint32_t y0, y1;
                        threefry2x32(t0, t1, 0u, ln, y0, y1);
                        const uint64_t u = (y0 ^ y1) >> 9;
                        int cnt;
                        if (u > T3) {
                            cnt = 4;
                            while (cnt < d.cdf_n && u > T[cnt]) ++cnt;
                        } else {
                            cnt = (u > T0) + (u > T1) + (u > T2);
                        }
                        add += static_cast<Real>(cnt) * wd;
                    }
                    if (valid) out[static_cast<int64_t>(kc + j) * a.N + g] = add;
                }
            }
            return;
        }
    }
    if (!valid) return;
    if (q1 - q0 == 1) {
        // one drive (the common case): its descriptor and the first CDF
        // thresholds in registers for the whole run of steps.  The count is
        // the number of leading thresholds below the draw, so the first four
        // compares decide it unless it is 4 or more.
        const DriveDev d = a.drives[a.pop_drive_list[q0]];
        const uint64_t *T = a.cdf + d.cdf_off;
        constexpr uint64_t kNone = ~0ull;  // no threshold: never below a 53-bit draw
        const uint64_t T0 = d.cdf_n > 0 ? T[0] : kNone, T1 = d.cdf_n > 1 ? T[1] : kNone,
                       T2 = d.cdf_n > 2 ? T[2] : kNone, T3 = d.cdf_n > 3 ? T[3] : kNone;
        const Real wd = static_cast<Real>(d.weight);
        for (int k = k0; k < k1; ++k) {
            const int64_t se = m0 + k - d.lag;
            Real add = Real(0);
            if (d.tmin < se && se <= d.tmax) {
                const uint64_t u = drive_draw(d, static_cast<uint32_t>(se), idx);
                int cnt;
                if (u > T3) {
                    cnt = 4;
                    while (cnt < d.cdf_n && u > T[cnt]) ++cnt;
                } else {
                    cnt = (u > T0) + (u > T1) + (u > T2);
                }
                add += static_cast<Real>(cnt) * wd;  // as the general path: 0 + count * weight
            }
            out[static_cast<int64_t>(k) * a.N + g] = add;
        }
        return;
    }
    for (int k = k0; k < k1; ++k) {
        const int64_t m = m0 + k;
        Real add = Real(0);
        for (int q = q0; q < q1; ++q) {
            const DriveDev &d = a.drives[a.pop_drive_list[q]];
            const int64_t se = m - d.lag;
            if (d.tmin < se && se <= d.tmax) {
                const uint64_t u = drive_draw(d, static_cast<uint32_t>(se), idx);
                const int cnt = poisson_from_table(a.cdf + d.cdf_off, d.cdf_n, u);
                add += static_cast<Real>(cnt) * static_cast<Real>(d.weight);
            }
        }
        out[static_cast<int64_t>(k) * a.N + g] = add;
    }
}

// PORTS: the receptor ports 'ex' / 'in_' keep rings of their own,
// ring_s[(port * L + slot) * tile + t] (the kernel models' ports,
// _kernel/models/iaf_psc_alpha.py 'ex' / 'in_'); otherwise one ring whose
// sum is split by sign (_base.py:312-382).
// NT threads per CTA: the update needs only one thread per neuron of the
// tile, but the delivery phases (record validation, bucket lookups, edge
// loads) are chains of dependent latencies, and more warps per SM hide them:
// NT x REGS stays at 56 K of the SM's 64 K registers, which leaves room for a
// 128-thread block of the drive pass running beside it.
// (measured on the 12 500-neuron network: 256 threads 11.9 ms per simulated
// second in FP32, 384 10.4, 512 9.65, 640 10.2, 768 10.4, 1024 11.2; FP64
// 14.2 at 256, 13.2 at 512)
template <typename Real>
struct TiledBlock {
    static constexpr int threads = 512, regs = 112;
};

template <typename Real, int MODEL, bool PORTS, int NT, int REGS>
__global__ void __maxnreg__(REGS) k_lif_tiled(const LifArgs<Real> a, const TiledArgs<Real> t2) {
    // half-warp hw reads records hw + kHalfWarps i, i < kRecPerHalf
    constexpr int kHalfWarps = NT / 16;
    constexpr int kRecPerHalf = (kMaxCtas + kHalfWarps - 1) / kHalfWarps;
    using Fix = typename FixOf<Real>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int W = a.W;
    constexpr int R = PORTS ? 2 : 1;
    constexpr uint32_t kPostMask = PORTS ? 0x7FFFu : 0xFFFFu;
    const TiledLayout lay = tiled_layout(sizeof(PopCoef<Real>), sizeof(ProjDev<Real>), sizeof(Real),
                                         a.npop, a.nproj, a.tile, a.L * R, W,
                                         t2.smem_ptr ? a.N + 1 : 0);
    PopCoef<Real> *s_coef = reinterpret_cast<PopCoef<Real> *>(smem_raw + lay.coef);
    ProjDev<Real> *s_proj = reinterpret_cast<ProjDev<Real> *>(smem_raw + lay.proj);
    Fix *ring_s = reinterpret_cast<Fix *>(smem_raw + lay.ring);  // fixed-point arrivals
    Real *drv_s = reinterpret_cast<Real *>(smem_raw + lay.drv);  // [2][W][tile]
    uint32_t *s_spk = reinterpret_cast<uint32_t *>(smem_raw + lay.spk);
    int *s_ptr = reinterpret_cast<int *>(smem_raw + lay.ptr);   // this tile's CSR bounds
    __shared__ int s_off[kMaxPops + 1];
    __shared__ Fix s_wproj[kMaxInputs];
    __shared__ int s_warp[32];
    __shared__ uint32_t s_list[kListCap];  // gathered spikes: pre gid << 5 | step in window
    __shared__ int s_ibeg[kListCap], s_ioff[kListCap + 1];
    __shared__ uint16_t s_espk[kEdgeCap];  // spike of each flattened edge of a pass
    __shared__ int s_nsp[2];  // spikes of the window, by window parity
    __shared__ int s_nlist, s_abort;

    const int tid = threadIdx.x, B = blockDim.x;
    const int G = gridDim.x, c = blockIdx.x;
    const int N = a.N, L = a.L, tile = a.tile;
    const size_t RS = static_cast<size_t>(t2.rec_stride);  // words from one record to the next
    const int cta0 = c * tile;
    const int nloc = max(0, min(tile, N - cta0));
    const int *gptr = t2.ptr + static_cast<size_t>(c) * (N + 1);  // this tile's bounds in HBM

    for (int i = tid; i < a.npop; i += B) {
        s_coef[i] = a.coef[i];
        s_off[i] = a.coef[i].off;
    }
    for (int i = tid; i < a.nproj; i += B) {
        s_proj[i] = a.projs[i];
        s_wproj[i] = t2.wproj[i];
    }
    if (t2.smem_ptr)
        for (int i = tid; i <= N; i += B) s_ptr[i] = gptr[i];
    // arrival ring of this tile (fixed point): global [L][R][N] -> shared
    // [R][L][tile]
    const Fix *ring_g = reinterpret_cast<const Fix *>(a.ring);
    for (int i = tid; i < R * L * tile; i += B) {
        const int pl = i / tile, tt = i % tile;
        const int port = pl / L, slot = pl % L;
        ring_s[i] = tt < nloc ? ring_g[(static_cast<size_t>(slot) * R + port) * N + cta0 + tt] : Fix(0);
    }
    if (tid == 0) {
        s_abort = 0;
        s_nsp[0] = 0;
        s_nsp[1] = 0;
    }
    __syncthreads();

    // neuron t of this tile lives in thread t's registers for the whole launch
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
    // this CTA's region of the spike record (no global atomic on the hot path),
    // continued across the launches of one run
    const int64_t rec_cap = a.spk_cap / G;
    int64_t *my_spk_step = a.spk_step + static_cast<size_t>(c) * rec_cap;
    int32_t *my_spk_gid = a.spk_gid + static_cast<size_t>(c) * rec_cap;
    int64_t rec_n = t2.rec_count[c];  // uniform across the CTA

    const int64_t n_end = a.step0 + a.n_steps;
    const int nwin = static_cast<int>((a.n_steps + W - 1) / W);
    const int lane = tid & 31, hw = tid >> 4, w = lane & 15;

    // drive of window j into drv_s[j & 1] (own neuron's entries, asynchronous)
    auto drive_prefetch = [&](int j) {
        if (j < nwin && own) {
            const int64_t m0 = a.step0 + static_cast<int64_t>(j) * W;
            const int Wk = static_cast<int>((n_end - m0) < W ? (n_end - m0) : W);
            Real *dst = drv_s + static_cast<size_t>(j & 1) * W * tile + tid;
            const Real *src = t2.drive + (m0 - t2.drive_step0) * N + g;
            for (int k = 0; k < Wk; ++k)
                __pipeline_memcpy_async(dst + k * tile, src + static_cast<int64_t>(k) * N, sizeof(Real));
        }
        __pipeline_commit();
    };
    // first loads of a poll of window e's records (word w of record hw + 16 i)
    auto poll_issue = [&](int e, uint32_t (&word)[kRecPerHalf]) {
        const uint32_t *recs =
            t2.list + (static_cast<size_t>(e & (kRecBufs - 1)) * t2.rec_rep + c % t2.rec_rep) * G * RS;
#pragma unroll
        for (int i = 0; i < kRecPerHalf; ++i) {
            const int j = hw + kHalfWarps * i;
            word[i] = j < G ? __ldcg(recs + j * RS + w) : 0u;
        }
    };
    // scatter the S gathered spikes in s_list / s_ibeg / s_ioff into the
    // ring (window slot slot0; all threads, ends with a block barrier)
    auto scatter = [&](int S, int slot0) {
        // 2. offsets of the buckets in the flattened edge list (and the
        //    spike of every edge of the first pass)
        const int T = block_scan_map(s_ioff, S, s_warp, s_espk, kEdgeCap);
        // 3. every edge of the window, in passes of kEdgeCap flattened edges:
        //    s_espk maps a flattened edge to its spike, then lane-interleaved
        //    threads (edge q0 + u B) take 32 consecutive edges per warp
        //    instruction -- independent index loads, and consecutive targets
        //    of one bucket for the shared-memory atomics
        for (int p0 = 0; p0 < T; p0 += kEdgeCap) {
            const int p1 = min(T, p0 + kEdgeCap);
            if (p0 > 0) {
                for (int i = tid; i < S; i += B) {
                    const int a0 = max(s_ioff[i], p0), a1 = min(s_ioff[i + 1], p1);
                    for (int q = a0; q < a1; ++q) s_espk[q - p0] = static_cast<uint16_t>(i);
                }
                __syncthreads();
            }
            for (int q0 = p0 + tid; q0 < p1; q0 += B * kEdgeUnroll) {
                int jj[kEdgeUnroll], nm[kEdgeUnroll];
#pragma unroll
                for (int u = 0; u < kEdgeUnroll; ++u) {
                    const int q = q0 + u * B;
                    jj[u] = -1;
                    nm[u] = 0;
                    if (q < p1) {
                        const int it = s_espk[q - p0];
                        jj[u] = s_ibeg[it] + (q - s_ioff[it]);
                        const int m = slot0 + static_cast<int>(s_list[it] & 31u);
                        nm[u] = m >= L ? m - L : m;
                    }
                }
                uint32_t ed[kEdgeUnroll];
                Fix wv[kEdgeUnroll];
#pragma unroll
                for (int u = 0; u < kEdgeUnroll; ++u) {
                    ed[u] = 0u;
                    wv[u] = Fix(0);
                    if (jj[u] >= 0) {
                        ed[u] = __ldg(t2.edges + jj[u]);
                        if (t2.wfix) wv[u] = __ldg(t2.wfix + jj[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kEdgeUnroll; ++u) {
                    if (jj[u] >= 0) {
                        if (!t2.wfix) wv[u] = s_wproj[ed[u] >> 24];
                        int slot = nm[u] + static_cast<int>((ed[u] >> 16) & 0xFFu);
                        if (slot >= L) slot -= L;
                        if (PORTS) slot += static_cast<int>((ed[u] >> 15) & 1u) * L;
                        fix_add(ring_s + slot * tile + (ed[u] & kPostMask), wv[u]);
                    }
                }
            }
            __syncthreads();
        }
    };
    // deliver the spikes of window e into the ring (all threads)
    auto deliver = [&](int e, uint32_t (&word)[kRecPerHalf], bool have) {
        const int buf = e & (kRecBufs - 1);
        const uint32_t tag = tag_of(e);
        const int64_t e0 = a.step0 + static_cast<int64_t>(e) * W;
        const int slot0 = static_cast<int>(e0 % L);
        const uint32_t *recs =
            t2.list + (static_cast<size_t>(buf) * t2.rec_rep + c % t2.rec_rep) * G * RS;
        // a gathered spike: its entry and the bounds of its edge bucket
        auto put = [&](int pos, int src, uint32_t word_) {
            const int pre = src * tile + static_cast<int>((word_ & kPayMask) >> 5);
            s_list[pos] = (static_cast<uint32_t>(pre) << 5) | (word_ & 31u);
            const int b0 = t2.smem_ptr ? s_ptr[pre] : __ldg(gptr + pre);
            const int b1 = t2.smem_ptr ? s_ptr[pre + 1] : __ldg(gptr + pre + 1);
            s_ibeg[pos] = b0;
            s_ioff[pos] = b1 - b0;
        };
        auto push = [&](int src, uint32_t word_) {
            const int pos = atomicAdd(&s_nlist, 1);
            if (pos < kListCap) put(pos, src, word_);
        };
        if (tid == 0) s_nlist = 0;
        __syncthreads();
        // 1. gather: half-warp hw reads records hw + 16 i, lane w word w; every
        //    polling round issues all of the lane's loads at once, then
        //    validates each record (count word and the entries it announces
        //    must carry the tag); a record's entries go to s_list once.
        unsigned pend = 0;  // bit i: record hw + 16 i still pending (uniform per half)
#pragma unroll
        for (int i = 0; i < kRecPerHalf; ++i)
            if (hw + kHalfWarps * i < G) pend |= 1u << i;
        // a first poll issued right after this CTA's own publish mostly finds
        // the other records not yet written and only adds to the L2 traffic
        // of the lines being written; waiting about one write latency first
        // saves a polling round
        if (!have && t2.poll_pause > 0) __nanosleep(t2.poll_pause);
        const uint64_t t_start = gtimer();
        bool first = true;
        while (__any_sync(0xffffffffu, pend != 0u)) {
            if (!(first && have)) {
#pragma unroll
                for (int i = 0; i < kRecPerHalf; ++i) {
                    const int j = hw + kHalfWarps * i;
                    word[i] = (pend >> i) & 1u ? __ldcg(recs + j * RS + w) : 0u;
                }
            }
            first = false;
#pragma unroll
            for (int i = 0; i < kRecPerHalf; ++i) {
                const int j = hw + kHalfWarps * i;
                const bool pending = (pend >> i) & 1u;
                const uint32_t head = __shfl_sync(0xffffffffu, word[i], lane & 16);
                const int cnt = (head & kTagMask) == tag ? static_cast<int>(head & kPayMask) : -1;
                const bool ok = !pending || (cnt >= 0 && (w == 0 || w > cnt ||
                                                          (word[i] & kTagMask) == tag));
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                const bool half_ok = ((lane & 16) ? (bal >> 16) : (bal & 0xFFFFu)) == 0xFFFFu;
                if (pending && half_ok) {
                    if (w >= 1 && w <= cnt) push(j, word[i]);
                    if (w == 0 && cnt > kRecInline) {  // overflow entries
                        const uint32_t *src =
                            t2.ovf + (static_cast<size_t>(buf) * G + j) * t2.list_cap;
                        bool gave_up = false;
                        for (int q = 0; q < cnt - kRecInline && !gave_up; ++q) {
                            uint32_t ow = __ldcg(src + q);
                            const uint64_t tq = gtimer();
                            while ((ow & kTagMask) != tag) {
                                // give up after the limit, or at once when any
                                // CTA has already raised the error flag
                                if (gtimer() - tq > kPollLimitNs || *(volatile int *)a.err != 0) {
                                    atomicCAS(a.err, 0, BSPK_DEV_ERR_TIMEOUT);
                                    s_abort = 1;
                                    gave_up = true;
                                    break;
                                }
                                ow = __ldcg(src + q);
                            }
                            if (!gave_up) push(j, ow);
                        }
                    }
                    pend &= ~(1u << i);
                }
            }
            if (__any_sync(0xffffffffu, pend != 0u && (gtimer() - t_start > kPollLimitNs ||
                                                       *(volatile int *)a.err != 0))) {
                if (lane == 0) {
                    atomicCAS(a.err, 0, BSPK_DEV_ERR_TIMEOUT);
                    s_abort = 1;
                }
                break;
            }
        }
        __syncthreads();
        if (s_abort) return;
        const int total = s_nlist;
        if (total <= kListCap) {
            scatter(total, slot0);
            return;
        }
        // more spikes than the list holds: deliver them in chunks of kListCap.
        // Spike x of the window is entry q of record j with x = off_j + q
        // (off_j = counts of the records before j), so every chunk takes a
        // fixed set of spikes; the fixed-point sums do not depend on how the
        // spikes are split.  The records were validated above and stay
        // unchanged until every CTA has delivered this window.
        for (int cb = 0; cb < total; cb += kListCap) {
            const int ce = min(total, cb + kListCap);
#pragma unroll 1
            for (int i = 0; i < kRecPerHalf; ++i) {
                const int j = hw + kHalfWarps * i;
                int part = 0;
                if (j < G)
                    for (int k = w; k < j; k += 16)
                        part += static_cast<int>(__ldcg(recs + k * RS) & kPayMask);
#pragma unroll
                for (int o = 8; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o, 16);
                if (j >= G) continue;
                const uint32_t head = __ldcg(recs + j * RS);
                const int cnt = static_cast<int>(head & kPayMask);
                const uint32_t *ovs = t2.ovf + (static_cast<size_t>(buf) * G + j) * t2.list_cap;
                const int q1 = min(cnt, ce - part);
                for (int q = max(0, cb - part) + w; q < q1; q += 16) {
                    const uint32_t wq = q < kRecInline ? __ldcg(recs + j * RS + 1 + q)
                                                       : __ldcg(ovs + (q - kRecInline));
                    const int pos = part + q - cb;
                    if ((wq & kTagMask) == tag) {
                        put(pos, j, wq);
                    } else {  // never expected: an empty bucket and an error
                        atomicCAS(a.err, 0, BSPK_DEV_ERR_BOUNDS);
                        s_list[pos] = 0u;
                        s_ibeg[pos] = 0;
                        s_ioff[pos] = 0;
                    }
                }
            }
            __syncthreads();
            scatter(ce - cb, slot0);
        }
    };

    uint32_t word[kRecPerHalf];
#pragma unroll
    for (int i = 0; i < kRecPerHalf; ++i) word[i] = 0u;
    drive_prefetch(0);
    for (int j = 0; j < nwin; ++j) {
        const int64_t n0 = a.step0 + static_cast<int64_t>(j) * W;
        const int Wk = static_cast<int>((n_end - n0) < W ? (n_end - n0) : W);
        const int slot0 = static_cast<int>(n0 % L);
        const int buf = j & (kRecBufs - 1);
        const uint32_t tag = tag_of(j);
        // this CTA's record in every replica (stride G * RS words)
        uint32_t *rec = t2.list + (static_cast<size_t>(buf) * t2.rec_rep * G + c) * RS;
        const size_t rstride = static_cast<size_t>(G) * RS;
        uint32_t *ovf = t2.ovf + (static_cast<size_t>(buf) * G + c) * t2.list_cap;
        const bool pre = a.pipe && j >= 1;
        if (pre) poll_issue(j - 1, word);
        __pipeline_wait_prior(0);  // this thread's drive entries of window j have landed

        // ---- update.  The window's inputs are read from shared memory into
        // registers first (kUpd steps at a time), so the steps' dependency
        // chain runs on registers only; spikes are collected in a bit mask
        // and written to the record after the loop.
        if (own) {
            const Real *drv = drv_s + static_cast<size_t>(j & 1) * W * tile + tid;
            const Real inv = t2.inv_scale;
            uint32_t spmask = 0u;
            int slot = slot0;
            for (int k0 = 0; k0 < Wk; k0 += kUpd) {
                const int kn = min(kUpd, Wk - k0);
                Real xe[kUpd], xi[kUpd];
#pragma unroll
                for (int u = 0; u < kUpd; ++u) {
                    xe[u] = Real(0);
                    xi[u] = Real(0);
                    if (u < kn) {
                        int sl = slot + u;  // slot + u < 2 L: kn <= W < L
                        if (sl >= L) sl -= L;
                        xe[u] = static_cast<Real>(ring_s[sl * tile + tid]) * inv + drv[(k0 + u) * tile];
                        ring_s[sl * tile + tid] = Fix(0);
                        if (PORTS) {
                            xi[u] = static_cast<Real>(ring_s[(L + sl) * tile + tid]) * inv;
                            ring_s[(L + sl) * tile + tid] = Fix(0);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < kUpd; ++u) {
                    if (u < kn) {
                        bool sp;
                        if (PORTS) {
                            if (MODEL == 0) sp = iaf_alpha_step_ports<Real>(cf, st, r, xe[u], xi[u]);
                            else sp = iaf_exp_step_ports<Real>(cf, st, r, xe[u], xi[u]);
                        } else {
                            if (MODEL == 0) sp = iaf_alpha_step<Real>(cf, st, r, xe[u]);
                            else sp = iaf_exp_step<Real>(cf, st, r, xe[u]);
                        }
                        spmask |= static_cast<uint32_t>(sp) << (k0 + u);
                        if (rslot >= 0)
                            a.v_out[static_cast<size_t>(n0 + k0 + u - a.run_step0) * a.n_rec + rslot] = st[0];
                    }
                }
                slot += kn;
                if (slot >= L) slot -= L;
            }
            while (spmask) {
                const int k = __ffs(static_cast<int>(spmask)) - 1;
                spmask &= spmask - 1u;
                const int pos = atomicAdd(&s_nsp[j & 1], 1);
                const uint32_t ent = (static_cast<uint32_t>(tid) << 5) | static_cast<uint32_t>(k);
                s_spk[pos] = ent;
                if (pos < kRecInline)
                    for (int q = 0; q < t2.rec_rep; ++q) rec[q * rstride + 1 + pos] = tag | ent;
                else if (pos - kRecInline < t2.list_cap) ovf[pos - kRecInline] = tag | ent;
            }
        }
        __syncthreads();
        const int nsp = s_nsp[j & 1];
        // the other parity's counter was last read before this barrier
        if (tid == 0) s_nsp[(j + 1) & 1] = 0;
        {
            // thread 16 q + w writes word w of replica q: the count word, or
            // the window's tag into the unused entry slots
            const int q = tid >> 4, wd = tid & 15;
            if (q < t2.rec_rep) {
                if (wd == 0) {
                    if (c != t2.hold_cta || j != t2.hold_win)
                        rec[q * rstride] = tag | static_cast<uint32_t>(nsp);
                } else if (wd - 1 >= nsp) {
                    rec[q * rstride + wd] = tag | kPayMask;
                }
            }
        }

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
        drive_prefetch(j + 1);
        if (!a.pipe) deliver(j, word, false);
        else if (j >= 1) deliver(j - 1, word, pre);
        __syncthreads();
        if (s_abort) return;
    }
    if (a.pipe && nwin >= 1) {
        deliver(nwin - 1, word, false);
        if (s_abort) return;
    }

    // ---- persist state, the tile's ring and this CTA's record count
    if (own) {
#pragma unroll
        for (int i = 0; i < 6; ++i) a.s[i][g] = st[i];
        a.r[g] = r;
    }
    Fix *ring_out = reinterpret_cast<Fix *>(a.ring);
    for (int i = tid; i < R * L * nloc; i += B) {
        const int pl = i / nloc, tt = i % nloc;
        const int port = pl / L, slot = pl % L;
        ring_out[(static_cast<size_t>(slot) * R + port) * N + cta0 + tt] = ring_s[pl * tile + tt];
    }
    if (tid == 0) t2.rec_count[c] = rec_n;
}

size_t lif_tiled_smem(int tile, int L, int W, int N, int npop, int nproj, bool dbl, bool smem_ptr,
                      bool ports) {
    return tiled_layout(dbl ? sizeof(PopCoef<double>) : sizeof(PopCoef<float>),
                        dbl ? sizeof(ProjDev<double>) : sizeof(ProjDev<float>), dbl ? 8 : 4, npop,
                        nproj, tile, L * (ports ? 2 : 1), W, smem_ptr ? N + 1 : 0)
        .total;
}

template <typename Real>
cudaError_t launch_lif_tiled(const LifArgs<Real> &a, const TiledArgs<Real> &t2, int grid,
                             cudaStream_t st) {
    const size_t smem = lif_tiled_smem(a.tile, a.L, a.W, a.N, a.npop, a.nproj, sizeof(Real) == 8,
                                       t2.smem_ptr != 0, t2.ports != 0);
    void *args[] = {const_cast<LifArgs<Real> *>(&a), const_cast<TiledArgs<Real> *>(&t2)};
    constexpr int NT = TiledBlock<Real>::threads, RG = TiledBlock<Real>::regs;
    const void *fn =
        t2.ports ? (a.model == 0 ? reinterpret_cast<const void *>(&k_lif_tiled<Real, 0, true, NT, RG>)
                                 : reinterpret_cast<const void *>(&k_lif_tiled<Real, 1, true, NT, RG>))
                 : (a.model == 0 ? reinterpret_cast<const void *>(&k_lif_tiled<Real, 0, false, NT, RG>)
                                 : reinterpret_cast<const void *>(&k_lif_tiled<Real, 1, false, NT, RG>));
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(NT), args, smem, st);
}

template <typename Real>
cudaError_t launch_drive_fill(const LifArgs<Real> &a, int64_t m0, int n, Real *out,
                              cudaStream_t st, bool beside) {
    if (n <= 0 || a.N <= 0) return cudaSuccess;
    const int threads = beside ? 128 : 256;
    const int gx = (a.N + threads - 1) / threads;
    const int gy = static_cast<int>(std::min<int64_t>(std::max<int64_t>(1, (148 * 16 + gx - 1) / gx),
                                                      std::min(n, 65535)));
    const int spb = (n + gy - 1) / gy;
    k_drive_fill<Real><<<dim3(gx, (n + spb - 1) / spb), threads, 0, st>>>(a, m0, n, spb, out);
    return cudaGetLastError();
}

// Recorded spikes of the per-CTA regions into one contiguous list (order
// free), dropping the holes left for unrecorded neurons (gid < 0).
__global__ void k_compact_spikes(int64_t region, const long long *rec_count, const int64_t *in_step,
                                 const int32_t *in_gid, int64_t *out_step, int32_t *out_gid,
                                 unsigned long long *out_n) {
    const int c = blockIdx.x;
    const int64_t k = rec_count[c] < region ? rec_count[c] : region;
    const int64_t base = static_cast<int64_t>(c) * region;
    for (int64_t i = threadIdx.x; i < k; i += blockDim.x) {
        const int32_t gg = in_gid[base + i];
        if (gg < 0) continue;
        const unsigned long long pos = atomicAdd(out_n, 1ull);
        out_step[pos] = in_step[base + i];
        out_gid[pos] = gg;
    }
}

cudaError_t launch_compact_spikes(int G, int64_t region, const long long *rec_count,
                                  const int64_t *in_step, const int32_t *in_gid, int64_t *out_step,
                                  int32_t *out_gid, unsigned long long *out_n, cudaStream_t st) {
    k_compact_spikes<<<G, 256, 0, st>>>(region, rec_count, in_step, in_gid, out_step, out_gid, out_n);
    return cudaGetLastError();
}

template cudaError_t launch_lif_tiled<float>(const LifArgs<float> &, const TiledArgs<float> &, int,
                                             cudaStream_t);
template cudaError_t launch_lif_tiled<double>(const LifArgs<double> &, const TiledArgs<double> &,
                                              int, cudaStream_t);
template cudaError_t launch_drive_fill<float>(const LifArgs<float> &, int64_t, int, float *,
                                              cudaStream_t, bool);
template cudaError_t launch_drive_fill<double>(const LifArgs<double> &, int64_t, int, double *,
                                               cudaStream_t, bool);

}  // namespace bspk
