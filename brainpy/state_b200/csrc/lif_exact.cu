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
                                const uint64_t u = drive_draw(d, static_cast<uint32_t>(se),
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

// ===================================================== no-allocation entry
//
// bspk_iaf_exact_run_noalloc: the deterministic FP64 kernel above, launched
// for one iaf_psc_alpha population (one Poisson drive, then one recurrent
// projection) without a plan and without any device allocation.  It is for
// callers that cannot call cudaMalloc: code running inside another
// framework's memory pool or allocator hooks (an XLA custom call, a plugin
// whose host forbids device allocations).  The caller passes every input and
// output buffer; everything else the kernel needs lives in one file-scope
// device array of fixed size (parameter tables, Poisson CDF, 64-step
// spike-history words, barrier counter, error flag, spike counter), so at
// most kNoAllocMaxNeurons neurons and a CDF of kNoAllocMaxCdf entries.  The
// kernel is a cooperative launch of up to 256 threads per CTA, so the
// network must also fit the CTAs the GPU can hold at once (256 per SM times
// the SM count on a B200, 37 888 neurons): the call checks that before it
// launches.
namespace {

constexpr int kNoAllocMaxNeurons = 1 << 16;
constexpr int kNoAllocMaxCdf = 4096;

struct NoAllocScratch {
    uint64_t hist[kNoAllocMaxNeurons];
    uint64_t cdf[kNoAllocMaxCdf];
    bspk::PopCoef<double> coef;
    bspk::DriveDev drive;
    bspk::ProjDev<double> proj;
    int in_ptr[2], in_list[2], drv_ptr[2], drv_list[1], out_ptr[2], out_list[1];
    unsigned int barrier;
    int err;
    unsigned long long spk_count;
};

// Shared by every call on a device and kept until the process exits; a call
// clears the parts that must start at zero.  Calls that overlap on the GPU
// (two streams at once) race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[256] = {};

// Copies the spike counter and error flag of the scratch array to the
// caller's outputs; a count above the caller's capacity (entries dropped)
// turns a zero status into the overflow code.
__global__ void k_noalloc_finish(const NoAllocScratch *S, int64_t cap, int64_t *count, int *status) {
    const unsigned long long n = S->spk_count;
    *count = static_cast<int64_t>(n);
    int e = S->err;
    if (e == 0 && n > static_cast<unsigned long long>(cap)) e = bspk::BSPK_DEV_ERR_OVERFLOW;
    *status = e;
}

}  // namespace

extern "C" int bspk_iaf_exact_run_noalloc(double dt, const double *params, int n_params, int n,
                                          const int64_t *in_indptr, const uint32_t *in_edges,
                                          const double *in_w, double w_const,
                                          int min_delay_steps, int max_delay_steps,
                                          double drive_rate_hz, double drive_weight,
                                          int drive_delay_steps, uint32_t drive_seed,
                                          double *state, int32_t *refr, int64_t n_steps,
                                          int64_t *spike_step, int32_t *spike_gid,
                                          int64_t spike_cap, int64_t *spike_count, int *status,
                                          void *stream) {
    using namespace bspk;
    if (!params || !in_indptr || !in_edges || !state || !refr || !spike_step || !spike_gid ||
        !spike_count || !status || n <= 0 || n_steps < 0 || spike_cap < 0 || !(dt > 0))
        return fail(BSPK_ERR_ARG, "bad argument");
    if (n > kNoAllocMaxNeurons)
        return fail(BSPK_ERR_ARG, "no-allocation entry point: more than 65536 neurons");
    if (min_delay_steps < 0 || max_delay_steps < min_delay_steps || max_delay_steps + 1 > 62)
        return fail(BSPK_ERR_ARG, "no-allocation entry point: delays must be 0..61 steps");
    const double lam = drive_rate_hz * dt / 1000.0;
    if (!(lam >= 0) || lam > 700.0) return fail(BSPK_ERR_ARG, "rate*dt/1000 must be in [0, 700]");
    const std::vector<uint64_t> cdf = host_poisson_thresholds(lam);
    if (static_cast<int>(cdf.size()) > kNoAllocMaxCdf) return fail(BSPK_ERR_ARG, "drive CDF too long");
    PopCoef<double> coef;
    int rc = host_make_coef(BSPK_IAF_PSC_ALPHA, std::vector<double>(params, params + n_params), dt,
                            &coef);
    if (rc) return rc;
    coef.off = 0;
    coef.n = n;

    int dev = 0;
    BSPK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(BSPK_ERR_ARG, "device ordinal out of range");
    void *base = nullptr;
    {
        // once per device, with that device current: the host-side symbol is a
        // stand-in, only the address returned here is valid on the device
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void *addr = nullptr;
            BSPK_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
            g_noalloc_addr[dev] = addr;
        }
        base = g_noalloc_addr[dev];
    }
    int sm = 0;
    BSPK_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));
    int block = ((n + sm - 1) / sm + 31) / 32 * 32;
    block = block < 64 ? 64 : (block > 256 ? 256 : block);
    const int grid = (n + block - 1) / block;
    // every CTA of the cooperative launch must be resident at once
    int per_sm = 0;
    BSPK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_lif_exact<0>, block,
        lif_exact_smem(block, 1, 1, 1, static_cast<int>(cdf.size()))));
    if (static_cast<int64_t>(per_sm) * sm < grid)
        return fail(BSPK_ERR_UNSUPPORTED,
                    "no-allocation entry point: " + std::to_string(n) + " neurons need " +
                        std::to_string(grid) + " co-resident CTAs of " + std::to_string(block) +
                        " threads; this GPU holds " + std::to_string(per_sm * sm) + " (at most " +
                        std::to_string(static_cast<int64_t>(per_sm) * sm * 256) + " neurons)");
    NoAllocScratch *S = static_cast<NoAllocScratch *>(base);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    DriveDev drive{};
    drive.pop = 0;
    drive.lag = drive_delay_steps + 1;  // the reference Simulator's holder lag
    drive.seed = drive_seed;
    drive.cdf_off = 0;
    drive.cdf_n = static_cast<int>(cdf.size());
    drive.receptor = 0;
    drive.weight = drive_weight;
    drive.tmin = 0;
    drive.tmax = drive_rate_hz > 0 ? (int64_t(1) << 62) : 0;
    ProjDev<double> proj{};
    proj.pre_pop = 0;
    proj.post_pop = 0;
    proj.post_off = 0;
    proj.homogeneous = in_w ? 0 : 1;
    proj.w0 = w_const;
    proj.cindptr = in_indptr;
    proj.cedges = in_edges;
    proj.cw = in_w;
    const int tables[10] = {0, 2, -1, 0, 0, 1, 0, 0, 0, 0};  // in_ptr, in_list, drv_ptr, drv_list, out
    BSPK_CUDA(cudaMemcpyAsync(S->cdf, cdf.data(), sizeof(uint64_t) * cdf.size(),
                              cudaMemcpyHostToDevice, st));
    BSPK_CUDA(cudaMemcpyAsync(&S->coef, &coef, sizeof(coef), cudaMemcpyHostToDevice, st));
    BSPK_CUDA(cudaMemcpyAsync(&S->drive, &drive, sizeof(drive), cudaMemcpyHostToDevice, st));
    BSPK_CUDA(cudaMemcpyAsync(&S->proj, &proj, sizeof(proj), cudaMemcpyHostToDevice, st));
    BSPK_CUDA(cudaMemcpyAsync(S->in_ptr, tables, sizeof(tables), cudaMemcpyHostToDevice, st));
    BSPK_CUDA(cudaMemsetAsync(S->hist, 0, sizeof(uint64_t) * n, st));
    BSPK_CUDA(cudaMemsetAsync(&S->barrier, 0, sizeof(unsigned int) + sizeof(int), st));
    BSPK_CUDA(cudaMemsetAsync(&S->spk_count, 0, sizeof(unsigned long long), st));
    // the copies above came from pageable host memory, so they completed
    // before cudaMemcpyAsync returned; the host tables may go out of scope

    const int max_lag = max_delay_steps + 1, min_lag = min_delay_steps + 1;
    int W = min_lag < kMaxWindow ? min_lag : kMaxWindow;
    if (W > 64 - max_lag) W = 64 - max_lag;
    if (W < 1) W = 1;

    LifArgs<double> a{};
    a.N = n;
    a.npop = 1;
    a.nproj = 1;
    a.ndrive = 1;
    a.coef = &S->coef;
    for (int i = 0; i < 6; ++i) a.s[i] = state + static_cast<size_t>(i) * n;
    a.r = refr;
    a.ring = nullptr;
    a.L = 1;
    a.projs = &S->proj;
    a.pop_out_ptr = S->out_ptr;
    a.pop_out_list = S->out_list;
    a.pop_in_ptr = S->in_ptr;
    a.pop_in_list = S->in_list;
    a.drives = &S->drive;
    a.pop_drive_ptr = S->drv_ptr;
    a.pop_drive_list = S->drv_list;
    a.cdf = S->cdf;
    a.cdf_total = static_cast<int>(cdf.size());
    a.step0 = 0;
    a.n_steps = n_steps;
    a.run_step0 = 0;
    a.W = W;
    a.tile = block;
    a.model = BSPK_IAF_PSC_ALPHA;
    a.spk_step = spike_step;
    a.spk_gid = spike_gid;
    a.spk_count = &S->spk_count;
    a.spk_cap = spike_cap;
    a.spk_flag = nullptr;
    a.rec_slot = nullptr;
    a.v_out = nullptr;
    a.n_rec = 0;
    a.hist = S->hist;
    a.barrier = &S->barrier;
    a.err = &S->err;
    if (n_steps > 0) {
        const cudaError_t e = launch_lif_exact(a, grid, block, st);
        if (e != cudaSuccess)
            return fail(BSPK_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    k_noalloc_finish<<<1, 1, 0, st>>>(S, spike_cap, spike_count, status);
    BSPK_CUDA(cudaGetLastError());
    return BSPK_OK;
}
