// batch_host.cpp -- the bspk_batch object behind the C ABI: instance
// descriptions, device layout (tiles, GPU-built connectivity, records),
// tile-to-CTA assignment and the autotuner.
//
// The reference batches with Runner(batch) (_kernel/runner.py:832-863), a
// vmap over trials of one plan, so every trial has the same structure.
// Here every instance is its own network (own sizes, parameters, seeds) and
// the whole batch advances in one cooperative launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "../../../include/bspk.h"
#include "batch_args.h"
#include "coef_cast.h"
#include "conn_gen.h"
#include "plan_internal.h"

using namespace bspk;

namespace {

const char *kIafStateNames[2][6] = {
    {"V_m", "I_syn_ex", "dI_syn_ex", "I_syn_in", "dI_syn_in", "y0"},
    {"V_m", "i_syn_ex", "i_syn_in", "i_0", "i_1", ""},
};

struct BPop {
    int n = 0, off = 0;
    std::vector<double> p;
    PopCoef<double> c{};
};
struct BProj {
    int pre = 0, post = 0, K = 0, autapses = 1, nbits = 32, lag = 0;
    int64_t seed = 0;
    double w = 0.0;
};
struct BDrive {
    int post = 0, lag = 0;
    double rate = 0.0, weight = 0.0;
    uint32_t seed = 0;
    int64_t tmin = 0, tmax = 0;
    std::vector<uint64_t> cdf;
};
struct BInst {
    std::vector<BPop> pops;
    std::vector<BProj> projs;
    std::vector<BDrive> drives;
    int n = 0, record = 0, W = 1, ntiles = 0, cdf_n = 0;
    int64_t g0 = 0, edges = 0;
    double inv_scale = 1.0;
};

}  // namespace

struct bspk_batch {
    bspk_config cfg{};
    int elt = 4;
    std::vector<BInst> inst;
    bool uploaded = false;
    int sm = 0, T = 0, cps = 0, G = 0, Wmax = 1;
    int64_t Ntot = 0, step = 0;
    cudaStream_t st = nullptr;
    // static device buffers
    std::vector<void *> allocs;
    void *d_s[6] = {};
    int *d_r = nullptr;
    unsigned int *d_cnt = nullptr;
    void *d_coef = nullptr;
    DriveDev *d_drives = nullptr;
    uint64_t *d_cdf = nullptr;
    void *d_projw = nullptr;
    int *d_err = nullptr;
    void *d_drive = nullptr;       // Poisson drive of one launch, [steps][Ntot]
    int64_t drive_steps = 0;
    // layout (depends on T) and assignment (depends on G)
    std::vector<void *> lay_allocs, asg_allocs;
    BatchInstDev *d_inst = nullptr;
    BatchTileDev *d_tiles = nullptr;
    int *d_ptr = nullptr;
    uint32_t *d_edges = nullptr;
    unsigned long long *d_recs = nullptr;
    int *d_part = nullptr;
    int64_t rec_words = 0;
    int *d_cta_ptr = nullptr, *d_cta_tiles = nullptr;
    int64_t *d_spk_step = nullptr;
    int32_t *d_spk_id = nullptr, *d_spk_inst = nullptr;
    long long *d_rec_count = nullptr;
    int64_t spk_cap = 0;  // per CTA
    std::vector<BatchInstDev> h_inst;
    std::vector<BatchTileDev> h_tiles;
    std::vector<double> rate_hz;  // per instance, for the cost model
    GenScratch gen;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t last_launches = 0;
    bool any_record = false;
};

namespace {

int balloc(std::vector<void *> &list, void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    list.push_back(*p);
    return BSPK_OK;
}

template <typename T>
int balloc_t(std::vector<void *> &list, T **p, size_t count) {
    void *raw = nullptr;
    int rc = balloc(list, &raw, sizeof(T) * count);
    *p = static_cast<T *>(raw);
    return rc;
}

void free_list(std::vector<void *> &list) {
    for (void *p : list) cudaFree(p);
    list.clear();
}

int check_inst(bspk_batch *b, int i) {
    if (!b) return fail(BSPK_ERR_ARG, "null batch");
    if (i < 0 || i >= static_cast<int>(b->inst.size())) return fail(BSPK_ERR_ARG, "instance index out of range");
    return BSPK_OK;
}

int lag_of(const bspk_batch *b, int delay_steps) {
    return b->cfg.semantics == BSPK_LEGACY ? delay_steps + 1 : delay_steps;
}

// Expected tile-window cost in microseconds: a fixed synchronisation and
// gather latency, the window's update steps, and the synaptic events that
// land in the tile (instance rate x edges into the tile).
double tile_cost(const bspk_batch *b, const BInst &I, const BatchTileDev &t, double rate_hz,
                 int64_t n_steps) {
    double e_tile = 0.0;
    for (const auto &P : I.projs) {
        const BPop &q = I.pops[P.post];
        const int lo = std::max(t.first, q.off), hi = std::min(t.first + t.n, q.off + q.n);
        if (hi > lo) e_tile += static_cast<double>(hi - lo) * P.K;
    }
    const double windows = std::ceil(static_cast<double>(n_steps) / I.W);
    const double ev_per_window = e_tile * rate_hz * b->cfg.dt * 1e-3 * I.W;
    return windows * (4.0 + 0.15 * I.W + 0.004 * ev_per_window);
}

// Device layout for tile size T: tiles, records and GPU-built connectivity.
int layout(bspk_batch *b, int T) {
    free_list(b->lay_allocs);
    b->T = T;
    b->h_inst.clear();
    b->h_tiles.clear();
    int64_t ptr_words = 0, edges = 0, rec_words = 0, cdf0 = 0;
    int drive0 = 0, coef0 = 0;
    for (size_t i = 0; i < b->inst.size(); ++i) {
        BInst &I = b->inst[i];
        I.ntiles = (I.n + T - 1) / T;
        if (I.ntiles > 1024) return fail(BSPK_ERR_UNSUPPORTED, "instance has more than 1024 tiles");
        int min_ref = 1 << 30;
        for (const auto &P : I.pops) min_ref = std::min(min_ref, P.c.ref_count);
        const int per_neuron = (I.W + min_ref) / (min_ref + 1);  // spikes per window at most
        BatchInstDev d{};
        d.n = I.n;
        d.W = I.W;
        d.tile0 = static_cast<int>(b->h_tiles.size());
        d.ntiles = I.ntiles;
        d.npop = static_cast<int>(I.pops.size());
        for (int p = 0; p <= d.npop; ++p) d.pop_off[p] = p < d.npop ? I.pops[p].off : I.n;
        d.coef0 = coef0;
        d.ndrive = static_cast<int>(I.drives.size());
        d.drive0 = drive0;
        d.cdf_n = I.cdf_n;
        d.cdf0 = cdf0;
        d.proj0 = static_cast<int>(i) * kBatchMaxProj;
        d.inv_scale = I.inv_scale;
        d.rec_cap = T * std::max(1, per_neuron);
        d.record = I.record;
        d.rec0 = rec_words;
        d.g0 = I.g0;
        d.ptr0 = ptr_words;
        d.edge0 = edges;
        b->h_inst.push_back(d);
        for (int t = 0; t < I.ntiles; ++t) {
            BatchTileDev td{};
            td.inst = static_cast<int>(i);
            td.tloc = t;
            td.first = t * T;
            td.n = std::min(T, I.n - t * T);
            b->h_tiles.push_back(td);
        }
        ptr_words += static_cast<int64_t>(I.ntiles) * I.n + 1;
        edges += I.edges;
        rec_words += static_cast<int64_t>(I.ntiles) * 2 * (1 + d.rec_cap);
        cdf0 += I.cdf_n;
        drive0 += d.ndrive;
        coef0 += d.npop;
    }
    int rc = balloc_t(b->lay_allocs, &b->d_ptr, ptr_words);
    if (!rc) rc = balloc_t(b->lay_allocs, &b->d_edges, std::max<int64_t>(edges, 1));
    if (!rc) rc = balloc_t(b->lay_allocs, &b->d_recs, rec_words);
    if (!rc) rc = balloc_t(b->lay_allocs, &b->d_part, b->h_tiles.size() + 1);
    if (!rc) rc = balloc_t(b->lay_allocs, &b->d_inst, b->h_inst.size());
    if (!rc) rc = balloc_t(b->lay_allocs, &b->d_tiles, b->h_tiles.size() + 1);
    if (rc) return rc;
    b->rec_words = rec_words;
    BSPK_CUDA(cudaMemsetAsync(b->d_recs, 0, sizeof(unsigned long long) * rec_words, b->st));
    BSPK_CUDA(cudaMemsetAsync(b->d_part, 0, sizeof(int) * (b->h_tiles.size() + 1), b->st));
    BSPK_CUDA(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), sizeof(BatchInstDev) * b->h_inst.size(),
                              cudaMemcpyHostToDevice, b->st));
    BSPK_CUDA(cudaMemcpyAsync(b->d_tiles, b->h_tiles.data(), sizeof(BatchTileDev) * b->h_tiles.size(),
                              cudaMemcpyHostToDevice, b->st));
    // connectivity, instance by instance
    for (size_t i = 0; i < b->inst.size(); ++i) {
        const BInst &I = b->inst[i];
        std::vector<FixedIndegreeDev> gens;
        std::vector<int> pre_off, post_off, slot;
        for (size_t p = 0; p < I.projs.size(); ++p) {
            const BProj &P = I.projs[p];
            FixedIndegreeDev g;
            rc = make_fixed_indegree_dev(P.seed, I.pops[P.pre].n, I.pops[P.post].n, P.K,
                                         P.pre == P.post, P.autapses != 0, P.nbits, &g);
            if (rc) return rc;
            gens.push_back(g);
            pre_off.push_back(I.pops[P.pre].off);
            post_off.push_back(I.pops[P.post].off);
            slot.push_back(static_cast<int>(p));
        }
        const BatchInstDev &d = b->h_inst[i];
        rc = gen_instance_tiles(b->gen, gens, pre_off, post_off, slot, I.n, T, I.ntiles,
                                b->d_ptr + d.ptr0, b->d_edges + d.edge0, b->st);
        if (rc) return rc;
    }
    BSPK_CUDA(cudaStreamSynchronize(b->st));
    b->gen.release();
    return BSPK_OK;
}

// Tiles to CTAs: longest-processing-time first onto the least-loaded CTA.
int assign(bspk_batch *b, int cps, int64_t n_steps_hint) {
    free_list(b->asg_allocs);
    b->cps = cps;
    b->G = cps * b->sm;
    const int G = b->G;
    const size_t nt = b->h_tiles.size();
    std::vector<double> cost(nt);
    for (size_t t = 0; t < nt; ++t) {
        const BatchTileDev &td = b->h_tiles[t];
        cost[t] = tile_cost(b, b->inst[td.inst], td, b->rate_hz[td.inst], n_steps_hint);
    }
    std::vector<int> order(nt);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    using Load = std::pair<double, int>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> pq;
    for (int c = 0; c < G; ++c) pq.push({0.0, c});
    std::vector<std::vector<int>> lists(G);
    for (int t : order) {
        Load l = pq.top();
        pq.pop();
        lists[l.second].push_back(t);
        pq.push({l.first + cost[t], l.second});
    }
    std::vector<int> cptr(G + 1, 0), ctiles;
    for (int c = 0; c < G; ++c) {
        std::sort(lists[c].begin(), lists[c].end());
        cptr[c + 1] = cptr[c] + static_cast<int>(lists[c].size());
        ctiles.insert(ctiles.end(), lists[c].begin(), lists[c].end());
    }
    int rc = balloc_t(b->asg_allocs, &b->d_cta_ptr, G + 1);
    if (!rc) rc = balloc_t(b->asg_allocs, &b->d_cta_tiles, std::max<size_t>(ctiles.size(), 1));
    if (!rc) rc = balloc_t(b->asg_allocs, &b->d_rec_count, G);
    if (rc) return rc;
    BSPK_CUDA(cudaMemcpyAsync(b->d_cta_ptr, cptr.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, b->st));
    if (!ctiles.empty())
        BSPK_CUDA(cudaMemcpyAsync(b->d_cta_tiles, ctiles.data(), sizeof(int) * ctiles.size(),
                                  cudaMemcpyHostToDevice, b->st));
    BSPK_CUDA(cudaMemsetAsync(b->d_rec_count, 0, sizeof(long long) * G, b->st));
    b->spk_cap = 0;
    b->d_spk_step = nullptr;
    b->d_spk_id = b->d_spk_inst = nullptr;
    if (b->any_record) {
        b->spk_cap = std::max<int64_t>(1024, b->cfg.spike_capacity / G);
        rc = balloc_t(b->asg_allocs, &b->d_spk_step, b->spk_cap * G);
        if (!rc) rc = balloc_t(b->asg_allocs, &b->d_spk_id, b->spk_cap * G);
        if (!rc) rc = balloc_t(b->asg_allocs, &b->d_spk_inst, b->spk_cap * G);
        if (rc) return rc;
    }
    BSPK_CUDA(cudaStreamSynchronize(b->st));
    return BSPK_OK;
}

int max_cps(bspk_batch *b, int T) {
    return b->elt == 8 ? lif_batch_max_ctas_per_sm<double>(b->cfg.model, T, b->Wmax)
                       : lif_batch_max_ctas_per_sm<float>(b->cfg.model, T, b->Wmax);
}

// One run: in chunks of at most kBatchDriveBudget bytes of drive, each a
// drive pass over (step, neuron) then the persistent kernel.
constexpr size_t kBatchDriveBudget = size_t(4) << 30;

template <typename Real>
int launch_typed(bspk_batch *b, int64_t n_steps, cudaStream_t st) {
    using Fix = typename FixOf<Real>::type;
    const size_t per_step = sizeof(Real) * static_cast<size_t>(b->Ntot);
    int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_steps, kBatchDriveBudget / per_step));
    if (chunk >= b->Wmax && chunk < n_steps) chunk -= chunk % b->Wmax;  // whole windows when they share W
    if (b->drive_steps < chunk) {
        for (auto it = b->allocs.begin(); it != b->allocs.end(); ++it)
            if (*it == b->d_drive) {
                cudaFree(*it);
                b->allocs.erase(it);
                break;
            }
        b->d_drive = nullptr;
        int rc = balloc(b->allocs, &b->d_drive, per_step * chunk);
        if (rc) return rc;
        b->drive_steps = chunk;
    }
    BSPK_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(int), st));
    if (b->d_rec_count) BSPK_CUDA(cudaMemsetAsync(b->d_rec_count, 0, sizeof(long long) * b->G, st));
    BSPK_CUDA(cudaEventRecord(b->ev0, st));
    int64_t launches = 0;
    for (int64_t done = 0; done < n_steps; done += chunk) {
        const int64_t n = std::min<int64_t>(chunk, n_steps - done);
        BatchArgs<Real> a{};
        a.n_tiles = static_cast<int>(b->h_tiles.size());
        a.n_inst = static_cast<int>(b->inst.size());
        a.T = b->T;
        a.Wmax = b->Wmax;
        a.inst = b->d_inst;
        a.tiles = b->d_tiles;
        a.cta_ptr = b->d_cta_ptr;
        a.cta_tiles = b->d_cta_tiles;
        a.drives = b->d_drives;
        a.cdf = b->d_cdf;
        a.r = b->d_r;
        a.ptr = b->d_ptr;
        a.edges = b->d_edges;
        a.recs = b->d_recs;
        a.part = b->d_part;
        a.spk_cnt = b->d_cnt;
        a.spk_step = b->d_spk_step;
        a.spk_id = b->d_spk_id;
        a.spk_inst = b->d_spk_inst;
        a.rec_count = b->d_rec_count;
        a.spk_cap = b->spk_cap;
        a.step0 = b->step + done;
        a.n_steps = n;
        a.n_total = b->Ntot;
        a.drive = static_cast<const Real *>(b->d_drive);
        a.drive_step0 = a.step0;
        a.err = b->d_err;
        a.coef = static_cast<const PopCoef<Real> *>(b->d_coef);
        a.proj_w = static_cast<const Fix *>(b->d_projw);
        for (int i = 0; i < 6; ++i) a.s[i] = static_cast<Real *>(b->d_s[i]);
        cudaError_t e = launch_batch_drive_fill<Real>(a, a.step0, static_cast<int>(n),
                                                      static_cast<Real *>(b->d_drive), st);
        if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("drive launch: ") + cudaGetErrorString(e));
        e = launch_lif_batch<Real>(a, b->cfg.model, b->G, st);
        if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
        launches += 2;
    }
    BSPK_CUDA(cudaEventRecord(b->ev1, st));
    b->last_launches = launches;
    b->step += n_steps;
    return BSPK_OK;
}

int launch(bspk_batch *b, int64_t n_steps, cudaStream_t st) {
    return b->elt == 8 ? launch_typed<double>(b, n_steps, st) : launch_typed<float>(b, n_steps, st);
}

int check_err(bspk_batch *b, cudaStream_t st) {
    int err = 0;
    BSPK_CUDA(cudaMemcpyAsync(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BSPK_CUDA(cudaStreamSynchronize(st));
    if (err == BSPK_DEV_ERR_TIMEOUT) return fail(BSPK_ERR_TIMEOUT, "a bounded device wait ran out");
    if (err == BSPK_DEV_ERR_OVERFLOW) return fail(BSPK_ERR_OVERFLOW, "spike record overflow");
    if (err) return fail(BSPK_ERR_CUDA, "device error " + std::to_string(err));
    return BSPK_OK;
}

// Snapshot of the evolving state (for the tuner's pilot runs).
struct Snapshot {
    std::vector<void *> bufs;
};

int snapshot(bspk_batch *b, Snapshot &s) {
    const size_t sb = static_cast<size_t>(b->elt) * b->Ntot;
    for (int i = 0; i < 6; ++i) {
        void *p = nullptr;
        BSPK_CUDA(cudaMalloc(&p, sb));
        BSPK_CUDA(cudaMemcpy(p, b->d_s[i], sb, cudaMemcpyDeviceToDevice));
        s.bufs.push_back(p);
    }
    void *p = nullptr;
    BSPK_CUDA(cudaMalloc(&p, 4 * b->Ntot));
    BSPK_CUDA(cudaMemcpy(p, b->d_r, 4 * b->Ntot, cudaMemcpyDeviceToDevice));
    s.bufs.push_back(p);
    return BSPK_OK;
}

int restore(bspk_batch *b, const Snapshot &s) {
    const size_t sb = static_cast<size_t>(b->elt) * b->Ntot;
    for (int i = 0; i < 6; ++i) BSPK_CUDA(cudaMemcpy(b->d_s[i], s.bufs[i], sb, cudaMemcpyDeviceToDevice));
    BSPK_CUDA(cudaMemcpy(b->d_r, s.bufs[6], 4 * b->Ntot, cudaMemcpyDeviceToDevice));
    BSPK_CUDA(cudaMemset(b->d_cnt, 0, 4 * b->Ntot));
    BSPK_CUDA(cudaMemset(b->d_recs, 0, sizeof(unsigned long long) * b->rec_words));
    BSPK_CUDA(cudaMemset(b->d_part, 0, sizeof(int) * (b->h_tiles.size() + 1)));
    BSPK_CUDA(cudaDeviceSynchronize());
    b->step = 0;
    return BSPK_OK;
}

void drop(Snapshot &s) {
    for (void *p : s.bufs) cudaFree(p);
    s.bufs.clear();
}

}  // namespace

extern "C" {

int bspk_batch_create(const bspk_config *cfg, bspk_batch **out) {
    if (!cfg || !out) return fail(BSPK_ERR_ARG, "null argument");
    if (!(cfg->dt > 0)) return fail(BSPK_ERR_ARG, "dt must be > 0");
    if (cfg->precision != 32 && cfg->precision != 64) return fail(BSPK_ERR_ARG, "precision must be 32 or 64");
    if (cfg->model != BSPK_IAF_PSC_ALPHA && cfg->model != BSPK_IAF_PSC_EXP)
        return fail(BSPK_ERR_UNSUPPORTED, "batches run iaf_psc_alpha or iaf_psc_exp instances");
    if (cfg->semantics != BSPK_LEGACY && cfg->semantics != BSPK_RING)
        return fail(BSPK_ERR_ARG, "unknown delivery semantics");
    if (cfg->deterministic) return fail(BSPK_ERR_UNSUPPORTED, "batches have no deterministic mode");
    bspk_batch *b = new bspk_batch();
    b->cfg = *cfg;
    if (b->cfg.spike_capacity <= 0) b->cfg.spike_capacity = 1 << 22;
    b->elt = cfg->precision == 64 ? 8 : 4;
    *out = b;
    return BSPK_OK;
}

int bspk_batch_destroy(bspk_batch *b) {
    if (!b) return BSPK_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    if (b->uploaded) cudaSetDevice(b->cfg.device);
    free_list(b->asg_allocs);
    free_list(b->lay_allocs);
    free_list(b->allocs);
    b->gen.release();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    cudaSetDevice(dev);
    delete b;
    return BSPK_OK;
}

int bspk_batch_instance_add(bspk_batch *b, int *inst) {
    if (!b) return fail(BSPK_ERR_ARG, "null batch");
    if (b->uploaded) return fail(BSPK_ERR_STATE, "batch already uploaded");
    b->inst.emplace_back();
    if (inst) *inst = static_cast<int>(b->inst.size()) - 1;
    return BSPK_OK;
}

int bspk_batch_pop_add(bspk_batch *b, int inst, int n, const double *params, int n_params, int *pop) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (b->uploaded) return fail(BSPK_ERR_STATE, "batch already uploaded");
    if (n <= 0 || !params) return fail(BSPK_ERR_ARG, "bad population");
    BInst &I = b->inst[inst];
    if (static_cast<int>(I.pops.size()) >= kBatchMaxPops) return fail(BSPK_ERR_ARG, "too many populations");
    if (static_cast<int64_t>(I.n) + n >= (int64_t(1) << (32 - kBatchStepBits)))
        return fail(BSPK_ERR_ARG, "instance too large");
    BPop P;
    P.n = n;
    P.off = I.n;
    P.p.assign(params, params + n_params);
    rc = host_make_coef(b->cfg.model, P.p, b->cfg.dt, &P.c);
    if (rc) return rc;
    P.c.off = P.off;
    P.c.n = n;
    I.pops.push_back(std::move(P));
    I.n += n;
    if (pop) *pop = static_cast<int>(I.pops.size()) - 1;
    return BSPK_OK;
}

int bspk_batch_fixed_indegree_add(bspk_batch *b, int inst, int pre_pop, int post_pop, int K,
                                  int64_t seed, int allow_autapses, int nbits, double weight,
                                  int delay_steps) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (b->uploaded) return fail(BSPK_ERR_STATE, "batch already uploaded");
    BInst &I = b->inst[inst];
    const int np = static_cast<int>(I.pops.size());
    if (pre_pop < 0 || pre_pop >= np || post_pop < 0 || post_pop >= np)
        return fail(BSPK_ERR_ARG, "population index out of range");
    if (static_cast<int>(I.projs.size()) >= kBatchMaxProj) return fail(BSPK_ERR_ARG, "too many projections");
    if (K < 0) return fail(BSPK_ERR_ARG, "K must be >= 0");
    if (nbits != 32 && nbits != 64) return fail(BSPK_ERR_ARG, "nbits must be 32 or 64");
    if (delay_steps < 1) return fail(BSPK_ERR_ARG, "delay must be at least one step");
    const bool excl = pre_pop == post_pop && !allow_autapses;
    if (K > 0 && (excl ? I.pops[pre_pop].n - 1 : I.pops[pre_pop].n) <= 0)
        return fail(BSPK_ERR_ARG, "no candidate pre neurons");
    const int lag = lag_of(b, delay_steps);
    for (const auto &Q : I.projs)
        if (Q.lag != lag)
            return fail(BSPK_ERR_UNSUPPORTED, "a batch instance needs one delay for all its projections");
    if (lag > kBatchMaxWindow) return fail(BSPK_ERR_UNSUPPORTED, "delay longer than 64 steps");
    BProj P;
    P.pre = pre_pop;
    P.post = post_pop;
    P.K = K;
    P.seed = seed;
    P.autapses = allow_autapses ? 1 : 0;
    P.nbits = nbits;
    P.w = weight;
    P.lag = lag;
    I.projs.push_back(P);
    I.edges += static_cast<int64_t>(I.pops[post_pop].n) * K;
    return BSPK_OK;
}

int bspk_batch_drive_add_poisson(bspk_batch *b, int inst, int post_pop, double rate_hz,
                                 double weight, int delay_steps, uint32_t seed, int64_t t_min_step,
                                 int64_t t_max_step) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (b->uploaded) return fail(BSPK_ERR_STATE, "batch already uploaded");
    BInst &I = b->inst[inst];
    if (post_pop < 0 || post_pop >= static_cast<int>(I.pops.size()))
        return fail(BSPK_ERR_ARG, "population index out of range");
    if (static_cast<int>(I.drives.size()) >= kBatchMaxDrives) return fail(BSPK_ERR_ARG, "too many drives");
    const double lam = rate_hz * b->cfg.dt / 1000.0;
    if (!(lam >= 0) || lam > 700.0) return fail(BSPK_ERR_ARG, "rate*dt/1000 must be in [0, 700]");
    if (delay_steps < 0) return fail(BSPK_ERR_ARG, "negative delay");
    BDrive D;
    D.post = post_pop;
    D.lag = lag_of(b, delay_steps);
    D.rate = rate_hz;
    D.weight = weight;
    D.seed = seed;
    D.tmin = t_min_step;
    D.tmax = rate_hz > 0 ? t_max_step : t_min_step;
    D.cdf = host_poisson_thresholds(lam);
    if (I.cdf_n + static_cast<int>(D.cdf.size()) > kBatchCdfCap)
        return fail(BSPK_ERR_UNSUPPORTED, "Poisson tables of an instance exceed 1024 entries");
    I.cdf_n += static_cast<int>(D.cdf.size());
    I.drives.push_back(std::move(D));
    return BSPK_OK;
}

int bspk_batch_record_spikes(bspk_batch *b, int inst, int on) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (b->uploaded) return fail(BSPK_ERR_STATE, "batch already uploaded");
    b->inst[inst].record = on ? 1 : 0;
    return BSPK_OK;
}

int bspk_batch_upload(bspk_batch *b, int tile, int ctas_per_sm, void *stream) {
    if (!b) return fail(BSPK_ERR_ARG, "null batch");
    if (b->uploaded) return fail(BSPK_ERR_STATE, "batch already uploaded");
    if (b->inst.empty()) return fail(BSPK_ERR_ARG, "empty batch");
    if (tile == 0) tile = 256;
    if (tile < 32 || tile > 512 || tile % 32) return fail(BSPK_ERR_ARG, "tile must be a multiple of 32 in [32, 512]");
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    cudaDeviceProp prop;
    BSPK_CUDA(cudaGetDeviceProperties(&prop, b->cfg.device));
    if (!prop.cooperativeLaunch) return fail(BSPK_ERR_UNSUPPORTED, "device lacks cooperative launch");
    b->sm = prop.multiProcessorCount;
    (void)stream;
    BSPK_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    BSPK_CUDA(cudaEventCreate(&b->ev0));
    BSPK_CUDA(cudaEventCreate(&b->ev1));
    // windows, offsets, tables
    b->Ntot = 0;
    b->Wmax = 1;
    b->any_record = false;
    std::vector<PopCoef<double>> coef;
    std::vector<DriveDev> drives;
    std::vector<uint64_t> cdf;
    std::vector<double> projw(b->inst.size() * kBatchMaxProj, 0.0);
    for (size_t i = 0; i < b->inst.size(); ++i) {
        BInst &I = b->inst[i];
        if (I.pops.empty()) return fail(BSPK_ERR_ARG, "instance without neurons");
        I.W = I.projs.empty() ? 16 : I.projs[0].lag;
        if (I.W < 1) return fail(BSPK_ERR_UNSUPPORTED, "recurrent arrival lag must be >= 1 step");
        b->Wmax = std::max(b->Wmax, I.W);
        I.g0 = b->Ntot;
        b->Ntot += I.n;
        b->any_record = b->any_record || I.record;
        for (const auto &P : I.pops) coef.push_back(P.c);
        int coff = 0;
        for (const auto &D : I.drives) {
            DriveDev d{};
            d.pop = D.post;
            d.lag = D.lag;
            d.seed = D.seed;
            d.cdf_off = coff;
            d.cdf_n = static_cast<int>(D.cdf.size());
            d.receptor = 0;
            d.weight = D.weight;
            d.tmin = D.tmin;
            d.tmax = D.tmax;
            drives.push_back(d);
            cdf.insert(cdf.end(), D.cdf.begin(), D.cdf.end());
            coff += d.cdf_n;
        }
        // fixed-point scale: an edge adds at most once per arrival step, so
        // no slot exceeds the largest per-neuron sum of |w| over in-edges
        std::vector<double> wsum(I.pops.size(), 0.0);
        for (const auto &P : I.projs) wsum[P.post] += std::fabs(P.w) * P.K;
        const double wmax = *std::max_element(wsum.begin(), wsum.end());
        const double limit = b->elt == 8 ? 4.0e18 : 2.0e9;
        int k = 40;
        if (wmax > 0.0) k = static_cast<int>(std::floor(std::log2(limit / wmax)));
        k = std::max(-60, std::min(k, b->elt == 8 ? 100 : 60));
        I.inv_scale = std::ldexp(1.0, -k);
        for (size_t p = 0; p < I.projs.size(); ++p)
            projw[i * kBatchMaxProj + p] = static_cast<double>(std::llrint(std::ldexp(I.projs[p].w, k)));
    }
    if (lif_batch_smem(tile, b->Wmax, b->elt == 8) > 160 * 1024)
        return fail(BSPK_ERR_UNSUPPORTED, "tile x window accumulator exceeds shared memory");
    b->rate_hz.assign(b->inst.size(), 10.0);
    // static buffers: SoA state, refractory counts, spike counts, tables
    const size_t sb = static_cast<size_t>(b->elt) * b->Ntot;
    int rc = BSPK_OK;
    for (int i = 0; i < 6 && !rc; ++i) rc = balloc(b->allocs, &b->d_s[i], sb);
    if (!rc) rc = balloc_t(b->allocs, &b->d_r, b->Ntot);
    if (!rc) rc = balloc_t(b->allocs, &b->d_cnt, b->Ntot);
    if (!rc) rc = balloc(b->allocs, &b->d_coef, (b->elt == 8 ? sizeof(PopCoef<double>) : sizeof(PopCoef<float>)) * coef.size());
    if (!rc) rc = balloc_t(b->allocs, &b->d_drives, std::max<size_t>(drives.size(), 1));
    if (!rc) rc = balloc_t(b->allocs, &b->d_cdf, std::max<size_t>(cdf.size(), 1));
    if (!rc) rc = balloc(b->allocs, &b->d_projw, static_cast<size_t>(b->elt) * projw.size());
    if (!rc) rc = balloc_t(b->allocs, &b->d_err, 1);
    if (rc) return rc;
    if (b->elt == 8) {
        BSPK_CUDA(cudaMemcpy(b->d_coef, coef.data(), sizeof(PopCoef<double>) * coef.size(), cudaMemcpyHostToDevice));
        std::vector<long long> pw(projw.size());
        for (size_t q = 0; q < projw.size(); ++q) pw[q] = static_cast<long long>(projw[q]);
        BSPK_CUDA(cudaMemcpy(b->d_projw, pw.data(), 8 * pw.size(), cudaMemcpyHostToDevice));
    } else {
        std::vector<PopCoef<float>> cf;
        for (const auto &c : coef) cf.push_back(cast_coef<float>(c));
        std::vector<int32_t> pw(projw.size());
        for (size_t q = 0; q < projw.size(); ++q) pw[q] = static_cast<int32_t>(projw[q]);
        BSPK_CUDA(cudaMemcpy(b->d_coef, cf.data(), sizeof(PopCoef<float>) * cf.size(), cudaMemcpyHostToDevice));
        BSPK_CUDA(cudaMemcpy(b->d_projw, pw.data(), 4 * pw.size(), cudaMemcpyHostToDevice));
    }
    if (!drives.empty())
        BSPK_CUDA(cudaMemcpy(b->d_drives, drives.data(), sizeof(DriveDev) * drives.size(), cudaMemcpyHostToDevice));
    if (!cdf.empty())
        BSPK_CUDA(cudaMemcpy(b->d_cdf, cdf.data(), sizeof(uint64_t) * cdf.size(), cudaMemcpyHostToDevice));
    // initial state: V_m = E_L, everything else 0
    {
        std::vector<double> v(b->Ntot);
        for (const auto &I : b->inst)
            for (const auto &P : I.pops)
                for (int k = 0; k < P.n; ++k) v[I.g0 + P.off + k] = P.c.E_L;
        for (int i = 0; i < 6; ++i) {
            if (i > 0) std::fill(v.begin(), v.end(), 0.0);
            if (b->elt == 8) {
                BSPK_CUDA(cudaMemcpy(b->d_s[i], v.data(), sb, cudaMemcpyHostToDevice));
            } else {
                std::vector<float> f(v.begin(), v.end());
                BSPK_CUDA(cudaMemcpy(b->d_s[i], f.data(), sb, cudaMemcpyHostToDevice));
            }
        }
        BSPK_CUDA(cudaMemset(b->d_r, 0, 4 * b->Ntot));
        BSPK_CUDA(cudaMemset(b->d_cnt, 0, 4 * b->Ntot));
    }
    rc = layout(b, tile);
    if (rc) return rc;
    const int mc = max_cps(b, tile);
    if (mc < 1) return fail(BSPK_ERR_UNSUPPORTED, "batch kernel does not fit on an SM with this tile");
    if (ctas_per_sm <= 0 || ctas_per_sm > mc) ctas_per_sm = mc;
    rc = assign(b, ctas_per_sm, 10000);
    if (rc) return rc;
    BSPK_CUDA(cudaDeviceSynchronize());
    b->uploaded = true;
    b->step = 0;
    return BSPK_OK;
}

int bspk_batch_run(bspk_batch *b, int64_t n_steps, void *stream) {
    if (!b || !b->uploaded) return fail(BSPK_ERR_STATE, "batch not uploaded");
    if (n_steps < 0) return fail(BSPK_ERR_ARG, "negative step count");
    if (n_steps == 0) return BSPK_OK;
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->st;
    int rc = launch(b, n_steps, st);
    if (rc) return rc;
    return check_err(b, st);
}

int bspk_batch_tune(bspk_batch *b, int64_t pilot_steps, int *tile_out, int *ctas_per_sm_out,
                    double *pilot_ms_out) {
    if (!b || !b->uploaded) return fail(BSPK_ERR_STATE, "batch not uploaded");
    if (b->step != 0) return fail(BSPK_ERR_STATE, "tune before the first run");
    if (pilot_steps <= 0) return fail(BSPK_ERR_ARG, "pilot_steps must be > 0");
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    Snapshot s0;
    int rc = snapshot(b, s0);
    // 1. rates of every instance from a pilot with the current shape
    if (!rc) rc = launch(b, pilot_steps, b->st);
    if (!rc) rc = check_err(b, b->st);
    if (!rc) {
        std::vector<unsigned int> cnt(b->Ntot);
        if (cudaMemcpy(cnt.data(), b->d_cnt, 4 * b->Ntot, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(BSPK_ERR_CUDA, "copy of spike counts failed");
        for (size_t i = 0; !rc && i < b->inst.size(); ++i) {
            const BInst &I = b->inst[i];
            double tot = 0.0;
            for (int k = 0; k < I.n; ++k) tot += cnt[I.g0 + k];
            b->rate_hz[i] = tot / I.n / (pilot_steps * b->cfg.dt * 1e-3);
        }
    }
    if (!rc) rc = restore(b, s0);
    // 2. tile size x CTAs per SM, each timed on the same pilot
    double best = 1e300;
    int best_T = b->T, best_c = b->cps;
    for (int T : {128, 256, 512}) {
        if (rc) break;
        if (lif_batch_smem(T, b->Wmax, b->elt == 8) > 160 * 1024) continue;
        bool too_many = false;
        for (const auto &I : b->inst) too_many = too_many || (I.n + T - 1) / T > 1024;
        if (too_many) continue;
        rc = layout(b, T);
        const int mc = rc ? 0 : max_cps(b, T);
        for (int c = 1; !rc && c <= std::min(mc, 4); ++c) {
            rc = assign(b, c, 10000);
            if (!rc) rc = launch(b, pilot_steps, b->st);
            if (!rc) rc = check_err(b, b->st);
            float ms = 0.f;
            if (!rc && cudaEventElapsedTime(&ms, b->ev0, b->ev1) != cudaSuccess)
                rc = fail(BSPK_ERR_CUDA, "event timing failed");
            if (!rc && ms < best) {
                best = ms;
                best_T = T;
                best_c = c;
            }
            if (!rc) rc = restore(b, s0);
        }
    }
    if (!rc && best_T != b->T) rc = layout(b, best_T);
    if (!rc) rc = assign(b, best_c, 10000);
    if (!rc) rc = restore(b, s0);
    drop(s0);
    if (rc) return rc;
    if (tile_out) *tile_out = best_T;
    if (ctas_per_sm_out) *ctas_per_sm_out = best_c;
    if (pilot_ms_out) *pilot_ms_out = best;
    return BSPK_OK;
}

int bspk_batch_shape(bspk_batch *b, int *tile, int *ctas_per_sm, int *grid, int64_t *n_tiles) {
    if (!b || !b->uploaded) return fail(BSPK_ERR_STATE, "batch not uploaded");
    if (tile) *tile = b->T;
    if (ctas_per_sm) *ctas_per_sm = b->cps;
    if (grid) *grid = b->G;
    if (n_tiles) *n_tiles = static_cast<int64_t>(b->h_tiles.size());
    return BSPK_OK;
}

int bspk_batch_state_set(bspk_batch *b, int inst, int pop, const char *name, const double *values) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (!b->uploaded) return fail(BSPK_ERR_STATE, "batch not uploaded");
    const BInst &I = b->inst[inst];
    if (pop < 0 || pop >= static_cast<int>(I.pops.size()) || !name || !values)
        return fail(BSPK_ERR_ARG, "bad arguments");
    const BPop &P = I.pops[pop];
    const int64_t g = I.g0 + P.off;
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    if (!strcmp(name, "r") || !strcmp(name, "refractory_step_count")) {
        std::vector<int> r(P.n);
        for (int k = 0; k < P.n; ++k) r[k] = static_cast<int>(values[k]);
        BSPK_CUDA(cudaMemcpy(b->d_r + g, r.data(), 4 * P.n, cudaMemcpyHostToDevice));
        BSPK_CUDA(cudaDeviceSynchronize());
        return BSPK_OK;
    }
    int slot = -1;
    for (int i = 0; i < 6; ++i)
        if (kIafStateNames[b->cfg.model][i][0] && !strcmp(kIafStateNames[b->cfg.model][i], name)) slot = i;
    if (slot < 0) return fail(BSPK_ERR_ARG, std::string("unknown state ") + name);
    char *base = static_cast<char *>(b->d_s[slot]) + static_cast<size_t>(b->elt) * g;
    if (b->elt == 8) {
        BSPK_CUDA(cudaMemcpy(base, values, 8 * P.n, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(values, values + P.n);
        BSPK_CUDA(cudaMemcpy(base, f.data(), 4 * P.n, cudaMemcpyHostToDevice));
    }
    BSPK_CUDA(cudaDeviceSynchronize());
    return BSPK_OK;
}

int bspk_batch_state_get(bspk_batch *b, int inst, int pop, const char *name, double *values) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (!b->uploaded) return fail(BSPK_ERR_STATE, "batch not uploaded");
    const BInst &I = b->inst[inst];
    if (pop < 0 || pop >= static_cast<int>(I.pops.size()) || !name || !values)
        return fail(BSPK_ERR_ARG, "bad arguments");
    const BPop &P = I.pops[pop];
    const int64_t g = I.g0 + P.off;
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    if (!strcmp(name, "r") || !strcmp(name, "refractory_step_count")) {
        std::vector<int> r(P.n);
        BSPK_CUDA(cudaMemcpy(r.data(), b->d_r + g, 4 * P.n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < P.n; ++k) values[k] = r[k];
        return BSPK_OK;
    }
    int slot = -1;
    for (int i = 0; i < 6; ++i)
        if (kIafStateNames[b->cfg.model][i][0] && !strcmp(kIafStateNames[b->cfg.model][i], name)) slot = i;
    if (slot < 0) return fail(BSPK_ERR_ARG, std::string("unknown state ") + name);
    const char *base = static_cast<const char *>(b->d_s[slot]) + static_cast<size_t>(b->elt) * g;
    if (b->elt == 8) {
        BSPK_CUDA(cudaMemcpy(values, base, 8 * P.n, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> f(P.n);
        BSPK_CUDA(cudaMemcpy(f.data(), base, 4 * P.n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < P.n; ++k) values[k] = f[k];
    }
    return BSPK_OK;
}

int bspk_batch_spike_counts(bspk_batch *b, int inst, int64_t *counts) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (!b->uploaded || !counts) return fail(BSPK_ERR_STATE, "batch not uploaded");
    const BInst &I = b->inst[inst];
    std::vector<unsigned int> c(I.n);
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    BSPK_CUDA(cudaMemcpy(c.data(), b->d_cnt + I.g0, 4 * I.n, cudaMemcpyDeviceToHost));
    for (int k = 0; k < I.n; ++k) counts[k] = c[k];
    return BSPK_OK;
}

int bspk_batch_spikes_get(bspk_batch *b, int inst, int64_t cap, int64_t *steps, int32_t *ids,
                          int64_t *n_out) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (!b->uploaded || !n_out) return fail(BSPK_ERR_STATE, "batch not uploaded");
    if (!b->inst[inst].record) return fail(BSPK_ERR_STATE, "spikes of this instance are not recorded");
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    std::vector<long long> rc_n(b->G);
    BSPK_CUDA(cudaMemcpy(rc_n.data(), b->d_rec_count, sizeof(long long) * b->G, cudaMemcpyDeviceToHost));
    int64_t n = 0;
    bool over = false;
    for (int c = 0; c < b->G; ++c) {
        const int64_t m = std::min<int64_t>(rc_n[c], b->spk_cap);
        over = over || rc_n[c] > b->spk_cap;
        if (m == 0) continue;
        std::vector<int64_t> s(m);
        std::vector<int32_t> id(m), in(m);
        const size_t o = static_cast<size_t>(c) * b->spk_cap;
        BSPK_CUDA(cudaMemcpy(s.data(), b->d_spk_step + o, 8 * m, cudaMemcpyDeviceToHost));
        BSPK_CUDA(cudaMemcpy(id.data(), b->d_spk_id + o, 4 * m, cudaMemcpyDeviceToHost));
        BSPK_CUDA(cudaMemcpy(in.data(), b->d_spk_inst + o, 4 * m, cudaMemcpyDeviceToHost));
        for (int64_t q = 0; q < m; ++q) {
            if (in[q] != inst) continue;
            if (n < cap) {
                if (steps) steps[n] = s[q];
                if (ids) ids[n] = id[q];
            }
            ++n;
        }
    }
    *n_out = n;
    if (over) return fail(BSPK_ERR_OVERFLOW, "spike record capacity exceeded in the last run");
    return BSPK_OK;
}

int bspk_batch_edges_get(bspk_batch *b, int inst, int64_t cap, int32_t *pre, int32_t *post,
                         int32_t *proj, int64_t *n_out) {
    int rc = check_inst(b, inst);
    if (rc) return rc;
    if (!b->uploaded || !n_out) return fail(BSPK_ERR_STATE, "batch not uploaded");
    const BInst &I = b->inst[inst];
    const BatchInstDev &d = b->h_inst[inst];
    BSPK_CUDA(cudaSetDevice(b->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    std::vector<int> ptr(static_cast<size_t>(I.ntiles) * I.n + 1);
    std::vector<uint32_t> ed(std::max<int64_t>(I.edges, 1));
    BSPK_CUDA(cudaMemcpy(ptr.data(), b->d_ptr + d.ptr0, 4 * ptr.size(), cudaMemcpyDeviceToHost));
    if (I.edges > 0)
        BSPK_CUDA(cudaMemcpy(ed.data(), b->d_edges + d.edge0, 4 * I.edges, cudaMemcpyDeviceToHost));
    int64_t n = 0;
    for (int t = 0; t < I.ntiles; ++t)
        for (int p = 0; p < I.n; ++p) {
            const size_t row = static_cast<size_t>(t) * I.n + p;
            for (int q = ptr[row]; q < ptr[row + 1]; ++q) {
                if (n < cap) {
                    if (pre) pre[n] = p;
                    if (post) post[n] = t * b->T + static_cast<int>(ed[q] & 0xFFFFu);
                    if (proj) proj[n] = static_cast<int>(ed[q] >> 16);
                }
                ++n;
            }
        }
    *n_out = n;
    return BSPK_OK;
}

int64_t bspk_batch_step_count(bspk_batch *b) { return b ? b->step : -1; }

int bspk_batch_last_kernel_time(bspk_batch *b, double *ms, int64_t *launches) {
    if (!b || !b->uploaded) return fail(BSPK_ERR_ARG, "bad arguments");
    BSPK_CUDA(cudaEventSynchronize(b->ev1));
    float f = 0.f;
    BSPK_CUDA(cudaEventElapsedTime(&f, b->ev0, b->ev1));
    if (ms) *ms = f;
    if (launches) *launches = b->last_launches;
    return BSPK_OK;
}

}  // extern "C"
