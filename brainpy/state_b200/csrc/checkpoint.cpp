// checkpoint.cpp -- snapshot / restore of every evolving device buffer.
//
// Layout: [magic u64][step i64][N i64][bytes of each section in order]:
// state slots, refractory counters, arrival ring, spike history, then per
// plastic projection its FP64 weights and pre/post traces.  Restore is a
// byte copy, so a restored run continues bit-exactly (the Simulator's cont()
// semantics, _nest_network/simulator.py:1822-1839).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "plan_internal.h"

using namespace bspk;

namespace {

constexpr uint64_t kMagic = 0x42535043504B3031ull;  // "BSPCPK01"

struct Section {
    void *ptr;
    size_t bytes;
};

std::vector<Section> sections(bspk_plan *p) {
    std::vector<Section> s;
    const int ns = model_n_slots(p->cfg.model);
    for (int i = 0; i < ns; ++i) s.push_back({p->d_s[i], static_cast<size_t>(p->elt) * p->N});
    s.push_back({p->d_r, sizeof(int) * static_cast<size_t>(p->N)});
    const int R = plan_n_receptors(p);
    s.push_back({p->d_ring, static_cast<size_t>(p->elt) * p->L * R * p->N});
    s.push_back({p->d_hist, sizeof(uint64_t) * static_cast<size_t>(p->N)});
    for (auto &J : p->projs) {
        if (!J.plastic) continue;
        s.push_back({J.d_wplastic, sizeof(double) * J.post_local.size()});
        s.push_back({J.d_pre_trace, sizeof(double) * p->pops[J.pre].n * J.trace_cols()});
        s.push_back({J.d_post_trace, sizeof(double) * p->pops[J.post].n * J.trace_cols()});
    }
    return s;
}

}  // namespace

extern "C" {

int bspk_checkpoint_size(bspk_plan *p, int64_t *bytes) {
    if (!p || !bytes) return fail(BSPK_ERR_ARG, "bad arguments");
    if (!p->uploaded) return fail(BSPK_ERR_STATE, "plan not uploaded");
    size_t total = 3 * sizeof(int64_t);
    for (auto &s : sections(p)) total += s.bytes;
    *bytes = static_cast<int64_t>(total);
    return BSPK_OK;
}

int bspk_checkpoint_save(bspk_plan *p, void *host_buf, int64_t bytes) {
    int64_t need = 0;
    int rc = bspk_checkpoint_size(p, &need);
    if (rc) return rc;
    if (!host_buf || bytes < need) return fail(BSPK_ERR_ARG, "checkpoint buffer too small");
    rc = sync_and_check(p);
    if (rc) return rc;
    char *b = static_cast<char *>(host_buf);
    const int64_t hdr[3] = {static_cast<int64_t>(kMagic), p->step, p->N};
    memcpy(b, hdr, sizeof(hdr));
    b += sizeof(hdr);
    for (auto &s : sections(p)) {
        BSPK_CUDA(cudaMemcpy(b, s.ptr, s.bytes, cudaMemcpyDeviceToHost));
        b += s.bytes;
    }
    return BSPK_OK;
}

int bspk_checkpoint_restore(bspk_plan *p, const void *host_buf, int64_t bytes) {
    int64_t need = 0;
    int rc = bspk_checkpoint_size(p, &need);
    if (rc) return rc;
    if (!host_buf || bytes < need) return fail(BSPK_ERR_ARG, "checkpoint buffer too small");
    const char *b = static_cast<const char *>(host_buf);
    int64_t hdr[3];
    memcpy(hdr, b, sizeof(hdr));
    if (static_cast<uint64_t>(hdr[0]) != kMagic || hdr[2] != p->N)
        return fail(BSPK_ERR_ARG, "checkpoint does not belong to this plan");
    BSPK_CUDA(cudaSetDevice(p->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    b += sizeof(hdr);
    // a pinned source is copied from directly; a pageable one through the
    // plan's pinned staging buffer (one host copy, then host-to-device copies
    // at link speed)
    const size_t body = static_cast<size_t>(need) - sizeof(hdr);
    cudaPointerAttributes attr{};
    const bool pinned = cudaPointerGetAttributes(&attr, host_buf) == cudaSuccess &&
                        attr.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a pageable pointer may leave an error behind
    const char *st = b;
    if (!pinned) {
        rc = plan_stage(p, body);
        if (rc) return rc;
        memcpy(p->h_stage, b, body);
        st = static_cast<const char *>(p->h_stage);
    }
    for (auto &s : sections(p)) {
        BSPK_CUDA(cudaMemcpy(s.ptr, st, s.bytes, cudaMemcpyHostToDevice));
        st += s.bytes;
    }
    p->step = hdr[1];
    p->restart_step = p->step;
    return BSPK_OK;
}

int bspk_host_alloc(int64_t bytes, void **ptr) {
    if (!ptr || bytes < 0) return fail(BSPK_ERR_ARG, "bad arguments");
    *ptr = nullptr;
    if (bytes == 0) return BSPK_OK;
    BSPK_CUDA(cudaHostAlloc(ptr, static_cast<size_t>(bytes), cudaHostAllocDefault));
    return BSPK_OK;
}

int bspk_host_free(void *ptr) {
    if (ptr) BSPK_CUDA(cudaFreeHost(ptr));
    return BSPK_OK;
}

}  // extern "C"
