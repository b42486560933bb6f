// conn_gen.cu -- fixed_indegree connectivity built on the GPU.
//
// Edges are drawn one thread per edge (conn_gen.cuh), keyed by their CSR
// row and sorted with a stable radix sort: the generation order is
// post-major (post j, then draw k), so a stable sort by row reproduces the
// reference's csr_structure (a stable argsort of the post-major edge list
// by pre, _nest_network/connectivity.py:39-53) edge for edge.  Row bounds
// come from the sorted keys (first position of every row).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "conn_gen.cuh"
#include "host_rng.h"
#include "plan_internal.h"

namespace bspk {

namespace {

// mode 0: one projection's CSR, key = pre, value = post (local indices).
// mode 1: batch tile layout, key = tile * n_inst + pre_gid, value =
//         post_in_tile | slot << 16 (pre/post numbered within the instance).
__global__ void k_gen_keys(FixedIndegreeDev g, int mode, int pre_off, int post_off, int n_inst,
                           int tile, uint32_t slot, uint32_t *keys, uint32_t *vals) {
    const int64_t E = static_cast<int64_t>(g.n_post) * g.K;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < E;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int j = static_cast<int>(e / g.K), k = static_cast<int>(e - static_cast<int64_t>(j) * g.K);
        const int c = fixed_indegree_draw(g, j, k);
        if (mode == 0) {
            keys[e] = static_cast<uint32_t>(c);
            vals[e] = static_cast<uint32_t>(j);
        } else {
            const int pre = pre_off + c, post = post_off + j;
            const int t = post / tile;
            keys[e] = static_cast<uint32_t>(t) * static_cast<uint32_t>(n_inst) + static_cast<uint32_t>(pre);
            vals[e] = static_cast<uint32_t>(post - t * tile) | (slot << 16);
        }
    }
}

// ptr[r] = first position q with keys[q] >= r, for r in [0, nrows]; keys sorted.
template <typename P>
__global__ void k_row_bounds(const uint32_t *keys, int64_t E, int64_t nrows, P *ptr) {
    for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q <= E;
         q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t lo = q == 0 ? -1 : static_cast<int64_t>(keys[q - 1]);
        const int64_t hi = q == E ? nrows : static_cast<int64_t>(keys[q]);
        for (int64_t r = lo + 1; r <= hi && r <= nrows; ++r) ptr[r] = static_cast<P>(q);
    }
}

int grid_for(int64_t n) {
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)));
}

}  // namespace

int make_fixed_indegree_dev(int64_t seed, int n_pre, int n_post, int K, bool pre_is_post,
                            bool allow_autapses, int nbits, FixedIndegreeDev *g) {
    if (n_pre <= 0 || n_post < 0 || K < 0) return fail(BSPK_ERR_ARG, "bad fixed_indegree sizes");
    if (nbits != 32 && nbits != 64) return fail(BSPK_ERR_ARG, "nbits must be 32 or 64");
    const bool excl = pre_is_post && !allow_autapses;
    const int ncand = excl ? n_pre - 1 : n_pre;
    if (K > 0 && ncand <= 0) return fail(BSPK_ERR_ARG, "no candidate pre neurons");
    const JaxKey kc = jax_fold(jax_key(seed), 0);
    g->kc0 = kc.k0;
    g->kc1 = kc.k1;
    g->n_pre = n_pre;
    g->n_post = n_post;
    g->K = K;
    g->excl_self = excl ? 1 : 0;
    g->nbits = nbits;
    g->span = static_cast<uint64_t>(ncand > 0 ? ncand : 1);
    const uint64_t mask = nbits == 64 ? ~0ull : 0xFFFFFFFFull;
    uint64_t mult = (uint64_t(1) << (nbits / 2)) % g->span;
    g->mult = ((mult * mult) & mask) % g->span;
    return BSPK_OK;
}

GenScratch::~GenScratch() { release(); }

void GenScratch::release() {
    cudaFree(k0);
    cudaFree(v0);
    cudaFree(k1);
    cudaFree(v1);
    cudaFree(tmp);
    k0 = v0 = k1 = v1 = nullptr;
    tmp = nullptr;
    tmp_bytes = 0;
    cap = 0;
}

int GenScratch::reserve(int64_t E) {
    if (E <= cap) return BSPK_OK;
    release();
    const size_t b = sizeof(uint32_t) * static_cast<size_t>(std::max<int64_t>(E, 1));
    BSPK_CUDA(cudaMalloc(&k0, b));
    BSPK_CUDA(cudaMalloc(&v0, b));
    BSPK_CUDA(cudaMalloc(&k1, b));
    BSPK_CUDA(cudaMalloc(&v1, b));
    cap = E;
    return BSPK_OK;
}

int GenScratch::sort(int64_t E, int end_bit, cudaStream_t st) {
    size_t need = 0;
    BSPK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, k0, k1, v0, v1, E, 0, end_bit, st));
    if (need > tmp_bytes) {
        cudaFree(tmp);
        tmp = nullptr;
        BSPK_CUDA(cudaMalloc(&tmp, need));
        tmp_bytes = need;
    }
    BSPK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, need, k0, k1, v0, v1, E, 0, end_bit, st));
    return BSPK_OK;
}

static int bits_for(uint64_t n) {
    int b = 1;
    while (b < 32 && (uint64_t(1) << b) <= n) ++b;
    return b;
}

// Batch layout of one instance: every fixed_indegree projection's edges
// keyed by (tile, pre) and sorted; row bounds into ptr (int32, relative to
// the instance's first edge), values into edges.
int gen_instance_tiles(GenScratch &sc, const std::vector<FixedIndegreeDev> &gens,
                       const std::vector<int> &pre_off, const std::vector<int> &post_off,
                       const std::vector<int> &slot, int n_inst, int tile, int ntiles,
                       int *d_ptr, uint32_t *d_edges, cudaStream_t st) {
    int64_t E = 0;
    for (const auto &g : gens) E += static_cast<int64_t>(g.n_post) * g.K;
    const int64_t nrows = static_cast<int64_t>(ntiles) * n_inst;
    if (nrows >= (int64_t(1) << 32) || E >= (int64_t(1) << 31))
        return fail(BSPK_ERR_UNSUPPORTED, "instance too large for the batch tile layout");
    int rc = sc.reserve(E);
    if (rc) return rc;
    int64_t at = 0;
    for (size_t p = 0; p < gens.size(); ++p) {
        const int64_t Ep = static_cast<int64_t>(gens[p].n_post) * gens[p].K;
        if (Ep > 0)
            k_gen_keys<<<grid_for(Ep), 256, 0, st>>>(gens[p], 1, pre_off[p], post_off[p], n_inst,
                                                    tile, static_cast<uint32_t>(slot[p]),
                                                    sc.k0 + at, sc.v0 + at);
        at += Ep;
    }
    BSPK_CUDA(cudaGetLastError());
    if (E > 0) {
        rc = sc.sort(E, bits_for(static_cast<uint64_t>(nrows)), st);
        if (rc) return rc;
        BSPK_CUDA(cudaMemcpyAsync(d_edges, sc.v1, sizeof(uint32_t) * E, cudaMemcpyDeviceToDevice, st));
    }
    k_row_bounds<int><<<grid_for(E + 1), 256, 0, st>>>(sc.k1, E, nrows, d_ptr);
    BSPK_CUDA(cudaGetLastError());
    return BSPK_OK;
}

}  // namespace bspk

using namespace bspk;

extern "C" int bspk_gen_fixed_indegree(int device, int64_t seed, int n_pre, int n_post, int K,
                                       int pre_is_post, int allow_autapses, int nbits,
                                       int64_t *indptr, int32_t *post_local) {
    if (!indptr || (!post_local && static_cast<int64_t>(n_post) * K > 0))
        return fail(BSPK_ERR_ARG, "null output");
    FixedIndegreeDev g;
    int rc = make_fixed_indegree_dev(seed, n_pre, n_post, K, pre_is_post != 0,
                                     allow_autapses != 0, nbits, &g);
    if (rc) return rc;
    const int64_t E = static_cast<int64_t>(n_post) * K;
    if (E >= (int64_t(1) << 31)) return fail(BSPK_ERR_UNSUPPORTED, "more than 2^31 edges");
    int prev = 0;
    BSPK_CUDA(cudaGetDevice(&prev));
    BSPK_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    BSPK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    GenScratch sc;
    int64_t *d_ptr = nullptr;
    rc = sc.reserve(E);
    if (!rc && cudaMalloc(&d_ptr, sizeof(int64_t) * (n_pre + 1)) != cudaSuccess)
        rc = fail(BSPK_ERR_CUDA, "cudaMalloc failed");
    if (!rc && E > 0) {
        k_gen_keys<<<grid_for(E), 256, 0, st>>>(g, 0, 0, 0, 0, 1, 0u, sc.k0, sc.v0);
        if (cudaGetLastError() != cudaSuccess) rc = fail(BSPK_ERR_CUDA, "generation launch failed");
        if (!rc) rc = sc.sort(E, bits_for(static_cast<uint64_t>(n_pre)), st);
    }
    if (!rc) {
        k_row_bounds<int64_t><<<grid_for(E + 1), 256, 0, st>>>(sc.k1, E, n_pre, d_ptr);
        if (cudaGetLastError() != cudaSuccess) rc = fail(BSPK_ERR_CUDA, "bounds launch failed");
    }
    if (!rc && cudaMemcpyAsync(indptr, d_ptr, sizeof(int64_t) * (n_pre + 1), cudaMemcpyDeviceToHost,
                               st) != cudaSuccess)
        rc = fail(BSPK_ERR_CUDA, "copy of indptr failed");
    if (!rc && E > 0 &&
        cudaMemcpyAsync(post_local, sc.v1, sizeof(int32_t) * E, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess)
        rc = fail(BSPK_ERR_CUDA, "copy of indices failed");
    if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = fail(BSPK_ERR_CUDA, "generation failed");
    cudaFree(d_ptr);
    sc.release();
    cudaStreamDestroy(st);
    cudaSetDevice(prev);
    return rc;
}
