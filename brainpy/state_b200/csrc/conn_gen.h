// conn_gen.h -- host interface of the GPU connectivity builder (conn_gen.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace bspk {

// One fixed_indegree projection's draw parameters (see conn_gen.cuh).
struct FixedIndegreeDev {
    uint32_t kc0, kc1;   // split(key(seed), 3)[0]
    int n_pre, n_post, K;
    int excl_self;       // pre and post are one population, no autapses
    int nbits;           // 32 or 64
    uint64_t span;       // number of candidates
    uint64_t mult;       // (2^(nbits/2) % span)^2 % span, masked to nbits
};

int make_fixed_indegree_dev(int64_t seed, int n_pre, int n_post, int K, bool pre_is_post,
                            bool allow_autapses, int nbits, FixedIndegreeDev *g);

// Device scratch of generation + stable radix sort, grown on demand.
struct GenScratch {
    uint32_t *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int64_t cap = 0;
    ~GenScratch();
    void release();
    int reserve(int64_t E);
    int sort(int64_t E, int end_bit, cudaStream_t st);
};

// Tile layout of one batch instance: the edges of every projection keyed by
// (tile, pre) and sorted stably; bounds ptr[tile * n_inst + pre] (int32,
// ntiles * n_inst + 1 entries) relative to the instance's first edge and
// edge words post_in_tile | slot << 16.
int gen_instance_tiles(GenScratch &sc, const std::vector<FixedIndegreeDev> &gens,
                       const std::vector<int> &pre_off, const std::vector<int> &post_off,
                       const std::vector<int> &slot, int n_inst, int tile, int ntiles,
                       int *d_ptr, uint32_t *d_edges, cudaStream_t st);

}  // namespace bspk
