// conn_gen.cuh -- device-side fixed_indegree sampling with the reference's
// key derivation (_nest_network/connectivity.py:101-135): for post j the K
// pre indices are randint(fold_in(split(key(seed), 3)[0], j), (K,), 0, n_cand)
// with JAX's threefry bits (partitionable layout: counter i -> threefry(key,
// (0, i))), candidates skipping j when autapses are excluded.  The draw of
// edge (j, k) depends only on (seed, j, k), so every edge is one independent
// thread: no ordering, no host round trip.
#pragma once
#include <cstdint>

#include "common.cuh"
#include "conn_gen.h"

namespace bspk {

__device__ __forceinline__ void jax_fold_dev(uint32_t k0, uint32_t k1, uint32_t d, uint32_t &o0,
                                             uint32_t &o1) {
    threefry2x32(k0, k1, 0u, d, o0, o1);
}

// Pre index (local to the pre population) of edge k into post j.
__device__ __forceinline__ int fixed_indegree_draw(const FixedIndegreeDev &g, int j, int k) {
    uint32_t kj0, kj1, ka0, ka1, kb0, kb1;
    jax_fold_dev(g.kc0, g.kc1, static_cast<uint32_t>(j), kj0, kj1);
    jax_fold_dev(kj0, kj1, 0u, ka0, ka1);
    jax_fold_dev(kj0, kj1, 1u, kb0, kb1);
    uint32_t a0, a1, b0, b1;
    threefry2x32(ka0, ka1, 0u, static_cast<uint32_t>(k), a0, a1);
    threefry2x32(kb0, kb1, 0u, static_cast<uint32_t>(k), b0, b1);
    uint64_t off;
    if (g.nbits == 64) {
        const uint64_t hi = (static_cast<uint64_t>(a0) << 32) | a1;
        const uint64_t lo = (static_cast<uint64_t>(b0) << 32) | b1;
        off = (hi % g.span) * g.mult;
        off = off + lo % g.span;
    } else {
        const uint64_t hi = a0 ^ a1, lo = b0 ^ b1;
        off = ((hi % g.span) * g.mult) & 0xFFFFFFFFull;
        off = (off + lo % g.span) & 0xFFFFFFFFull;
    }
    int c = static_cast<int>(off % g.span);
    if (g.excl_self && c >= j) c += 1;
    return c;
}

}  // namespace bspk
