// host_rng.h -- host-side connectivity sampling with the reference's key
// derivation (jax.random on the threefry PRNG, partitionable layout), and the
// CSR construction of _nest_network/connectivity.py:39-53.
#pragma once
#include <cstdint>
#include <thread>
#include <vector>

namespace bspk {

inline void tf2x32(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1, uint32_t &y0, uint32_t &y1) {
    auto rotl = [](uint32_t v, int r) { return (v << r) | (v >> (32 - r)); };
    const uint32_t k2 = k0 ^ k1 ^ 0x1BD11BDAu;
    const uint32_t ks[3] = {k0, k1, k2};
    static const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
    uint32_t a = x0 + k0, b = x1 + k1;
    for (int g = 1; g <= 5; ++g) {
        const int* r = rot + ((g - 1) & 1) * 4;
        for (int i = 0; i < 4; ++i) {
            a += b;
            b = rotl(b, r[i]);
            b ^= a;
        }
        a += ks[g % 3];
        b += ks[(g + 1) % 3] + static_cast<uint32_t>(g);
    }
    y0 = a;
    y1 = b;
}

// key(seed) -> [seed >> 32, seed & 0xffffffff]; fold_in(k, d) and
// split(k, n)[i] are threefry(k, [0, d]) / threefry(k, [0, i]).
struct JaxKey {
    uint32_t k0, k1;
};
inline JaxKey jax_key(int64_t seed) {
    const uint64_t s = static_cast<uint64_t>(seed);
    return {static_cast<uint32_t>(s >> 32), static_cast<uint32_t>(s)};
}
inline JaxKey jax_fold(JaxKey k, uint32_t d) {
    JaxKey o;
    tf2x32(k.k0, k.k1, 0u, d, o.k0, o.k1);
    return o;
}

// randint(key, (K,), 0, span) with nbits-wide bits: two bit streams from
// split(key, 2), offset = ((hi % span) * (2^nbits % span) + lo % span) % span.
inline void jax_randint_span(JaxKey key, int K, uint64_t span, int nbits, int64_t *out) {
    const JaxKey ka = jax_fold(key, 0), kb = jax_fold(key, 1);
    const uint64_t mask = nbits == 64 ? ~0ull : 0xFFFFFFFFull;
    if (span == 0) span = 1;
    uint64_t mult = (uint64_t(1) << (nbits / 2)) % span;
    mult = ((mult * mult) & mask) % span;
    for (int i = 0; i < K; ++i) {
        uint32_t a0, a1, b0, b1;
        tf2x32(ka.k0, ka.k1, 0u, static_cast<uint32_t>(i), a0, a1);
        tf2x32(kb.k0, kb.k1, 0u, static_cast<uint32_t>(i), b0, b1);
        const uint64_t hi = nbits == 64 ? ((uint64_t(a0) << 32) | a1) : uint64_t(a0 ^ a1);
        const uint64_t lo = nbits == 64 ? ((uint64_t(b0) << 32) | b1) : uint64_t(b0 ^ b1);
        uint64_t off = ((hi % span) * mult) & mask;
        off = (off + lo % span) & mask;
        out[i] = static_cast<int64_t>(off % span);
    }
}

// Legacy fixed_indegree: per post j, K draws with replacement from the
// candidate list (all pres, or all but j without autapses); post-major output.
inline int host_fixed_indegree(int64_t seed, int n_pre, int n_post, int K, bool pre_is_post,
                               bool allow_autapses, int nbits, int32_t *pre, int32_t *post) {
    const JaxKey k_conn = jax_fold(jax_key(seed), 0);  // split(key, 3)[0]
    const bool excl = pre_is_post && !allow_autapses;
    const int ncand = excl ? n_pre - 1 : n_pre;
    if (K > 0 && ncand <= 0) return -1;
    unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (static_cast<int64_t>(n_post) * K < 200000) nth = 1;
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < nth; ++t) {
        ts.emplace_back([=]() {
            std::vector<int64_t> idx(K > 0 ? K : 1);
            for (int j = static_cast<int>(t); j < n_post; j += static_cast<int>(nth)) {
                jax_randint_span(jax_fold(k_conn, static_cast<uint32_t>(j)), K,
                                 static_cast<uint64_t>(ncand), nbits, idx.data());
                for (int k = 0; k < K; ++k) {
                    int64_t c = idx[k];
                    if (excl && c >= j) c += 1;
                    pre[static_cast<int64_t>(j) * K + k] = static_cast<int32_t>(c);
                    post[static_cast<int64_t>(j) * K + k] = j;
                }
            }
        });
    }
    for (auto &th : ts) th.join();
    return 0;
}

// Stable sort of edges by pre (counting sort) -> (order, indices, indptr).
inline void host_csr_structure(const int32_t *pre, const int32_t *post, int64_t E, int n_pre,
                               int64_t *order, int32_t *indices, int64_t *indptr) {
    for (int i = 0; i <= n_pre; ++i) indptr[i] = 0;
    for (int64_t e = 0; e < E; ++e) indptr[pre[e] + 1]++;
    for (int i = 0; i < n_pre; ++i) indptr[i + 1] += indptr[i];
    std::vector<int64_t> fill(indptr, indptr + n_pre);
    for (int64_t e = 0; e < E; ++e) {
        const int64_t q = fill[pre[e]]++;
        order[q] = e;
        indices[q] = post[e];
    }
}

}  // namespace bspk
