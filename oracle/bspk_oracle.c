/*
 * bspk_oracle.c -- float64 CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * A single-threaded restatement of the reference's network step, written to
 * follow the reference's own structure rather than the GPU's: every
 * projection builds a dense contribution vector that is added to the post
 * population's input in creation order, exactly as the reference Simulator
 * does.  Each function cites the reference file:line it restates (paths are
 * relative to the brainspike project root).
 *
 * Compile with -ffp-contract=off: the reference's float64 arithmetic is
 * unfused multiply and add.
 */
#include "bspk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ RNG */

static inline uint32_t rotl32(uint32_t v, int r) { return (v << r) | (v >> (32 - r)); }

/* Threefry-2x32-20 (Salmon, Moraes, Dror, Shaw, SC'11): 5 groups of 4
 * rounds, rotation schedule {13,15,26,6},{17,29,16,24}, key schedule with
 * parity constant 0x1BD11BDA, key injection after every group. */
void bo_threefry2x32(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1,
                     uint32_t *y0, uint32_t *y1) {
    static const int R[2][4] = {{13, 15, 26, 6}, {17, 29, 16, 24}};
    uint32_t ks[3] = {k0, k1, k0 ^ k1 ^ 0x1BD11BDAu};
    uint32_t a = x0 + ks[0], b = x1 + ks[1];
    for (int g = 0; g < 5; ++g) {
        for (int i = 0; i < 4; ++i) {
            a += b;
            b = rotl32(b, R[g & 1][i]);
            b ^= a;
        }
        a += ks[(g + 1) % 3];
        b += ks[(g + 2) % 3] + (uint32_t)(g + 1);
    }
    *y0 = a;
    *y1 = b;
}

/* jax.random.key(seed): [seed >> 32, seed & 0xFFFFFFFF] (JAX threefry_seed). */
void bo_jax_key(int64_t seed, uint32_t key[2]) {
    uint64_t s = (uint64_t)seed;
    key[0] = (uint32_t)(s >> 32);
    key[1] = (uint32_t)(s & 0xFFFFFFFFu);
}

/* jax.random.fold_in(key, data): threefry(key, [0, data]). */
void bo_jax_fold_in(const uint32_t key[2], uint32_t data, uint32_t out[2]) {
    bo_threefry2x32(key[0], key[1], 0u, data, &out[0], &out[1]);
}

/* jax.random.split(key, num), partitionable layout: subkey i =
 * threefry(key, [hi(i), lo(i)]). */
void bo_jax_split(const uint32_t key[2], int num, uint32_t *out) {
    for (int i = 0; i < num; ++i)
        bo_threefry2x32(key[0], key[1], 0u, (uint32_t)i, &out[2 * i], &out[2 * i + 1]);
}

/* random_bits, partitionable layout: element i = threefry(key, [hi(i), lo(i)]);
 * 32-bit -> y0 ^ y1, 64-bit -> (y0 << 32) | y1. */
void bo_jax_random_bits(const uint32_t key[2], int nbits, int64_t n, uint64_t *out) {
    for (int64_t i = 0; i < n; ++i) {
        uint32_t y0, y1;
        bo_threefry2x32(key[0], key[1], (uint32_t)((uint64_t)i >> 32), (uint32_t)i, &y0, &y1);
        out[i] = nbits == 64 ? (((uint64_t)y0 << 32) | y1) : (uint64_t)(y0 ^ y1);
    }
}

void bo_jax_random_bits_at(const uint32_t key[2], int nbits, int64_t i, uint64_t *out) {
    uint32_t y0, y1;
    bo_threefry2x32(key[0], key[1], (uint32_t)((uint64_t)i >> 32), (uint32_t)i, &y0, &y1);
    *out = nbits == 64 ? (((uint64_t)y0 << 32) | y1) : (uint64_t)(y0 ^ y1);
}

/* jax.random.randint(key, (n,), minval, maxval): two bit streams from
 * split(key), remainder combination with multiplier 2**nbits % span, all in
 * nbits-wide unsigned arithmetic. */
void bo_jax_randint(const uint32_t key[2], int64_t n, int64_t minval, int64_t maxval,
                    int nbits, int64_t *out) {
    uint32_t ks[4];
    bo_jax_split(key, 2, ks);
    uint64_t *hb = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    uint64_t *lb = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    bo_jax_random_bits(ks, nbits, n, hb);
    bo_jax_random_bits(ks + 2, nbits, n, lb);
    uint64_t mask = nbits == 64 ? ~0ull : 0xFFFFFFFFull;
    uint64_t span = (uint64_t)(maxval - minval) & mask;
    if (maxval <= minval) span = 1;
    uint64_t mult = ((uint64_t)1 << (nbits / 2)) % span;
    mult = (mult * mult) & mask;
    mult %= span;
    for (int64_t i = 0; i < n; ++i) {
        uint64_t off = (((hb[i] % span) * mult) & mask);
        off = (off + (lb[i] % span)) & mask;
        off %= span;
        out[i] = minval + (int64_t)off;
    }
    free(hb);
    free(lb);
}

/* _nest_network/connectivity.py:101-135 (sample_fixed_indegree) with the
 * projection key of _nest_network/event_proj.py:147-149: key(seed) -> split 3
 * -> k_conn; per post j: choice(fold_in(k_conn, j), candidates, K,
 * replace=True) == candidates[randint(sub, K, 0, len(candidates))]. */
int bo_fixed_indegree(int64_t seed, int n_pre, int n_post, int K, int pre_is_post,
                      int allow_autapses, int nbits, int32_t *pre_out, int32_t *post_out) {
    uint32_t key[2], ks[6], sub[2];
    bo_jax_key(seed, key);
    bo_jax_split(key, 3, ks);
    int64_t *idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)(K > 0 ? K : 1));
    for (int j = 0; j < n_post; ++j) {
        bo_jax_fold_in(ks, (uint32_t)j, sub);
        int excl = pre_is_post && !allow_autapses;
        int ncand = excl ? n_pre - 1 : n_pre;
        if (ncand <= 0 && K > 0) { free(idx); return -1; }
        bo_jax_randint(sub, K, 0, ncand, nbits, idx);
        for (int k = 0; k < K; ++k) {
            int64_t c = idx[k];
            if (excl && c >= j) c += 1; /* candidates = [0..j) ++ (j..n_pre) */
            pre_out[(int64_t)j * K + k] = (int32_t)c;
            post_out[(int64_t)j * K + k] = j;
        }
    }
    free(idx);
    return 0;
}

/* _nest_network/connectivity.py:39-53: stable argsort by pre, bincount indptr */
int bo_csr_structure(const int32_t *pre, const int32_t *post, int64_t n_edges, int n_pre,
                     int64_t *order_out, int32_t *indices_out, int64_t *indptr_out) {
    for (int i = 0; i <= n_pre; ++i) indptr_out[i] = 0;
    for (int64_t e = 0; e < n_edges; ++e) {
        if (pre[e] < 0 || pre[e] >= n_pre) return -1;
        indptr_out[pre[e] + 1]++;
    }
    for (int i = 0; i < n_pre; ++i) indptr_out[i + 1] += indptr_out[i];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_pre + 1));
    memcpy(fill, indptr_out, sizeof(int64_t) * (size_t)(n_pre + 1));
    for (int64_t e = 0; e < n_edges; ++e) { /* counting sort == stable argsort */
        int64_t p = fill[pre[e]]++;
        order_out[p] = e;
        indices_out[p] = post[e];
    }
    free(fill);
    return 0;
}

/* Poisson drive stream (the product's own, restated here): 64 random bits
 * from threefry((seed, stream), (step, idx)), 53-bit uniform, inversion by
 * sequential search.  Replaces jax.random.poisson of
 * _nest_device/poisson_generator.py:492-499 (not reproducible: it depends on
 * XLA's float32 log and a split chain). */
double bo_uniform01(uint32_t seed, uint32_t stream, uint32_t step, uint32_t idx) {
    uint32_t y0, y1;
    bo_threefry2x32(seed, stream, step, idx, &y0, &y1);
    uint64_t b = ((uint64_t)y0 << 32) | y1;
    return (double)(b >> 11) * 0x1.0p-53;
}

/* Inversion by sequential search over the CDF F[0] = exp(-lam),
 * p_k = p_{k-1} * lam / k, F[k] = F[k-1] + p_k; the table ends where F stops
 * growing (at most 4096 entries) and a u beyond it maps to the table length. */
int bo_poisson(double lam, double exp_neg_lam, double u) {
    int k = 0;
    double p = exp_neg_lam, F = p;
    while (u > F) {
        if (k + 1 >= 4096) return k + 1;
        p = p * lam;
        p = p / (double)(k + 1);
        double Fn = F + p;
        if (!(Fn > F)) return k + 1;
        F = Fn;
        k += 1;
    }
    return k;
}

/* ------------------------------------------ jax.random distributions */

/* jax.random.uniform(key, (n,), dtype, minval, maxval) (jax/_src/random.py
 * _uniform): nbits random bits per element (partitionable layout), the top
 * nmant bits OR-ed under the exponent of 1.0, bitcast, minus 1.0, then
 * floats * (maxval - minval) + minval and max(minval, .).  float32 for
 * nbits 32, float64 for 64; every operation rounds in that type. */
void bo_jax_uniform(const uint32_t key[2], int nbits, int64_t n, double lo, double hi,
                    double *out) {
    for (int64_t i = 0; i < n; ++i) {
        uint64_t bits;
        bo_jax_random_bits_at(key, nbits, i, &bits);
        if (nbits == 32) {
            uint32_t b = ((uint32_t)bits >> (32 - 23)) | 0x3F800000u;
            float f;
            memcpy(&f, &b, 4);
            volatile float floats = f - 1.0f;
            volatile float span = (float)hi - (float)lo;
            volatile float scaled = floats * span;
            volatile float v = scaled + (float)lo;
            out[i] = v > (float)lo ? v : (float)lo;
        } else {
            uint64_t b = (bits >> (64 - 52)) | 0x3FF0000000000000ull;
            double f;
            memcpy(&f, &b, 8);
            volatile double floats = f - 1.0;
            volatile double scaled = floats * (hi - lo);
            volatile double v = scaled + lo;
            out[i] = v > lo ? v : lo;
        }
    }
}

/* XLA's float32 ErfInv (M. Giles, "Approximating the erfinv function",
 * single-precision form): w = -log1p(-x*x); w < 5: Horner in w - 2.5, else
 * in sqrt(w) - 3; times x; +-1 -> +-inf. */
static float erfinv32(float x) {
    static const float lt5[9] = {2.81022636e-08f, 3.43273939e-07f, -3.5233877e-06f,
                                 -4.39150654e-06f, 0.00021858087f, -0.00125372503f,
                                 -0.00417768164f, 0.246640727f, 1.50140941f};
    static const float ge5[9] = {-0.000200214257f, 0.000100950558f, 0.00134934322f,
                                 -0.00367342844f, 0.00573950773f, -0.0076224613f,
                                 0.00943887047f, 1.00167406f, 2.83297682f};
    volatile float xx = x * x;
    float w = -log1pf(-xx);
    const float *c = w < 5.0f ? lt5 : ge5;
    w = w < 5.0f ? w - 2.5f : sqrtf(w) - 3.0f;
    float p = c[0];
    for (int i = 1; i < 9; ++i) {
        volatile float pw = p * w;
        p = c[i] + pw;
    }
    if (fabsf(x) == 1.0f) return x * INFINITY;
    return p * x;
}

/* float64 erfinv by bisection on erfl (long double), a different route from
 * the library's Newton steps; the result is the double nearest the root. */
static double erfinv64(double x) {
    if (fabs(x) == 1.0) return x * INFINITY;
    if (x == 0.0) return x;
    long double ax = fabsl((long double)x), a = 0.0L, b = 10.0L;
    for (int it = 0; it < 200; ++it) {
        long double m = 0.5L * (a + b);
        long double f = ax < 0.5L ? erfl(m) - ax : (1.0L - ax) - erfcl(m);
        if (f > 0) b = m; else a = m;  /* f grows with m on both branches */
        if (b - a <= 1e-30L * b) break;
    }
    double y = (double)(0.5L * (a + b));
    return x < 0 ? -y : y;
}

/* jax.random.normal(key, (n,), dtype) (jax/_src/random.py _normal_real):
 * u = uniform(key, minval = nextafter(-1, 0), maxval = 1), then
 * sqrt(2) * erfinv(u) in the dtype. */
void bo_jax_normal(const uint32_t key[2], int nbits, int64_t n, double *out) {
    double *u = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (nbits == 32) {
        bo_jax_uniform(key, 32, n, (double)nextafterf(-1.0f, 0.0f), 1.0, u);
        for (int64_t i = 0; i < n; ++i) {
            volatile float e = erfinv32((float)u[i]);
            out[i] = (float)(1.41421354f * e);
        }
    } else {
        bo_jax_uniform(key, 64, n, nextafter(-1.0, 0.0), 1.0, u);
        for (int64_t i = 0; i < n; ++i) out[i] = 1.4142135623730951 * erfinv64(u[i]);
    }
    free(u);
}

/* ------------------------------------- kernel-path poisson_generator */

static float ftz32(float v) { return fabsf(v) < 1.17549435e-38f ? 0.0f : v; }

/* One unit's count (_kernel/models/devices.py:46-67, _inversion), from the
 * step key of its block and its lane: u = jax.random.uniform(key, (1024,),
 * float32)[lane]; p = exp(-lam); F = p; k = 0; twelve terms k += u >= F,
 * p = p * lam / i, F += p (i = 1..12); then while u >= F and p > 0 the same
 * with i = 13, 14, ...  float32 throughout, subnormal results flushed to
 * zero (XLA's CPU setting). */
int64_t bo_kernel_poisson_count(const uint32_t step_key[2], uint32_t lane, float lam) {
    uint32_t y0, y1;
    bo_threefry2x32(step_key[0], step_key[1], 0u, lane, &y0, &y1);
    uint32_t b = ((y0 ^ y1) >> 9) | 0x3F800000u;
    float f;
    memcpy(&f, &b, 4);
    float u = f - 1.0f;
    float p = ftz32((float)exp(-(double)lam));
    float F = p;
    int64_t k = 0;
    for (int i = 1; i <= 12; ++i) {
        k += u >= F;
        volatile float pl = p * lam;
        p = ftz32(ftz32(pl) / (float)i);
        volatile float Fn = F + p;
        F = Fn;
    }
    for (int i = 13; u >= F && p > 0.0f; ++i) {
        k += 1;
        volatile float pl = p * lam;
        p = ftz32(ftz32(pl) / (float)i);
        volatile float Fn = F + p;
        F = Fn;
    }
    return k;
}

/* The step key of block b of a device population at step n of trial t:
 * fold(fold(fold(obj, b), n), t) (_kernel/rng.py:335-356, 338-420); an
 * unbatched run is trial 0. */
void bo_kernel_step_key_trial(const uint32_t obj[2], uint32_t block, uint32_t step, uint32_t trial,
                              uint32_t out[2]) {
    uint32_t a[2], c[2];
    bo_jax_fold_in(obj, block, a);
    bo_jax_fold_in(a, step, c);
    bo_jax_fold_in(c, trial, out);
}
void bo_kernel_step_key(const uint32_t obj[2], uint32_t block, uint32_t step, uint32_t out[2]) {
    bo_kernel_step_key_trial(obj, block, step, 0u, out);
}

/* ----------------------------------------------------------- propagators */

/* _nest_base/utils.py:177-229 (alpha_propagator_p31_p32), NEST
 * IAFPropagatorAlpha with the singular fallbacks. */
void bo_alpha_p31_p32(double tau_syn, double tau_m, double c_m, double h,
                      double *p31, double *p32) {
    double beta = tau_syn * tau_m / (tau_m - tau_syn);
    double gamma = beta / c_m;
    double inv_beta = (tau_m - tau_syn) / (tau_syn * tau_m);
    double exp_h_tau_syn = exp(-h / tau_syn);
    double expm1_h_tau = expm1(h * inv_beta);
    double p32_raw = gamma * exp_h_tau_syn * expm1_h_tau;
    double exp_h_tau_m = exp(-h / tau_m);
    double p32_singular = h / c_m * exp_h_tau_m;
    int reg32 = isfinite(p32_raw) && fabs(p32_raw) >= 2.2250738585072014e-308 && p32_raw > 0.0;
    *p32 = reg32 ? p32_raw : p32_singular;
    double h_min_regular = 1e-7 * tau_m * tau_m / fabs(tau_m - tau_syn);
    int reg31 = isfinite(h_min_regular) && (h > h_min_regular);
    double p31_regular = gamma * exp_h_tau_syn * (beta * expm1_h_tau - h);
    double p31_singular = 0.5 * h * h / c_m * exp_h_tau_m;
    *p31 = reg31 ? p31_regular : p31_singular;
}

/* _nest_base/utils.py:126-174 (propagator_exp) */
double bo_propagator_exp(double tau_syn, double tau_m, double c_m, double h) {
    double beta = tau_syn * tau_m / (tau_m - tau_syn);
    double gamma = beta / c_m;
    double inv_beta = (tau_m - tau_syn) / (tau_syn * tau_m);
    double exp_h_tau_syn = exp(-h / tau_syn);
    double expm1_h_tau = expm1(h * inv_beta);
    double p32_raw = gamma * exp_h_tau_syn * expm1_h_tau;
    int reg = isfinite(p32_raw) && fabs(p32_raw) >= 2.2250738585072014e-308 && p32_raw > 0.0;
    double p32_singular = h / c_m * exp(-h / tau_m);
    return reg ? p32_raw : p32_singular;
}

/* ------------------------------------------------------------- simulator */

#define NS 9  /* state slots per neuron */
#define RCH 4 /* input channels (receptor ports) per neuron */

typedef struct {
    int n, off;
    double p[24];
    /* iaf_psc_alpha coefficients (_nest_neuron/iaf_psc_alpha.py:451-479) */
    double P11ex, P21ex, P22ex, P11in, P21in, P22in, expm1_tm, P30, P31ex, P32ex,
        P31in, P32in, epsc, ipsc;
    /* iaf_psc_exp coefficients (_nest_neuron/iaf_psc_exp.py:492-512) */
    double eP11ex, eP11in, eP22, eP21ex, eP21in, eP20;
    /* iaf_psc_exp_multisynapse (_nest_neuron/iaf_psc_exp_multisynapse.py:523-552):
     * per-receptor decay and membrane coupling (eP22 / eP20 are the membrane's) */
    double msP11[RCH], msP21[RCH];
    int nrec;
    int ref_count;
} pop_t;

typedef struct {
    int kind; /* 0 csr, 1 drive */
    int pre_pop, post_pop, receptor;
    int64_t n_edges;
    int64_t *indptr;
    int32_t *post, *delay;
    double *w;
    int max_delay;
    int hdelay; /* the one delay of every edge, or -1 when they differ */
    /* drive */
    double rate, weight, lam, enl;
    int ddelay;
    uint32_t seed;
    int64_t tmin, tmax;
    uint32_t trial; /* keyed drive: trial index of its step keys */
    /* keyed drive (the kernel path's stream): object key, first unit, lam */
    int keyed;
    uint32_t okey[2];
    int64_t unit_off;
    float lam32;
    /* stdp */
    int plastic;
    int rule; /* 0: stdp_synapse (pair), 1: stdp_triplet_synapse */
    double tau_plus, tau_minus, lambda_, alpha, mu_plus, mu_minus, wmax, dec_pre, dec_post;
    double *pre_trace, *post_trace;
    /* triplet: slow traces r2 / o2 and the four amplitudes */
    double dec_pre2, dec_post2, a2p, a3p, a2m, a3m;
    double *pre_trace2, *post_trace2;
} input_t;

struct bo_sim {
    double dt;
    int sem, model;
    int ports; /* iaf models: 1 = ports 0 ('ex') / 1 ('in_') apart, signs kept */
    int npop, nin, ntot;
    pop_t pops[64];
    input_t ins[256];
    double *st[NS]; /* SoA state, ntot each */
    int *ref;       /* refractory counters */
    /* spike history: hist[(m mod H) * ntot + gid] */
    int H;
    unsigned char *hist;
    /* ring (RING semantics): ring[ch][slot][gid] */
    int L;
    double *ring;
    int nrec;
    int32_t *rec;
    int64_t step;
    int64_t rk_substeps;
    int threads;  /* OpenMP threads of the independent per-neuron phases */
    uint32_t trial; /* trial index of the keyed drives' step keys */
    double *acc; /* [RCH][ntot] input accumulator */
    double *y;   /* [2][ntot] per-projection vector */
};

static const char *state_names[6][NS] = {
    {"V_m", "I_syn_ex", "dI_syn_ex", "I_syn_in", "dI_syn_in", "y0", "", "", ""},
    {"V_m", "i_syn_ex", "i_syn_in", "i_0", "i_1", "", "", "", ""},
    {"V_m", "dg_ex", "g_ex", "dg_in", "g_in", "w", "h", "I_stim", ""},
    {"V_m", "g_ex", "g_in", "h", "I_stim", "", "", "", ""},
    {"V_m", "dg_ex", "g_ex", "dg_in", "g_in", "h", "I_stim", "", ""},
    {"V_m", "i_const", "i_syn_0", "i_syn_1", "i_syn_2", "i_syn_3", "", "", ""},
};

/* ODE leaves of a conductance model; its slots are the leaves, h, I_stim */
static int n_ode(int model) {
    return model == BO_AEIF_COND_ALPHA ? 6 : (model == BO_IAF_COND_EXP ? 3 : 5);
}

bo_sim *bo_create(double dt, int semantics, int model) {
    bo_sim *s = (bo_sim *)calloc(1, sizeof(bo_sim));
    s->dt = dt;
    s->sem = semantics;
    s->model = model;
    return s;
}

void bo_destroy(bo_sim *s) {
    if (!s) return;
    for (int i = 0; i < NS; ++i) free(s->st[i]);
    free(s->ref);
    free(s->hist);
    free(s->ring);
    free(s->rec);
    free(s->acc);
    free(s->y);
    for (int i = 0; i < s->nin; ++i) {
        input_t *in = &s->ins[i];
        free(in->indptr);
        free(in->post);
        free(in->delay);
        free(in->w);
        free(in->pre_trace);
        free(in->post_trace);
        free(in->pre_trace2);
        free(in->post_trace2);
    }
    free(s);
}

static void grow_state(bo_sim *s, int old_n, int new_n) {
    for (int i = 0; i < NS; ++i) {
        s->st[i] = (double *)realloc(s->st[i], sizeof(double) * (size_t)new_n);
        for (int k = old_n; k < new_n; ++k) s->st[i][k] = 0.0;
    }
    s->ref = (int *)realloc(s->ref, sizeof(int) * (size_t)new_n);
    for (int k = old_n; k < new_n; ++k) s->ref[k] = 0;
}

/* parameter order per model (NEST names):
 * iaf_psc_alpha: E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in I_e V_min
 * iaf_psc_exp:   E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in I_e
 * aeif_cond_alpha: V_peak V_reset t_ref g_L C_m E_ex E_in E_L Delta_T tau_w a b
 *                  V_th tau_syn_ex tau_syn_in I_e gsl_error_tol
 * iaf_cond_exp, iaf_cond_alpha: E_L C_m t_ref V_th V_reset E_ex E_in g_L
 *                  tau_syn_ex tau_syn_in I_e gsl_error_tol
 * iaf_psc_exp_multisynapse: E_L C_m tau_m t_ref V_th V_reset I_e n_receptors
 *                  tau_syn[0..n_receptors-1] (n_receptors <= 4) */
int bo_add_pop(bo_sim *s, int n, const double *params, int n_params) {
    if (s->npop >= 64 || n_params > 24 || n < 0) return -1;
    pop_t *P = &s->pops[s->npop];
    memset(P, 0, sizeof(*P));
    P->n = n;
    P->off = s->ntot;
    memcpy(P->p, params, sizeof(double) * (size_t)n_params);
    double h = s->dt;
    if (s->model == BO_IAF_PSC_ALPHA) {
        double tau_m = P->p[2], c_m = P->p[1], tex = P->p[6], tin = P->p[7];
        P->P11ex = exp(-h / tex);
        P->P22ex = P->P11ex;
        P->P21ex = h * P->P11ex;
        P->P11in = exp(-h / tin);
        P->P22in = P->P11in;
        P->P21in = h * P->P11in;
        P->expm1_tm = expm1(-h / tau_m);
        P->P30 = -tau_m / c_m * P->expm1_tm;
        bo_alpha_p31_p32(tex, tau_m, c_m, h, &P->P31ex, &P->P32ex);
        bo_alpha_p31_p32(tin, tau_m, c_m, h, &P->P31in, &P->P32in);
        P->epsc = 2.718281828459045 / tex;
        P->ipsc = 2.718281828459045 / tin;
        P->ref_count = (int)ceil(P->p[3] / h);
    } else if (s->model == BO_IAF_PSC_EXP) {
        double tau_m = P->p[2], c_m = P->p[1], tex = P->p[6], tin = P->p[7];
        P->eP11ex = exp(-h / tex);
        P->eP11in = exp(-h / tin);
        P->eP22 = exp(-h / tau_m);
        P->eP21ex = bo_propagator_exp(tex, tau_m, c_m, h);
        P->eP21in = bo_propagator_exp(tin, tau_m, c_m, h);
        P->eP20 = tau_m / c_m * (1.0 - exp(-h / tau_m));
        P->ref_count = (int)ceil(P->p[3] / h);
    } else if (s->model == BO_IAF_PSC_EXP_MULTISYNAPSE) {
        double tau_m = P->p[2], c_m = P->p[1];
        P->nrec = (int)P->p[7];
        if (P->nrec < 1 || P->nrec > RCH || n_params < 8 + P->nrec) return -1;
        P->eP22 = exp(-h / tau_m);
        P->eP20 = tau_m / c_m * (1.0 - P->eP22);
        for (int k = 0; k < P->nrec; ++k) {
            P->msP11[k] = exp(-h / P->p[8 + k]);
            P->msP21[k] = bo_propagator_exp(P->p[8 + k], tau_m, c_m, h);
        }
        P->ref_count = (int)ceil(P->p[3] / h);
    } else {
        P->ref_count = (int)ceil(P->p[2] / h);
    }
    int old = s->ntot;
    s->ntot += n;
    grow_state(s, old, s->ntot);
    for (int k = old; k < s->ntot; ++k) {
        if (s->model == BO_AEIF_COND_ALPHA) {
            s->st[0][k] = P->p[7]; /* V_m = E_L */
            s->st[6][k] = h;       /* integration_step = dt (aeif_cond_alpha.py:527) */
        } else if (s->model == BO_IAF_PSC_EXP_MULTISYNAPSE) {
            s->st[0][k] = -70.0; /* V_initializer (iaf_psc_exp_multisynapse.py:406) */
        } else if (s->model == BO_IAF_COND_EXP || s->model == BO_IAF_COND_ALPHA) {
            s->st[0][k] = -70.0;                 /* V_initializer (iaf_cond_exp.py:310) */
            s->st[n_ode(s->model)][k] = h;       /* integration_step = dt */
        } else {
            s->st[0][k] = P->p[0]; /* V_m = E_L */
        }
    }
    return s->npop++;
}

static int state_slot(bo_sim *s, const char *name) {
    if (!strcmp(name, "r")) return 100;
    for (int i = 0; i < NS; ++i)
        if (state_names[s->model][i][0] && !strcmp(state_names[s->model][i], name)) return i;
    return -1;
}

int bo_set_state(bo_sim *s, int pop, const char *name, const double *values) {
    int slot = state_slot(s, name);
    if (slot < 0 || pop < 0 || pop >= s->npop) return -1;
    pop_t *P = &s->pops[pop];
    for (int k = 0; k < P->n; ++k) {
        if (slot == 100) s->ref[P->off + k] = (int)values[k];
        else s->st[slot][P->off + k] = values[k];
    }
    return 0;
}

int bo_get_state(bo_sim *s, int pop, const char *name, double *values) {
    int slot = state_slot(s, name);
    if (slot < 0 || pop < 0 || pop >= s->npop) return -1;
    pop_t *P = &s->pops[pop];
    for (int k = 0; k < P->n; ++k)
        values[k] = slot == 100 ? (double)s->ref[P->off + k] : s->st[slot][P->off + k];
    return 0;
}

int bo_add_proj(bo_sim *s, int pre_pop, int post_pop, int64_t n_edges,
                const int64_t *indptr, const int32_t *post_local, const double *w,
                const int32_t *delay_steps, int receptor) {
    if (s->nin >= 256 || pre_pop < 0 || pre_pop >= s->npop || post_pop < 0 ||
        post_pop >= s->npop)
        return -1;
    if (receptor < 0 || receptor >= RCH) return -1;
    input_t *in = &s->ins[s->nin];
    memset(in, 0, sizeof(*in));
    in->kind = 0;
    in->pre_pop = pre_pop;
    in->post_pop = post_pop;
    in->receptor = receptor;
    in->n_edges = n_edges;
    int npre = s->pops[pre_pop].n;
    in->indptr = (int64_t *)malloc(sizeof(int64_t) * (size_t)(npre + 1));
    memcpy(in->indptr, indptr, sizeof(int64_t) * (size_t)(npre + 1));
    size_t ne = (size_t)(n_edges > 0 ? n_edges : 1);
    in->post = (int32_t *)malloc(sizeof(int32_t) * ne);
    in->delay = (int32_t *)malloc(sizeof(int32_t) * ne);
    in->w = (double *)malloc(sizeof(double) * ne);
    int maxd = 0;
    in->hdelay = n_edges > 0 ? delay_steps[0] : -1;
    for (int64_t e = 0; e < n_edges; ++e) {
        if (post_local[e] < 0 || post_local[e] >= s->pops[post_pop].n) return -2;
        if (delay_steps[e] < (s->sem == BO_RING ? 1 : 0)) return -3;
        in->post[e] = post_local[e];
        in->delay[e] = delay_steps[e];
        in->w[e] = w[e];
        if (delay_steps[e] > maxd) maxd = delay_steps[e];
        if (delay_steps[e] != in->hdelay) in->hdelay = -1;
    }
    in->max_delay = maxd;
    return s->nin++;
}

int bo_add_drive(bo_sim *s, int post_pop, double rate_hz, double weight, int delay_steps,
                 uint32_t seed, int64_t t_min_step, int64_t t_max_step, int receptor) {
    if (s->nin >= 256 || post_pop < 0 || post_pop >= s->npop) return -1;
    if (receptor < 0 || receptor >= RCH) return -1;
    input_t *in = &s->ins[s->nin];
    memset(in, 0, sizeof(*in));
    in->kind = 1;
    in->post_pop = post_pop;
    in->receptor = receptor;
    in->rate = rate_hz;
    in->weight = weight;
    /* lam = rate * dt_ms / 1000 (poisson_generator.py:578) */
    in->lam = rate_hz * s->dt / 1000.0;
    in->enl = exp(-in->lam);
    in->ddelay = delay_steps;
    in->max_delay = delay_steps;
    in->seed = seed;
    in->tmin = t_min_step;
    in->tmax = t_max_step;
    return s->nin++;
}

void bo_set_trial(bo_sim *s, uint32_t trial) {
    s->trial = trial;
    for (int i = 0; i < s->nin; ++i) s->ins[i].trial = trial;
}

int bo_add_drive_keyed(bo_sim *s, int post_pop, double rate_hz, double weight, int delay_steps,
                       const uint32_t okey[2], int64_t unit_off, int64_t t_min_step,
                       int64_t t_max_step, int receptor) {
    int id = bo_add_drive(s, post_pop, rate_hz, weight, delay_steps, 0u, t_min_step, t_max_step,
                          receptor);
    if (id < 0) return id;
    input_t *in = &s->ins[id];
    in->keyed = 1;
    in->trial = s->trial;
    in->okey[0] = okey[0];
    in->okey[1] = okey[1];
    in->unit_off = unit_off;
    /* lam = rate [kHz] * dt [ms] in float32 (_kernel/models/devices.py:203) */
    in->lam32 = (float)(rate_hz * s->dt / 1000.0);
    return id;
}

int bo_set_stdp(bo_sim *s, int proj, double tau_plus, double tau_minus, double lambda_,
                double alpha, double mu_plus, double mu_minus, double wmax) {
    if (proj < 0 || proj >= s->nin || s->ins[proj].kind != 0) return -1;
    input_t *in = &s->ins[proj];
    in->plastic = 1;
    in->tau_plus = tau_plus;
    in->tau_minus = tau_minus;
    in->lambda_ = lambda_;
    in->alpha = alpha;
    in->mu_plus = mu_plus;
    in->mu_minus = mu_minus;
    in->wmax = wmax;
    /* trace decay exp(-dt / tau) (event_plastic.py:405) */
    in->dec_pre = exp(-s->dt / tau_plus);
    in->dec_post = exp(-s->dt / tau_minus);
    in->pre_trace = (double *)calloc((size_t)s->pops[in->pre_pop].n, sizeof(double));
    in->post_trace = (double *)calloc((size_t)s->pops[in->post_pop].n, sizeof(double));
    return 0;
}

/* stdp_triplet_synapse (_nest_plasticity/stdp_triplet_synapse.py:160-197):
 * fast and slow traces per side (r1, r2 with tau_plus, tau_plus_triplet;
 * o1, o2 with tau_minus, tau_minus_triplet), all decay-then-add. */
int bo_set_stdp_triplet(bo_sim *s, int proj, double tau_plus, double tau_plus_triplet,
                        double tau_minus, double tau_minus_triplet, double a2p, double a3p,
                        double a2m, double a3m, double wmax) {
    if (proj < 0 || proj >= s->nin || s->ins[proj].kind != 0) return -1;
    input_t *in = &s->ins[proj];
    in->plastic = 1;
    in->rule = 1;
    in->tau_plus = tau_plus;
    in->tau_minus = tau_minus;
    in->a2p = a2p;
    in->a3p = a3p;
    in->a2m = a2m;
    in->a3m = a3m;
    in->wmax = wmax;
    in->dec_pre = exp(-s->dt / tau_plus);
    in->dec_post = exp(-s->dt / tau_minus);
    in->dec_pre2 = exp(-s->dt / tau_plus_triplet);
    in->dec_post2 = exp(-s->dt / tau_minus_triplet);
    in->pre_trace = (double *)calloc((size_t)s->pops[in->pre_pop].n, sizeof(double));
    in->post_trace = (double *)calloc((size_t)s->pops[in->post_pop].n, sizeof(double));
    in->pre_trace2 = (double *)calloc((size_t)s->pops[in->pre_pop].n, sizeof(double));
    in->post_trace2 = (double *)calloc((size_t)s->pops[in->post_pop].n, sizeof(double));
    return 0;
}

/* The triplet rule on one edge (stdp_triplet_synapse.py:179-197): every trace
 * excludes this step's own spike; potentiation on a post spike reads the fast
 * pre trace weighted by the slow post trace, then depression on a pre spike
 * reads the fast post trace weighted by the slow pre trace; w in [0, Wmax]. */
double bo_triplet_update(double w, double pre_s, double post_s, double r1_tr, double r2_tr,
                         double o1_tr, double o2_tr, double a2p, double a3p, double a2m,
                         double a3m, double wmax) {
    double r1 = r1_tr - pre_s, r2 = r2_tr - pre_s, o1 = o1_tr - post_s, o2 = o2_tr - post_s;
    if (post_s > 0.0) {
        double nw = w + r1 * (a2p + a3p * o2);
        w = nw < wmax ? nw : wmax;
    }
    if (pre_s > 0.0) {
        double nw = w - o1 * (a2m + a3m * r2);
        w = nw > 0.0 ? nw : 0.0;
    }
    return w;
}

int bo_get_weights(bo_sim *s, int proj, double *w_out) {
    if (proj < 0 || proj >= s->nin || s->ins[proj].kind != 0) return -1;
    memcpy(w_out, s->ins[proj].w, sizeof(double) * (size_t)s->ins[proj].n_edges);
    return 0;
}

int bo_record_v(bo_sim *s, int n, const int32_t *gids) {
    free(s->rec);
    s->rec = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        if (gids[i] < 0 || gids[i] >= s->ntot) return -1;
        s->rec[i] = gids[i];
    }
    s->nrec = n;
    return 0;
}

int64_t bo_step_count(bo_sim *s) { return s->step; }
int bo_n_total(bo_sim *s) { return s->ntot; }
int64_t bo_rk_substeps(bo_sim *s) { return s->rk_substeps; }

/* Threads for the per-neuron phases (input take, drives, neuron updates).
 * Delivery, recording and every sum stay serial in their fixed order, so the
 * results do not depend on the thread count. */
void bo_set_threads(bo_sim *s, int n) { s->threads = n > 0 ? n : 1; }

/* Receptor ports of the iaf models: 0 = one summed input split by sign
 * (Simulator), 1 = ports 0 / 1 apart with signs kept (kernel models). */
void bo_set_ports(bo_sim *s, int separate) { s->ports = separate ? 1 : 0; }

static void alloc_buffers(bo_sim *s) {
    if (s->hist) return;
    int maxd = 0;
    for (int i = 0; i < s->nin; ++i)
        if (s->ins[i].max_delay > maxd) maxd = s->ins[i].max_delay;
    s->H = maxd + 3;
    s->hist = (unsigned char *)calloc((size_t)s->H * (size_t)s->ntot, 1);
    s->L = maxd + 1;
    s->ring = (double *)calloc((size_t)RCH * (size_t)s->L * (size_t)s->ntot, sizeof(double));
    s->acc = (double *)calloc((size_t)RCH * (size_t)s->ntot, sizeof(double));
    s->y = (double *)calloc((size_t)2 * (size_t)s->ntot, sizeof(double));
}

static inline int fired(bo_sim *s, int64_t m, int gid) {
    if (m < 0) return 0;
    return s->hist[(size_t)(m % s->H) * (size_t)s->ntot + (size_t)gid];
}

static int64_t drive_count(const input_t *in, int64_t emit_step, int t) {
    /* active iff t_min < step <= t_max (poisson_generator.py:566-567) */
    if (!(in->tmin < emit_step && emit_step <= in->tmax) || in->rate <= 0.0) return 0;
    if (in->keyed) {
        /* the kernel path: unit = unit_off + t, block unit >> 10, lane
         * unit & 1023 (_kernel/rng.py draw_blocked, GID_BLOCK = 1024) */
        uint64_t unit = (uint64_t)in->unit_off + (uint64_t)t;
        uint32_t sk[2];
        bo_kernel_step_key_trial(in->okey, (uint32_t)(unit >> 10), (uint32_t)emit_step, in->trial, sk);
        return bo_kernel_poisson_count(sk, (uint32_t)(unit & 1023u), in->lam32);
    }
    double u = bo_uniform01(in->seed, 0u, (uint32_t)emit_step, (uint32_t)t);
    return bo_poisson(in->lam, in->enl, u);
}

/* _nest_plasticity/stdp_synapse.py:163-169 */
static double stdp_facilitate(const input_t *in, double w, double kplus) {
    double nw = w / in->wmax + in->lambda_ * pow(1.0 - w / in->wmax, in->mu_plus) * kplus;
    return nw < 1.0 ? nw * in->wmax : in->wmax;
}
static double stdp_depress(const input_t *in, double w, double kminus) {
    double nw = w / in->wmax - in->alpha * in->lambda_ * pow(w / in->wmax, in->mu_minus) * kminus;
    return nw > 0.0 ? nw * in->wmax : 0.0;
}

/* LEGACY phase 1 for one input: builds y (the projection's contribution to
 * its post population) as the reference does.
 *  - drive: y = delayed count * weight (event_proj.py:311-312, the one_to_one
 *    generator path of simulator.py:1437-1463);
 *  - static CSR: y[post] += w over edges of spiking (delayed) pres, rows in
 *    ascending pre order (projections.py:56-59);
 *  - plastic: traces decay-then-add, facilitation on post spike then
 *    depression on pre spike, delivery of the updated weight
 *    (event_plastic.py:390-518, stdp_synapse.py:171-179). */
static void legacy_input(bo_sim *s, input_t *in, int64_t n, double *y) {
    pop_t *Q = &s->pops[in->post_pop];
    for (int t = 0; t < Q->n; ++t) y[t] = 0.0;
    if (in->kind == 1) {
        int64_t emit = n - (in->ddelay + 1);
#pragma omp parallel for num_threads(s->threads > 0 ? s->threads : 1) schedule(static)
        for (int t = 0; t < Q->n; ++t) {
            int64_t c = drive_count(in, emit, t);
            y[t] = (double)c * in->weight;
        }
        return;
    }
    pop_t *P = &s->pops[in->pre_pop];
    if (!in->plastic) {
        if (in->hdelay >= 0) {
            /* one delay: test each row once (the same sums in the same order) */
            for (int i = 0; i < P->n; ++i) {
                if (!fired(s, n - (in->hdelay + 1), P->off + i)) continue;
                for (int64_t e = in->indptr[i]; e < in->indptr[i + 1]; ++e)
                    y[in->post[e]] += in->w[e];
            }
            return;
        }
        for (int i = 0; i < P->n; ++i)
            for (int64_t e = in->indptr[i]; e < in->indptr[i + 1]; ++e)
                if (fired(s, n - (in->delay[e] + 1), P->off + i)) y[in->post[e]] += in->w[e];
        return;
    }
    /* plastic: homogeneous delay of the projection's InputDelay */
    int D = in->n_edges > 0 ? in->delay[0] : 0;
    for (int i = 0; i < P->n; ++i) {
        double x = (double)fired(s, n - (D + 1), P->off + i);
        in->pre_trace[i] = in->pre_trace[i] * in->dec_pre + x;
        if (in->rule == 1) in->pre_trace2[i] = in->pre_trace2[i] * in->dec_pre2 + x;
    }
    for (int j = 0; j < Q->n; ++j) {
        double x = (double)fired(s, n - 1, Q->off + j);
        in->post_trace[j] = in->post_trace[j] * in->dec_post + x;
        if (in->rule == 1) in->post_trace2[j] = in->post_trace2[j] * in->dec_post2 + x;
    }
    for (int i = 0; i < P->n; ++i) {
        double pre_f = (double)fired(s, n - (D + 1), P->off + i);
        for (int64_t e = in->indptr[i]; e < in->indptr[i + 1]; ++e) {
            int j = in->post[e];
            double post_f = (double)fired(s, n - 1, Q->off + j);
            double w = in->w[e];
            if (in->rule == 1) {
                w = bo_triplet_update(w, pre_f, post_f, in->pre_trace[i], in->pre_trace2[i],
                                      in->post_trace[j], in->post_trace2[j], in->a2p, in->a3p,
                                      in->a2m, in->a3m, in->wmax);
            } else {
                double kplus = in->pre_trace[i] - pre_f;
                double kminus = in->post_trace[j] - post_f;
                if (post_f > 0.0) w = stdp_facilitate(in, w, kplus);
                if (pre_f > 0.0) w = stdp_depress(in, w, kminus);
            }
            in->w[e] = w;
            if (pre_f != 0.0) y[j] += w;
        }
    }
}

/* _nest_neuron/iaf_psc_alpha.py:558-684 */
/* w_ex / w_in: this step's jumps into the excitatory and inhibitory ports;
 * the summed-input form below splits one input by sign (iaf_psc_alpha.py:617-619),
 * the kernel models' ports keep them apart (_kernel/models/iaf_psc_alpha.py) */
static int step_iaf_alpha_ports(bo_sim *s, pop_t *P, int g, double w_ex, double w_in,
                                double x_next) {
    double V = s->st[0][g], Iex = s->st[1][g], dIex = s->st[2][g], Iin = s->st[3][g],
           dIin = s->st[4][g], y0 = s->st[5][g];
    int r = s->ref[g];
    double E_L = P->p[0], I_e = P->p[8], V_min = P->p[9];
    double y3 = V - E_L;
    double theta = P->p[4] - E_L;
    double v_reset = P->p[5] - E_L;
    if (r == 0) {
        double c = P->P30 * (y0 + I_e) + P->P31ex * dIex + P->P32ex * Iex + P->P31in * dIin +
                   P->P32in * Iin + P->expm1_tm * y3 + y3;
        double lower = V_min - E_L;
        if (!(c >= lower)) c = lower; /* maximum(y3, V_min - E_L); -inf => no clip */
        y3 = c;
    } else {
        r = r - 1;
    }
    double Iex_n = P->P21ex * dIex + P->P22ex * Iex;
    double dIex_n = dIex * P->P11ex;
    dIex_n = dIex_n + P->epsc * w_ex;
    double Iin_n = P->P21in * dIin + P->P22in * Iin;
    double dIin_n = dIin * P->P11in;
    dIin_n = dIin_n + P->ipsc * w_in;
    int spike = y3 >= theta;
    if (spike) {
        r = P->ref_count;
        y3 = v_reset;
    }
    s->st[0][g] = y3 + E_L;
    s->st[1][g] = Iex_n;
    s->st[2][g] = dIex_n;
    s->st[3][g] = Iin_n;
    s->st[4][g] = dIin_n;
    s->st[5][g] = x_next;
    s->ref[g] = r;
    return spike;
}

/* _nest_neuron/iaf_psc_exp.py:552-682 (deterministic threshold branch) */
static int step_iaf_exp_ports(bo_sim *s, pop_t *P, int g, double w_ex, double w_in,
                              double x_next) {
    double V = s->st[0][g], iex = s->st[1][g], iin = s->st[2][g], i0 = s->st[3][g],
           i1 = s->st[4][g];
    int r = s->ref[g];
    double E_L = P->p[0], I_e = P->p[8];
    double V_rel = V - E_L;
    double theta = P->p[4] - E_L;
    double V_reset_rel = P->p[5] - E_L;
    if (r == 0) {
        V_rel = V_rel * P->eP22 + iex * P->eP21ex + iin * P->eP21in + (I_e + i0) * P->eP20;
    } else {
        r = r - 1;
    }
    iex = iex * P->eP11ex;
    iin = iin * P->eP11in;
    iex = iex + (1.0 - P->eP11ex) * i1;
    iex = iex + w_ex;
    iin = iin + w_in;
    int spike = V_rel >= theta;
    if (spike) {
        r = P->ref_count;
        V_rel = V_reset_rel;
    }
    s->st[0][g] = V_rel + E_L;
    s->st[1][g] = iex;
    s->st[2][g] = iin;
    s->st[3][g] = x_next;
    s->st[4][g] = 0.0;
    s->ref[g] = r;
    return spike;
}

static int step_iaf_alpha(bo_sim *s, pop_t *P, int g, double w_all, double x_next) {
    return step_iaf_alpha_ports(s, P, g, w_all > 0.0 ? w_all : 0.0, w_all < 0.0 ? w_all : 0.0,
                                x_next);
}
static int step_iaf_exp(bo_sim *s, pop_t *P, int g, double w_all, double x_next) {
    return step_iaf_exp_ports(s, P, g, w_all > 0.0 ? w_all : 0.0, w_all < 0.0 ? w_all : 0.0,
                              x_next);
}

/* _nest_neuron/iaf_psc_exp_multisynapse.py:716-790: exact membrane step with
 * every receptor's current summed in receptor order, refractory countdown,
 * receptor decay plus this step's weights, threshold and reset.  Slots:
 * V_m, i_const, i_syn_0..3. */
static int step_iaf_ms(bo_sim *s, pop_t *P, int g, const double *w, double x_next) {
    double E_L = P->p[0], I_e = P->p[6];
    double V_rel = s->st[0][g] - E_L, i_const = s->st[1][g];
    double theta = P->p[4] - E_L, V_reset_rel = P->p[5] - E_L;
    int r = s->ref[g];
    if (r == 0) {
        double syn = P->msP21[0] * s->st[2][g];
        for (int k = 1; k < P->nrec; ++k) syn = syn + P->msP21[k] * s->st[2 + k][g];
        V_rel = V_rel * P->eP22 + (I_e + i_const) * P->eP20 + syn;
    } else {
        r = r - 1;
    }
    for (int k = 0; k < P->nrec; ++k) s->st[2 + k][g] = s->st[2 + k][g] * P->msP11[k] + w[k];
    int spike = V_rel >= theta;
    if (spike) {
        r = P->ref_count;
        V_rel = V_reset_rel;
    }
    s->st[0][g] = V_rel + E_L;
    s->st[1][g] = x_next;
    s->ref[g] = r;
    return spike;
}

/* ---- aeif_cond_alpha + RKF45 (_nest_neuron/aeif_cond_alpha.py:554-747,
 *      _nest_base/utils.py:266-279, :436-479, :583-718) */

static const double RK_A[6][5] = {
    {0, 0, 0, 0, 0},
    {1.0 / 4, 0, 0, 0, 0},
    {3.0 / 32, 9.0 / 32, 0, 0, 0},
    {1932.0 / 2197, -7200.0 / 2197, 7296.0 / 2197, 0, 0},
    {439.0 / 216, -8.0, 3680.0 / 513, -845.0 / 4104, 0},
    {-8.0 / 27, 2.0, -3544.0 / 2565, 1859.0 / 4104, -11.0 / 40},
};
static const double RK_B[6] = {16.0 / 135, 0.0, 6656.0 / 12825, 28561.0 / 56430, -9.0 / 50,
                               2.0 / 55};
static const double RK_BH[6] = {25.0 / 216, 0.0, 1408.0 / 2565, 2197.0 / 4104, -1.0 / 5, 0.0};

static void aeif_vf(const pop_t *P, int r, double i_stim, const double *y, double *dy) {
    double V_peak = P->p[0], V_reset = P->p[1], g_L = P->p[3], C_m = P->p[4], E_ex = P->p[5],
           E_in = P->p[6], E_L = P->p[7], Delta_T = P->p[8], tau_w = P->p[9], a = P->p[10],
           V_th = P->p[12], tex = P->p[13], tin = P->p[14], I_e = P->p[15];
    int refr = r > 0;
    double v_eff = refr ? V_reset : (y[0] < V_peak ? y[0] : (y[0] != y[0] ? y[0] : V_peak));
    double i_ex = y[2] * (v_eff - E_ex);
    double i_in = y[4] * (v_eff - E_in);
    double dts = Delta_T == 0.0 ? 1.0 : Delta_T;
    double arg = (v_eff - V_th) / dts;
    if (arg < -500.0) arg = -500.0;
    if (arg > 500.0) arg = 500.0;
    double i_spike = g_L * Delta_T * exp(arg);
    double dV = (-g_L * (v_eff - E_L) + i_spike - i_ex - i_in - y[5] + I_e + i_stim) / C_m;
    dy[0] = refr ? 0.0 : dV;
    dy[1] = -y[1] / tex;
    dy[2] = y[1] - y[2] / tex;
    dy[3] = -y[3] / tin;
    dy[4] = y[3] - y[4] / tin;
    dy[5] = (a * (v_eff - E_L) - y[5]) / tau_w;
}

static inline double nanmax(double a, double b) {
    if (a != a || b != b) return NAN;
    return a > b ? a : b;
}

/* iaf_cond_exp (_nest_neuron/iaf_cond_exp.py:456-490; y = V, g_ex, g_in) and
 * iaf_cond_alpha (_nest_neuron/iaf_cond_alpha.py:459-491; y = V, dg_ex, g_ex,
 * dg_in, g_in): the membrane sees min(V, V_th), or V_reset while refractory */
static void iaf_cond_vf(int model, const pop_t *P, int r, double i_stim, const double *y,
                        double *dy) {
    double E_L = P->p[0], C_m = P->p[1], V_th = P->p[3], V_reset = P->p[4], E_ex = P->p[5],
           E_in = P->p[6], g_L = P->p[7], tex = P->p[8], tin = P->p[9], I_e = P->p[10];
    int refr = r > 0;
    double v_eff = refr ? V_reset : (y[0] < V_th ? y[0] : (y[0] != y[0] ? y[0] : V_th));
    double gex = model == BO_IAF_COND_EXP ? y[1] : y[2];
    double gin = model == BO_IAF_COND_EXP ? y[2] : y[4];
    double i_syn_exc = gex * (v_eff - E_ex);
    double i_syn_inh = gin * (v_eff - E_in);
    double i_leak = g_L * (v_eff - E_L);
    double dV = (-i_leak - i_syn_exc - i_syn_inh + I_e + i_stim) / C_m;
    dy[0] = refr ? 0.0 : dV;
    if (model == BO_IAF_COND_EXP) {
        dy[1] = -y[1] / tex;
        dy[2] = -y[2] / tin;
    } else {
        dy[1] = -y[1] / tex;
        dy[2] = y[1] - y[2] / tex;
        dy[3] = -y[3] / tin;
        dy[4] = y[3] - y[4] / tin;
    }
}

/* One dt of a conductance model: the adaptive RKF45 loop with the model's
 * in-loop event (aeif_cond_alpha.py:594-625, iaf_cond_exp.py:487-517,
 * iaf_cond_alpha.py:493-521), then the refractory countdown and the
 * synaptic jumps (aeif_cond_alpha.py:709-728, iaf_cond_exp.py:594-614,
 * iaf_cond_alpha.py:602-624). */
static int step_cond(bo_sim *s, pop_t *P, int g, double w_ex, double w_in, double x_next,
                     int *unstable) {
    const int model = s->model, ns = n_ode(model);
    const int aeif = model == BO_AEIF_COND_ALPHA;
    const double dt = s->dt, min_h = 1e-8, atol = aeif ? P->p[16] : P->p[11];
    const int max_iters = model == BO_IAF_COND_EXP ? 10000 : 100000; /* _MAX_ITERS */
    double y[6];
    for (int i = 0; i < ns; ++i) y[i] = s->st[i][g];
    double h = s->st[ns][g], i_stim = s->st[ns + 1][g];
    int r = s->ref[g];
    double V_reset = aeif ? P->p[1] : P->p[4], b = aeif ? P->p[11] : 0.0;
    double v_peak_detect = aeif ? (P->p[8] > 0.0 ? P->p[0] : P->p[12]) : P->p[3];
    int spiked = 0;
    double t_loc = 0.0;
    if (h < min_h) h = min_h;
    int iters = 0;
    double k[6][6];
    while (t_loc < dt && iters < max_iters) {
        double hh = h < dt - t_loc ? h : dt - t_loc;
        h = hh > min_h ? hh : min_h;
        for (int st = 0; st < 6; ++st) {
            double yi[6];
            if (st == 0) {
                for (int i = 0; i < ns; ++i) yi[i] = y[i];
            } else {
                for (int i = 0; i < ns; ++i) {
                    double acc = 0.0;
                    int first = 1;
                    for (int j = 0; j < st; ++j) {
                        if (RK_A[st][j] == 0.0) continue;
                        double term = RK_A[st][j] * k[j][i];
                        acc = first ? term : acc + term;
                        first = 0;
                    }
                    yi[i] = y[i] + h * acc;
                }
            }
            if (aeif) aeif_vf(P, r, i_stim, yi, k[st]);
            else iaf_cond_vf(model, P, r, i_stim, yi, k[st]);
        }
        double yh[6], ye[6], err = 0.0;
        for (int i = 0; i < ns; ++i) {
            double acc = 0.0, eacc = 0.0;
            int first = 1, efirst = 1;
            for (int j = 0; j < 6; ++j) {
                if (RK_B[j] != 0.0) {
                    double term = RK_B[j] * k[j][i];
                    acc = first ? term : acc + term;
                    first = 0;
                }
                double be = RK_B[j] - RK_BH[j];
                if (be != 0.0) {
                    double term = be * k[j][i];
                    eacc = efirst ? term : eacc + term;
                    efirst = 0;
                }
            }
            yh[i] = y[i] + h * acc;
            ye[i] = h * eacc;
            double ay = fabs(y[i]) > fabs(yh[i]) ? fabs(y[i]) : fabs(yh[i]);
            double e = fabs(ye[i]) / (atol + 0.0 * ay);
            err = i == 0 ? e : nanmax(err, e);
        }
        if (err != err) err = INFINITY;
        int accept = (err <= 1.0) || (h <= min_h);
        if (accept) {
            for (int i = 0; i < ns; ++i) y[i] = yh[i];
            t_loc = t_loc + h;
            /* _event_fn: instability guard on the pre-reset state (AdEx:
             * V and w; iaf_cond_exp: V; iaf_cond_alpha: none) */
            if (aeif && (y[0] < -1e3 || y[5] < -1e6 || y[5] > 1e6)) *unstable = 1;
            if (model == BO_IAF_COND_EXP && y[0] < -1e3) *unstable = 1;
            if (r > 0) y[0] = V_reset;
            if (r <= 0 && y[0] >= v_peak_detect) {
                spiked = 1;
                y[0] = V_reset;
                if (aeif) y[5] = y[5] + b;
                if (P->ref_count > 0) r = P->ref_count + 1;
            }
        }
        double err_sg = err > 1e-30 ? err : 1e-30;
        double inv_err = 1.0 / err_sg;
        if (accept) {
            double fac = err_sg <= 1e-30 ? 5.0 : 0.9 * pow(inv_err, 1.0 / 5.0);
            if (!(err_sg <= 1e-30)) fac = fac < 0.2 ? 0.2 : (fac > 5.0 ? 5.0 : fac);
            double hn = h * fac;
            h = hn > min_h ? hn : min_h;
        } else {
            double fac = 0.9 * pow(inv_err, 1.0 / 4.0);
            fac = fac < 0.2 ? 0.2 : (fac > 1.0 ? 1.0 : fac);
            double hn = h * fac;
            h = hn > min_h ? hn : min_h;
        }
        iters++;
    }
#pragma omp atomic
    s->rk_substeps += iters;
    if (r > 0) r = r - 1;
    /* synaptic jumps after integration: g += w (iaf_cond_exp), dg += e / tau * w
     * (alpha kernels) */
    if (model == BO_IAF_COND_EXP) {
        y[1] = y[1] + w_ex;
        y[2] = y[2] + w_in;
    } else {
        double tex = aeif ? P->p[13] : P->p[8], tin = aeif ? P->p[14] : P->p[9];
        y[1] = y[1] + (2.718281828459045 / tex) * w_ex;
        y[3] = y[3] + (2.718281828459045 / tin) * w_in;
    }
    for (int i = 0; i < ns; ++i) s->st[i][g] = y[i];
    s->st[ns][g] = h;
    s->st[ns + 1][g] = x_next;
    s->ref[g] = r;
    return spiked;
}


/* One model update of neuron gid with explicit inputs (golden tests):
 * w0 = summed delta input (current models) or the excitatory conductance
 * jump (aeif), w1 = inhibitory conductance jump (aeif only), x_next =
 * current input buffered for the next step. */
int bo_step_neuron_ms(bo_sim *s, int gid, const double *w, double x_next) {
    if (gid < 0 || gid >= s->ntot || s->model != BO_IAF_PSC_EXP_MULTISYNAPSE) return -1;
    int p = 0;
    while (p + 1 < s->npop && s->pops[p + 1].off <= gid) ++p;
    return step_iaf_ms(s, &s->pops[p], gid, w, x_next);
}

int bo_step_neuron(bo_sim *s, int gid, double w0, double w1, double x_next) {
    if (gid < 0 || gid >= s->ntot) return -1;
    int p = 0;
    while (p + 1 < s->npop && s->pops[p + 1].off <= gid) ++p;
    pop_t *P = &s->pops[p];
    int unstable = 0;
    if (s->model == BO_IAF_PSC_ALPHA) return step_iaf_alpha(s, P, gid, w0, x_next);
    if (s->model == BO_IAF_PSC_EXP) return step_iaf_exp(s, P, gid, w0, x_next);
    int sp = step_cond(s, P, gid, w0, w1, x_next, &unstable);
    return unstable ? -2 : sp;
}

int64_t bo_run(bo_sim *s, int64_t n_steps, int64_t *spk_step, int32_t *spk_gid,
               int64_t cap, double *v_out) {
    alloc_buffers(s);
    int N = s->ntot;
    int64_t nspk = 0;
    int unstable = 0;
    for (int64_t it = 0; it < n_steps; ++it) {
        int64_t n = s->step;
        double *acc0 = s->acc, *acc1 = s->acc + N;
        if (s->sem == BO_LEGACY) {
            /* phase 1: every input's contribution, summed in creation order
             * (simulator.py:1728-1731, _base.py:312-382), per receptor port */
            for (size_t q = 0; q < (size_t)RCH * (size_t)N; ++q) s->acc[q] = 0.0;
            for (int i = 0; i < s->nin; ++i) {
                input_t *in = &s->ins[i];
                pop_t *Q = &s->pops[in->post_pop];
                legacy_input(s, in, n, s->y);
                double *acc = s->acc + (size_t)in->receptor * (size_t)N;
                for (int t = 0; t < Q->n; ++t) acc[Q->off + t] = acc[Q->off + t] + s->y[t];
            }
        } else {
            /* PostRing.take: read slot n mod L and clear it (delays.py:291-306) */
            size_t slot = (size_t)(n % s->L);
            for (int c = 0; c < RCH; ++c) {
                double *rc = s->ring + ((size_t)c * (size_t)s->L + slot) * (size_t)N;
                double *ac = s->acc + (size_t)c * (size_t)N;
                for (int g = 0; g < N; ++g) {
                    ac[g] = rc[g];
                    rc[g] = 0.0;
                }
            }
        }
        /* phase 2: neurons (NEST order inside each model), independent per
         * neuron; the spike list is then collected in gid order */
        unsigned char *hrow = s->hist + (size_t)(n % s->H) * (size_t)N;
        for (int p = 0; p < s->npop; ++p) {
            pop_t *P = &s->pops[p];
            int uns = 0;
#pragma omp parallel for num_threads(s->threads > 0 ? s->threads : 1) schedule(static) reduction(| : uns)
            for (int k = 0; k < P->n; ++k) {
                int g = P->off + k, sp;
                if (s->model == BO_IAF_PSC_ALPHA && s->ports)
                    sp = step_iaf_alpha_ports(s, P, g, acc0[g], acc1[g], 0.0);
                else if (s->model == BO_IAF_PSC_EXP && s->ports)
                    sp = step_iaf_exp_ports(s, P, g, acc0[g], acc1[g], 0.0);
                else if (s->model == BO_IAF_PSC_ALPHA) sp = step_iaf_alpha(s, P, g, acc0[g], 0.0);
                else if (s->model == BO_IAF_PSC_EXP) sp = step_iaf_exp(s, P, g, acc0[g], 0.0);
                else if (s->model == BO_IAF_PSC_EXP_MULTISYNAPSE) {
                    double w[RCH];
                    for (int c = 0; c < RCH; ++c) w[c] = s->acc[(size_t)c * (size_t)N + (size_t)g];
                    sp = step_iaf_ms(s, P, g, w, 0.0);
                } else sp = step_cond(s, P, g, acc0[g], acc1[g], 0.0, &uns);
                hrow[g] = (unsigned char)sp;
            }
            unstable |= uns;
            for (int k = 0; k < P->n; ++k) {
                int g = P->off + k;
                if (hrow[g]) {
                    if (nspk < cap) {
                        spk_step[nspk] = n;
                        spk_gid[nspk] = g;
                    }
                    nspk++;
                }
            }
        }
        if (s->sem == BO_RING) {
            /* deposit: event of step n over delay d -> slot (n + d) mod L
             * (delay_scatter.py:243-282, runner.py:659-672) */
            for (int i = 0; i < s->nin; ++i) {
                input_t *in = &s->ins[i];
                pop_t *Q = &s->pops[in->post_pop];
                double *rb = s->ring + (size_t)in->receptor * (size_t)s->L * (size_t)N;
                if (in->kind == 1) {
                    size_t slot = (size_t)((n + in->ddelay) % s->L);
#pragma omp parallel for num_threads(s->threads > 0 ? s->threads : 1) schedule(static)
                    for (int t = 0; t < Q->n; ++t) {
                        int64_t c = drive_count(in, n, t);
                        if (c) rb[slot * (size_t)N + (size_t)(Q->off + t)] += (double)c * in->weight;
                    }
                    continue;
                }
                pop_t *P = &s->pops[in->pre_pop];
                for (int pi = 0; pi < P->n; ++pi) {
                    if (!hrow[P->off + pi]) continue;
                    for (int64_t e = in->indptr[pi]; e < in->indptr[pi + 1]; ++e) {
                        size_t slot = (size_t)((n + in->delay[e]) % s->L);
                        rb[slot * (size_t)N + (size_t)(Q->off + in->post[e])] += in->w[e];
                    }
                }
            }
        }
        if (v_out)
            for (int r = 0; r < s->nrec; ++r) v_out[it * s->nrec + r] = s->st[0][s->rec[r]];
        s->step++;
    }
    if (unstable) return -2;
    return nspk;
}
