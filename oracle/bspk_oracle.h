/*
 * bspk_oracle.h -- float64 CPU oracle for the spiking-network step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a single-threaded, float64 restatement
 * of the reference (brainspike, formerly chaobrain/brainpy.state) network
 * step, used as the checker of the CUDA library.  Only tests/, the smoke
 * check of __graft_entry__ and the cpu_baseline / reference arms of bench.py
 * may load it.  The product library never links or calls it.
 *
 * Pinning: the neuron updates, propagators, ring semantics and STDP rule are
 * checked against the golden vectors of the reference's own tests
 * (tests/test_oracle_golden.py); the Threefry-2x32 block cipher against the
 * Random123 known-answer vectors.  The JAX key-derivation layer above the
 * cipher (fold_in / split / randint) and the Poisson stream are NOT pinned:
 * JAX cannot run in this build environment (see the module docstring of
 * oracle/oracle.py).
 */
#ifndef BSPK_ORACLE_H
#define BSPK_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* neuron models (same ids as the product library) */
enum {
    BO_IAF_PSC_ALPHA = 0,
    BO_IAF_PSC_EXP = 1,
    BO_AEIF_COND_ALPHA = 2,
    BO_IAF_COND_EXP = 3,
    BO_IAF_COND_ALPHA = 4,
    BO_IAF_PSC_EXP_MULTISYNAPSE = 5
};

/* delivery semantics
 *  LEGACY: reference Simulator -- a spike of step m reaches the update of
 *          step m + D + 1 (holder lag + InputDelay), each projection's
 *          contributions are summed as one vector, projections are added in
 *          creation order (_nest_network/simulator.py:1719-1788,
 *          _nest_network/delay.py:114-128, _base.py:312-382).
 *  RING:   kernel DelayScatter/PostRing -- an event of step n over delay d is
 *          added to arrival slot (n + d) mod L, slot n is read and cleared at
 *          the start of step n (_kernel/delay_scatter.py:1-25,
 *          _kernel/delays.py:260-319).
 */
enum { BO_LEGACY = 0, BO_RING = 1 };

typedef struct bo_sim bo_sim;

/* Threefry-2x32, 20 rounds (Salmon et al., SC'11). */
void bo_threefry2x32(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1,
                     uint32_t *y0, uint32_t *y1);
/* JAX-style key derivation (threefry, partitionable layout). */
void bo_jax_key(int64_t seed, uint32_t key[2]);
void bo_jax_fold_in(const uint32_t key[2], uint32_t data, uint32_t out[2]);
void bo_jax_split(const uint32_t key[2], int num, uint32_t *out /* num*2 */);
void bo_jax_random_bits(const uint32_t key[2], int nbits, int64_t n, uint64_t *out);
void bo_jax_randint(const uint32_t key[2], int64_t n, int64_t minval, int64_t maxval,
                    int nbits, int64_t *out);
void bo_jax_random_bits_at(const uint32_t key[2], int nbits, int64_t i, uint64_t *out);
/* jax.random.uniform / normal (float32 for nbits 32, float64 for 64) */
void bo_jax_uniform(const uint32_t key[2], int nbits, int64_t n, double lo, double hi,
                    double *out);
void bo_jax_normal(const uint32_t key[2], int nbits, int64_t n, double *out);
/* kernel-path poisson_generator: step key of a block, count of one unit */
void bo_kernel_step_key(const uint32_t obj[2], uint32_t block, uint32_t step, uint32_t out[2]);
void bo_kernel_step_key_trial(const uint32_t obj[2], uint32_t block, uint32_t step, uint32_t trial,
                              uint32_t out[2]);
/* trial index folded into every keyed drive's step keys (default 0) */
void bo_set_trial(bo_sim *s, uint32_t trial);
int64_t bo_kernel_poisson_count(const uint32_t step_key[2], uint32_t lane, float lam);
/* legacy fixed-indegree sampler (connectivity.py:101-135): post-major edges */
int bo_fixed_indegree(int64_t seed, int n_pre, int n_post, int K, int pre_is_post,
                      int allow_autapses, int nbits, int32_t *pre_out, int32_t *post_out);
/* CSR by stable argsort on pre (connectivity.py:39-53) */
int bo_csr_structure(const int32_t *pre, const int32_t *post, int64_t n_edges, int n_pre,
                     int64_t *order_out, int32_t *indices_out, int64_t *indptr_out);

/* product Poisson stream (restated): uniform + inversion */
double bo_uniform01(uint32_t seed, uint32_t stream, uint32_t step, uint32_t idx);
int bo_poisson(double lam, double exp_neg_lam, double u);

/* propagators (_nest_base/utils.py:126-229) */
void bo_alpha_p31_p32(double tau_syn, double tau_m, double c_m, double h,
                      double *p31, double *p32);
double bo_propagator_exp(double tau_syn, double tau_m, double c_m, double h);

/* simulator */
bo_sim *bo_create(double dt, int semantics, int model);
void bo_destroy(bo_sim *s);
int bo_add_pop(bo_sim *s, int n, const double *params, int n_params);
int bo_set_state(bo_sim *s, int pop, const char *name, const double *values);
int bo_get_state(bo_sim *s, int pop, const char *name, double *values);
int bo_add_proj(bo_sim *s, int pre_pop, int post_pop, int64_t n_edges,
                const int64_t *indptr, const int32_t *post_local, const double *w,
                const int32_t *delay_steps, int receptor);
int bo_add_drive(bo_sim *s, int post_pop, double rate_hz, double weight, int delay_steps,
                 uint32_t seed, int64_t t_min_step, int64_t t_max_step, int receptor);
/* drive on the kernel path's stream of the device population with object
 * key okey; unit unit_off + t drives neuron t of post_pop */
int bo_add_drive_keyed(bo_sim *s, int post_pop, double rate_hz, double weight, int delay_steps,
                       const uint32_t okey[2], int64_t unit_off, int64_t t_min_step,
                       int64_t t_max_step, int receptor);
int bo_set_stdp(bo_sim *s, int proj, double tau_plus, double tau_minus, double lambda_,
                double alpha, double mu_plus, double mu_minus, double wmax);
int bo_set_stdp_triplet(bo_sim *s, int proj, double tau_plus, double tau_plus_triplet,
                        double tau_minus, double tau_minus_triplet, double a2p, double a3p,
                        double a2m, double a3m, double wmax);
double bo_triplet_update(double w, double pre_s, double post_s, double r1_tr, double r2_tr,
                         double o1_tr, double o2_tr, double a2p, double a3p, double a2m,
                         double a3m, double wmax);
int bo_get_weights(bo_sim *s, int proj, double *w_out);
int bo_record_v(bo_sim *s, int n, const int32_t *gids);
/* run n_steps; spikes appended as (step, gid) pairs up to cap; returns the
 * number of spikes written (negative = error).  v_out: [n_steps][n_rec]. */
int64_t bo_run(bo_sim *s, int64_t n_steps, int64_t *spk_step, int32_t *spk_gid,
               int64_t cap, double *v_out);
int bo_step_neuron(bo_sim *s, int gid, double w0, double w1, double x_next);
/* One iaf_psc_exp_multisynapse update of gid with one weight per receptor
 * (w[0..3], pA) and the current buffered for the next step. */
int bo_step_neuron_ms(bo_sim *s, int gid, const double *w, double x_next);
int64_t bo_step_count(bo_sim *s);
int bo_n_total(bo_sim *s);
int64_t bo_rk_substeps(bo_sim *s);
void bo_set_threads(bo_sim *s, int n);
void bo_set_ports(bo_sim *s, int separate);

/* Surrogate-gradient BPTT through a recurrent iaf_psc_exp network
 * (bspk_oracle_bptt.c).  W is given row-major over post neurons:
 * row_ptr[n+1], col[nnz] = pre, w[nnz]; w_in is [n][n_in]; inputs are
 * counts [n_steps][batch][n_in]; targets [n_steps][batch][n_readout].
 * dw / dw_in may be NULL (forward only). */
typedef struct {
    double dt;
    int n, n_in, batch, n_steps, n_readout;
    double readout_tau, slope;
    int relaxed, detach_reset;
    double params[9]; /* E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in I_e */
} bo_bptt_cfg;
int bo_lif_bptt(const bo_bptt_cfg *c, const int64_t *row_ptr, const int32_t *col, int64_t nnz,
                const double *w, const double *w_in, const uint8_t *inputs, const double *targets,
                double *loss, double *dw, double *dw_in, int64_t *n_spikes);

#ifdef __cplusplus
}
#endif
#endif
