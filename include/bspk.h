/*
 * bspk.h -- C ABI of libbspk.so, the B200 (sm_100a) network-step library.
 *
 * The reference (brainspike, formerly chaobrain/brainpy.state) has no native
 * ABI: its hot path is Python/JAX with brainevent operators.  Each entry
 * point below replaces one reference interface, cited as
 * <file>:<line> relative to the brainspike project root.
 *
 * Conventions
 *  - Every function returns an int status (BSPK_OK = 0, negative = error);
 *    bspk_last_error() returns a thread-local message for the last failure.
 *  - Host pointers passed in are borrowed for the duration of the call.
 *  - The plan owns all device buffers.  `stream` is a cudaStream_t passed as
 *    void* (NULL = the legacy default stream).  One plan is driven from one
 *    stream at a time; calls on one plan are not re-entrant.
 *  - Units are NEST's: ms, mV, pA, pF, nS, Hz.
 */
#ifndef BSPK_H
#define BSPK_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    BSPK_OK = 0,
    BSPK_ERR_ARG = -1,       /* bad argument (ValueError in the reference) */
    BSPK_ERR_STATE = -2,     /* call out of order (e.g. add after upload) */
    BSPK_ERR_CUDA = -3,      /* CUDA runtime failure */
    BSPK_ERR_UNSUPPORTED = -4,
    BSPK_ERR_TIMEOUT = -5,   /* a bounded device wait ran out */
    BSPK_ERR_UNSTABLE = -6,  /* aeif_cond_alpha / iaf_cond_exp instability guard */
    BSPK_ERR_OVERFLOW = -7,  /* a device buffer (spike record) overflowed */
    BSPK_ERR_RKCAP = -8      /* RKF45 iteration cap reached */
};

/* neuron models: iaf_psc_alpha (_nest_neuron/iaf_psc_alpha.py:558),
 * iaf_psc_exp (_nest_neuron/iaf_psc_exp.py:552), aeif_cond_alpha
 * (_nest_neuron/aeif_cond_alpha.py:627), iaf_cond_exp
 * (_nest_neuron/iaf_cond_exp.py:519), iaf_cond_alpha
 * (_nest_neuron/iaf_cond_alpha.py:523), iaf_psc_exp_multisynapse
 * (_nest_neuron/iaf_psc_exp_multisynapse.py:651).  Models 2-4 are conductance
 * models integrated by adaptive RKF45 with receptor ports 0 (g_ex) and
 * 1 (g_in); model 5 has up to 4 current receptors (ports 0..n-1), each with
 * its own exponential synaptic time constant. */
enum {
    BSPK_IAF_PSC_ALPHA = 0,
    BSPK_IAF_PSC_EXP = 1,
    BSPK_AEIF_COND_ALPHA = 2,
    BSPK_IAF_COND_EXP = 3,
    BSPK_IAF_COND_ALPHA = 4,
    BSPK_IAF_PSC_EXP_MULTISYNAPSE = 5
};

/* delivery semantics:
 *  LEGACY: Simulator timing, a spike of step m reaches step m + D + 1
 *          (_nest_network/simulator.py:1719-1788, delay.py:114-128);
 *  RING:   kernel/NEST timing, an event of step n over delay d arrives at
 *          step n + d (_kernel/delay_scatter.py:1-25, _kernel/delays.py:260). */
enum { BSPK_LEGACY = 0, BSPK_RING = 1 };

typedef struct bspk_plan bspk_plan;

typedef struct {
    double dt;              /* ms */
    int precision;          /* 32 or 64: state, ring and weight arithmetic */
    int semantics;          /* BSPK_LEGACY or BSPK_RING */
    int deterministic;      /* 1: FP64 pull delivery, bit-reproducible order */
    int model;              /* one neuron model per plan */
    int device;             /* CUDA device ordinal */
    int64_t spike_capacity; /* recorded spike events kept on the device */
} bspk_config;

typedef struct {
    double tau_plus, tau_minus, lambda_, alpha, mu_plus, mu_minus, Wmax;
} bspk_stdp_params;

/* stdp_triplet_synapse parameters (_nest_plasticity/stdp_triplet_synapse.py:
 * 126-141): fast/slow trace constants per side and the pair (A2) and
 * triplet (A3) amplitudes; weights stay in [0, Wmax]. */
typedef struct {
    double tau_plus, tau_plus_triplet, tau_minus, tau_minus_triplet;
    double Aplus, Aplus_triplet, Aminus, Aminus_triplet, Wmax;
} bspk_stdp_triplet_params;

/* Library version string and build arch. */
const char *bspk_version(void);
const char *bspk_last_error(void);

/* Plan lifecycle.  Replaces Simulator(dt) + brainstate.environ precision
 * (_nest_network/simulator.py:417-456). */
int bspk_plan_create(const bspk_config *cfg, bspk_plan **out);
int bspk_plan_destroy(bspk_plan *plan);

/* Population of `n` neurons with per-population NEST parameters in the
 * model's fixed order (iaf_psc_alpha: E_L C_m tau_m t_ref V_th
 * V_reset tau_syn_ex tau_syn_in I_e V_min; iaf_psc_exp the same without V_min;
 * aeif_cond_alpha V_peak V_reset t_ref g_L C_m E_ex E_in E_L Delta_T tau_w a b
 * V_th tau_syn_ex tau_syn_in I_e gsl_error_tol; iaf_cond_exp and
 * iaf_cond_alpha E_L C_m t_ref V_th V_reset E_ex E_in g_L tau_syn_ex
 * tau_syn_in I_e gsl_error_tol; iaf_psc_exp_multisynapse E_L C_m tau_m t_ref
 * V_th V_reset I_e n_receptors tau_syn[0..n_receptors-1], n_receptors <= 4).
 * Propagators are computed
 * here in float64.  Replaces Simulator.create (simulator.py:458) and the
 * models' _precompute_propagators (iaf_psc_alpha.py:451-479,
 * iaf_psc_exp.py:492-512). */
int bspk_pop_add(bspk_plan *plan, int n, const double *params, int n_params, int *pop_id);

/* Static CSR projection (rows = pre neurons of pre_pop, local indices):
 * indptr[n_pre+1], post_local[E], w[E] (pA or nS), delay_steps[E] (the
 * reference's delay in steps; LEGACY adds the holder lag), receptor 0/1
 * (conductance models: 0 = g_ex, 1 = g_in).  Replaces the brainevent
 * CSR + BinaryArray event matmul (_nest_network/projections.py:36-59,
 * event_proj.py:293-325) and DelayScatter (_kernel/delay_scatter.py:109). */
int bspk_proj_add_csr(bspk_plan *plan, int pre_pop, int post_pop, int64_t n_edges,
                      const int64_t *indptr, const int32_t *post_local, const double *w,
                      const int32_t *delay_steps, int receptor, int *proj_id);

/* fixed_indegree projection sampled inside the library with the reference's
 * key derivation (jax.random.key(seed) -> split(3)[0] -> fold_in(post) ->
 * randint with nbits-wide bits), then CSR by stable pre sort.  Replaces
 * sample_fixed_indegree + csr_structure (_nest_network/connectivity.py:39-53,
 * :101-135).  `delay_steps` may be NULL (then `delay_const` for all edges). */
int bspk_proj_add_fixed_indegree(bspk_plan *plan, int pre_pop, int post_pop, int K,
                                 int64_t seed, int allow_autapses, int nbits, double weight,
                                 const int32_t *delay_steps, int delay_const, int receptor,
                                 int *proj_id);

/* The same with per-edge weights w_draw[n_post * K] in the sampler's edge
 * order (post-major, draw order, before the CSR sort) -- the order in which
 * the reference draws distributed weights from the projection's k_w key
 * (_nest_network/event_proj.py:148-149, 286-291); NULL means `weight` for
 * every edge.  delay_steps, when given, is in the same order. */
int bspk_proj_add_fixed_indegree_w(bspk_plan *plan, int pre_pop, int post_pop, int K,
                                   int64_t seed, int allow_autapses, int nbits, double weight,
                                   const double *w_draw, const int32_t *delay_steps,
                                   int delay_const, int receptor, int *proj_id);

/* Poisson drive, one independent train per target neuron of post_pop (the
 * Simulator realises a generator per target, simulator.py:1437-1463):
 * count ~ Poisson(rate*dt/1000) per step, active iff t_min < step <= t_max
 * (poisson_generator.py:501-579), delivered with weight after delay_steps. */
int bspk_drive_add_poisson(bspk_plan *plan, int post_pop, double rate_hz, double weight,
                           int delay_steps, uint32_t seed, int64_t t_min_step,
                           int64_t t_max_step, int receptor, int *drive_id);

/* Poisson drive on the reference kernel path's stream: the poisson_generator
 * device population with object key obj_key = fold(fold(PRNGKey(seed),
 * hi), lo) of its name id (_kernel/rng.py:153-176), whose unit
 * unit_off + i drives neuron i of post_pop one_to_one.  Per emission step n
 * the units of block b draw jax.random.uniform(fold(fold(fold(obj, b), n), t),
 * (1024,), float32) with t the plan's trial (0 unless bspk_plan_set_trial)
 * (block keys, _kernel/rng.py:338-420) and the count is
 * the CDF inversion of _kernel/models/devices.py:46-67 in float32, active iff
 * t_min < n <= t_max; the counts arrive delay_steps later with weight.
 * Replaces poisson_counts (_kernel/models/devices.py:70-145); rate*dt/1000
 * must be below 10 (the reference switches to jax.random.poisson there,
 * which is not restated: BSPK_ERR_UNSUPPORTED). */
int bspk_drive_add_poisson_keyed(bspk_plan *plan, int post_pop, double rate_hz, double weight,
                                 int delay_steps, const uint32_t *obj_key, int64_t unit_off,
                                 int64_t t_min_step, int64_t t_max_step, int receptor,
                                 int *drive_id);
/* The trial index every keyed drive of the plan folds into its step keys in
 * place of 0: fold(fold(fold(obj, b), n), trial) -- trial b of the kernel
 * path's batched runs (Runner(batch=B), 'independent': trial b; 'common' and
 * unbatched runs: 0), _kernel/rng.py:335-356 and _kernel/runner.py:84-113.
 * Set before upload (BSPK_ERR_STATE after). */
int bspk_plan_set_trial(bspk_plan *plan, uint32_t trial);

/* The reference's random draws on the host (JAX's threefry PRNG,
 * partitionable layout): fold_in (jax.random.fold_in), uniform
 * (jax.random.uniform(key, (n,), float32 if bits == 32 else float64, lo,
 * hi), results widened to double) and normal (jax.random.normal, the same
 * dtypes).  The front ends draw the reference's per-edge delays, distributed
 * weights and initial states with them (_kernel/params.py:183-330,
 * _kernel/compiler.py:819-850, _dist.py:40-77).  uniform and fold_in are
 * bit-exact restatements; normal evaluates erfinv as XLA does for float32
 * (M. Giles' polynomial on -log1p(-x^2)) and to within an ulp or two for
 * float64, so its last bits can differ from XLA's where log1p or erfinv
 * round differently. */
int bspk_jax_fold_in(const uint32_t *key, uint32_t data, uint32_t *out);
int bspk_jax_uniform(const uint32_t *key, int64_t n, int bits, double lo, double hi,
                     double *out);
int bspk_jax_normal(const uint32_t *key, int64_t n, int bits, double *out);
/* The kernel-path Poisson table of bspk_drive_add_poisson_keyed for one
 * rate: up to cap integer thresholds t_k = ceil(F_k * 2^23) - 1 of the
 * float32 CDF, *n_out = the table's length (tests and tools). */
int bspk_kernel_poisson_table(double rate_hz, double dt_ms, int cap, uint64_t *thresholds,
                              int *n_out);

/* Copy a projection's CSR (host copy: indptr[n_pre+1], post_local[E],
 * delay_steps[E], w[E] as given or as sampled).  Replaces the structure
 * arrays read back from a brainevent CSR (_nest_network/projections.py:51-54). */
int bspk_proj_csr_get(bspk_plan *plan, int proj_id, int64_t *indptr, int32_t *post_local,
                      int32_t *delay_steps, double *w);

/* Per-edge weights of a projection, in its CSR order (bspk_proj_csr_get),
 * before upload: distributed weights on connectivity drawn by the library
 * (the reference's connect(weight=<Distribution>), connectivity.py:385-405). */
int bspk_proj_set_weights(bspk_plan *plan, int proj_id, int64_t n_edges, const double *w);

/* Make a CSR projection plastic with the pair STDP rule of
 * _nest_plasticity/stdp_synapse.py:163-179 driven by the eager substrate of
 * _nest_network/event_plastic.py:390-518 (weights kept in FP64). */
int bspk_stdp_attach(bspk_plan *plan, int proj_id, const bspk_stdp_params *p);

/* Make a CSR projection plastic with the triplet rule of
 * _nest_plasticity/stdp_triplet_synapse.py:179-197 (two traces per side) on
 * the same eager substrate and FP64 weights as bspk_stdp_attach.
 * stdp_synapse_hom (_nest_plasticity/stdp_synapse_hom.py) is the pair rule
 * of bspk_stdp_attach under another name. */
int bspk_stdp_triplet_attach(bspk_plan *plan, int proj_id, const bspk_stdp_triplet_params *p);

/* fixed_indegree with multapses as the kernel front end draws it
 * (_kernel/connectivity/rules.py:226-265, keys of _kernel/rng.py:106-300):
 * for post neuron j of part q of the post view (population name id
 * (part_hi[q], part_lo[q]), local id l = post_local[j]),
 *   key_j = fold(fold(fold(fold(fold(obj, hi_q), lo_q), l / 1024), 2^32 - 1), l % 1024),
 *   obj   = fold(fold(PRNGKey(seed), proj_hi), proj_lo)  (the projection name's id),
 * and its K sources are randint(key_j, (K,), 0, n_pre - has_self) with 32-bit
 * draws, shifted past self_pos[j] (its own position in the pre view, -1 or
 * NULL for none, which excludes autapses).  src_pos[j * K + k] are positions
 * in the pre view.  Host code, no GPU. */
int bspk_kernel_fixed_indegree(uint32_t seed, uint32_t proj_hi, uint32_t proj_lo, int n_parts,
                               const uint32_t *part_hi, const uint32_t *part_lo,
                               const int64_t *part_len, const int64_t *post_local,
                               const int64_t *self_pos, int64_t n_pre, int K, int32_t *src_pos);

/* Receptor ports of the iaf_psc models.  0 (default): every input is summed
 * and the sum split by sign into the excitatory and inhibitory currents, as
 * the Simulator does (_base.py:312-382, iaf_psc_alpha.py:617-619).
 * 1: port 0 ('ex') and port 1 ('in_') stay apart and keep their weights'
 * signs, as the kernel models' receptor ports do
 * (_kernel/models/iaf_psc_alpha.py, iaf_psc_exp.py inputs); such plans run on
 * the per-step engine.  Call before adding projections or drives. */
int bspk_plan_set_ports(bspk_plan *plan, int separate);

/* Test hook for failure detection (no counterpart in the reference): in the
 * next bspk_run of a plan on the tiled path, CTA `cta` does not publish the
 * header of its spike record of window `window` (windows of the run's first
 * launch, from 0).  No other CTA can then complete that window: each one's
 * bounded wait gives up after 2 s, the kernel returns, and the first
 * synchronising call after the run (bspk_spikes_get, bspk_v_get, ...)
 * returns BSPK_ERR_TIMEOUT.  The CUDA context stays usable; the plan's state after
 * such a run is not meaningful.  The hook applies to one run only. */
int bspk_debug_withhold_record(bspk_plan *plan, int cta, int window);

/* Recording taps (simulator.py:645-662, :1858-1870): V_m of the listed
 * neurons every step; spikes of all neurons (or of the flagged ones). */
int bspk_record_v(bspk_plan *plan, int n, const int32_t *gids);
int bspk_record_spikes_of(bspk_plan *plan, int n, const int32_t *gids);

/* Upload structure and state to the device (after all adds). */
int bspk_plan_upload(bspk_plan *plan, void *stream);

/* Advance n_steps (Simulator.simulate/cont, simulator.py:1790-1883; kernel
 * Program.rollout, _kernel/runner.py:689-779).  Asynchronous on `stream`. */
int bspk_run(bspk_plan *plan, int64_t n_steps, void *stream);
/* One step of the network (the single-step target a jax.ffi program calls
 * inside its own loop; bspk_run(plan, 1, stream)). */
int bspk_step_fused(bspk_plan *plan, void *stream);
/* Options of the tiled path (none changes a result):
 *  record_copies (1..16, default 1): each CTA's per-window spike record is
 *    written that many times and CTA c polls copy c % record_copies, so each
 *    record line is read by G / record_copies CTAs;
 *  poll_pause_ns (default 400): pause before a window's first record poll;
 *  drive_overlap (default 1): the Poisson drive of the steps after each
 *    persistent launch is computed on a side stream beside it (double
 *    buffer; a run that continues where the previous one ended finds its
 *    first drive ready); 0 runs every drive pass before its launch on the
 *    caller's stream;
 *  drive_chunk_steps (default 0 = up to 512 MB of drive per launch): the
 *    steps of one persistent launch; small chunks keep the two drive buffers
 *    resident in L2 beside the edge arrays, at one launch per chunk;
 *  record_stride_bytes (64..65536, multiple of 64; default 64): distance
 *    between two CTAs' records, which spreads the polled lines over L2. */
int bspk_plan_set_tiled_options(bspk_plan *plan, int record_copies, int poll_pause_ns,
                                int drive_overlap, int drive_chunk_steps,
                                int record_stride_bytes);
int bspk_plan_get_tiled_options(bspk_plan *plan, int *record_copies, int *poll_pause_ns,
                                int *drive_overlap, int *drive_chunk_steps,
                                int *record_stride_bytes);
/* Autotuner of the tiled path (no counterpart in the reference; the batch
 * path's is bspk_batch_tune).  Times pilot runs of pilot_steps on the plan's
 * own network for each CTA count G in {G0, 3/4 G0, 1/2 G0} (G0: the upload's
 * choice, one CTA per SM for large networks) whose tile fits
 * (a tile per CTA, rebuilt for each G) and each poll pause in {200, 400, 700}
 * ns (the faster of two pilots each), with the plan's state saved before and
 * restored after every pilot (the
 * plan is left where it was, at the best shape).  *grid, *poll_pause_ns and
 * *pilot_ms (the best pilot's device time) are optional.  Results of later
 * runs do not depend on the shape.  BSPK_ERR_STATE unless the plan is
 * uploaded and on the tiled path. */
int bspk_plan_tune_tiled(bspk_plan *plan, int64_t pilot_steps, int *grid, int *poll_pause_ns,
                         double *pilot_ms);

/* Synchronise and copy out what the last bspk_run recorded.
 * spikes: (step, gid) pairs in no particular order, *n_out = count. */
int bspk_spikes_get(bspk_plan *plan, int64_t cap, int64_t *steps, int32_t *gids,
                    int64_t *n_out);
/* V_m trace of the last run: [n_steps][n_rec] as double. */
int bspk_v_get(bspk_plan *plan, double *out);
/* The same V_m traces in float32 (the device's own values for a precision-32
 * plan, rounded for a precision-64 one). */
int bspk_v_get_f32(bspk_plan *plan, float *out);
int bspk_weights_get(bspk_plan *plan, int proj_id, double *w_csr_order);
/* Per-step weight trajectory of a plastic projection (Simulator.record_weight
 * and SimulationResult.weight_trace, _nest_network/simulator.py:382-396,
 * :884-910, :1868-1880): with recording on, every bspk_run stores the FP64
 * weights after each of its steps, [n_steps][n_edges] in CSR order, on the
 * device (n_steps * n_edges * 8 bytes).  weight_trace_get synchronises and
 * copies the last run's trajectory (*n_steps = its length; out may be NULL to
 * query it). */
int bspk_record_weights(bspk_plan *plan, int proj_id, int on);
int bspk_weight_trace_get(bspk_plan *plan, int proj_id, int64_t *n_steps, double *out);
int bspk_state_get(bspk_plan *plan, int pop, const char *name, double *values);
int bspk_state_set(bspk_plan *plan, int pop, const char *name, const double *values);
int64_t bspk_step_count(bspk_plan *plan);
/* The kernel family an uploaded plan runs on: "tiled" (target-partitioned
 * persistent kernel, ring in shared memory), "global_ring" (persistent
 * kernel with the ring in global memory, for tiles too large for shared
 * memory), "exact" (deterministic FP64 pull), "per_step" (conductance
 * models, separate ports or plasticity, one launch sequence per time step),
 * "windowed" (the same networks when every lag is >= 2 steps and at most
 * one pair-rule projection with one lag is plastic: each launch sequence
 * advances a window of W = min(lag, 32, 64 - max lag) steps, the neuron
 * kernel running its W steps back to back); "" before upload. */
const char *bspk_plan_engine(bspk_plan *plan);
/* Switch an uploaded plan that can run windowed between the windowed (1)
 * and the per-step (0) form; results agree up to the order of floating-point
 * additions into the conductance inputs.  Runs with weight recording
 * (bspk_record_weights) always take the per-step form.  Setting 1 on a plan
 * that cannot run windowed is BSPK_ERR_UNSUPPORTED. */
int bspk_plan_set_windowed(bspk_plan *plan, int on);
/* The tiled kernel sums arrivals in fixed point: weights are rounded once to
 * rint(w * 2^k) (int32 for FP32 plans, int64 for FP64 plans) with k chosen so
 * that no ring slot can overflow; *bits = k of an uploaded tiled plan. */
int bspk_plan_ring_fraction_bits(bspk_plan *plan, int *bits);

/* Timing of the dominant kernel of the last bspk_run (CUDA events on the
 * launching stream): total ms and number of launches. */
int bspk_last_kernel_time(bspk_plan *plan, double *ms, int64_t *launches);

/* RKF45 substeps (accepted and rejected) of every conductance-model neuron
 * since the plan was uploaded: the integrator's work, the counterpart of the
 * reference's per-neuron iteration count (_nest_base/utils.py:583-718).
 * Synchronises the plan's stream. */
int bspk_rk_substeps(bspk_plan *plan, int64_t *total);

/* Checkpoint of every device buffer that evolves (state, rings, spike
 * history, plastic weights and traces, step counter); restore is bit-exact
 * (simulator.py:1822-1839 continues without re-init). */
int bspk_checkpoint_size(bspk_plan *plan, int64_t *bytes);
int bspk_checkpoint_save(bspk_plan *plan, void *host_buf, int64_t bytes);
int bspk_checkpoint_restore(bspk_plan *plan, const void *host_buf, int64_t bytes);
/* Page-locked host memory for checkpoints and read-backs: a restore from it
 * is one host-to-device copy per section (no staging copy). */
int bspk_host_alloc(int64_t bytes, void **ptr);
int bspk_host_free(void *ptr);

/* fixed_indegree connectivity drawn on the GPU (one thread per edge, the
 * same key derivation and bits as bspk_proj_add_fixed_indegree) and sorted
 * into CSR by a stable radix sort, returned to host buffers indptr[n_pre+1]
 * and post_local[n_post*K].  Replaces sample_fixed_indegree + csr_structure
 * (_nest_network/connectivity.py:39-53, :101-135; kernel rule
 * _kernel/connectivity/rules.py:192-251), whose host build dominates the
 * reference's network construction. */
int bspk_gen_fixed_indegree(int device, int64_t seed, int n_pre, int n_post, int K,
                            int pre_is_post, int allow_autapses, int nbits, int64_t *indptr,
                            int32_t *post_local);

/* ---------------------------------------------------------------- batches
 * Many independent iaf networks ("instances") of uneven sizes advanced by
 * one persistent cooperative launch.  The reference batches only identical
 * structures (Runner(batch) vmap, _kernel/runner.py:832-863, trial keys
 * _kernel/rng.py:435-479); an instance here has its own populations,
 * fixed_indegree projections (built on the GPU at upload), Poisson drives
 * and seeds.  All projections of one instance share one delay (its
 * window); config fields as for plans (deterministic must be 0, model an
 * iaf model shared by all instances). */
typedef struct bspk_batch bspk_batch;
int bspk_batch_create(const bspk_config *cfg, bspk_batch **out);
int bspk_batch_destroy(bspk_batch *batch);
int bspk_batch_instance_add(bspk_batch *batch, int *inst);
int bspk_batch_pop_add(bspk_batch *batch, int inst, int n, const double *params, int n_params,
                       int *pop);
int bspk_batch_fixed_indegree_add(bspk_batch *batch, int inst, int pre_pop, int post_pop, int K,
                                  int64_t seed, int allow_autapses, int nbits, double weight,
                                  int delay_steps);
int bspk_batch_drive_add_poisson(bspk_batch *batch, int inst, int post_pop, double rate_hz,
                                 double weight, int delay_steps, uint32_t seed,
                                 int64_t t_min_step, int64_t t_max_step);
int bspk_batch_record_spikes(bspk_batch *batch, int inst, int on);
/* Build the device layout: tile = neurons per tile and threads per CTA
 * (multiple of 32 in [32, 512]; 0 = 256), ctas_per_sm <= 0 = as many as fit. */
int bspk_batch_upload(bspk_batch *batch, int tile, int ctas_per_sm, void *stream);
/* Autotuner: measures every instance's rate on a pilot run, then times
 * tile sizes x CTAs per SM on the same pilot (tile-to-CTA assignment by
 * longest-processing-time first over the calibrated cost model) and keeps
 * the fastest; the state is restored to what it was before the call. */
int bspk_batch_tune(bspk_batch *batch, int64_t pilot_steps, int *tile, int *ctas_per_sm,
                    double *pilot_ms);
int bspk_batch_shape(bspk_batch *batch, int *tile, int *ctas_per_sm, int *grid, int64_t *n_tiles);
int bspk_batch_run(bspk_batch *batch, int64_t n_steps, void *stream);
int bspk_batch_state_set(bspk_batch *batch, int inst, int pop, const char *name,
                         const double *values);
int bspk_batch_state_get(bspk_batch *batch, int inst, int pop, const char *name, double *values);
/* Spikes per neuron of an instance since upload. */
int bspk_batch_spike_counts(bspk_batch *batch, int inst, int64_t *counts);
/* (step, neuron) spikes of a recorded instance in the last run. */
int bspk_batch_spikes_get(bspk_batch *batch, int inst, int64_t cap, int64_t *steps, int32_t *ids,
                          int64_t *n_out);
/* An instance's edges as (pre, post, projection) in tile-CSR order. */
int bspk_batch_edges_get(bspk_batch *batch, int inst, int64_t cap, int32_t *pre, int32_t *post,
                         int32_t *proj, int64_t *n_out);
int64_t bspk_batch_step_count(bspk_batch *batch);
int bspk_batch_last_kernel_time(bspk_batch *batch, double *ms, int64_t *launches);

/* ---------------------------------------------------------------- gradients
 * Surrogate-gradient BPTT through a recurrent iaf_psc_exp network with a
 * hand-written adjoint: the forward pass stores checkpoints every
 * ckpt_every steps, the backward pass recomputes each segment from its
 * checkpoint and sweeps the adjoint through it.  Replaces jax.grad over the
 * reference's episode scan (BPTT._episode/_objective,
 * _kernel/learn/bptt.py:437-491) for this model: hard forward with the
 * count_ste surrogate (_kernel/spiking.py:65-88), soft reset gradient unless
 * detach_reset (SpikeRule._jump, _kernel/spiking.py:449-466), or the relaxed
 * forward (_check_relaxed, :422-447); loss = mean (z - y)^2 of readout rates
 * z_t = alpha z_{t-1} + c s_t (rate_mse, _kernel/learn/bptt.py:142-214).
 * Surrogate: fast sigmoid of the given slope (1/mV) as a smooth step,
 * s(m) = (1 + b m / (1 + b|m|)) / 2 with derivative (b/2) / (1 + b|m|)^2.
 * Structure: W row-major over post neurons (row_ptr[n+1], col[nnz] = pre).
 * Operands of forward/backward are DEVICE pointers of the precision's type
 * (float or double): w[nnz], w_in[n][n_in], inputs = uint8 counts
 * [n_steps][batch][n_in], targets [n_steps][batch][n_readout]; loss is a
 * device double (NULL: kept inside the handle), n_spikes an optional device
 * int64.  backward writes dL/dw and dL/dw_in for the operands of the last
 * forward on the handle. */
typedef struct {
    double dt;
    int precision;          /* 32 or 64 */
    int n, n_in, batch, n_steps, ckpt_every, n_readout;
    double readout_tau;     /* ms */
    double slope;           /* 1/mV */
    int relaxed, detach_reset, device;
    double params[9];       /* iaf_psc_exp: E_L C_m tau_m t_ref V_th V_reset tau_syn_ex tau_syn_in I_e */
} bspk_adjoint_config;
typedef struct bspk_adjoint bspk_adjoint;
int bspk_adjoint_create(const bspk_adjoint_config *cfg, const int64_t *row_ptr,
                        const int32_t *col, int64_t nnz, bspk_adjoint **out);
int bspk_adjoint_destroy(bspk_adjoint *adj);
/* CTAs per trial of the forward and adjoint kernels: 1, or 2 as a
 * thread-block cluster that splits a trial's neurons in half (chosen at
 * create when the batch leaves each trial two SMs, n >= 64 and the readouts
 * lie in the first half).  Both give bit-identical results. */
int bspk_adjoint_ctas_per_trial(const bspk_adjoint *adj);
int bspk_adjoint_forward(bspk_adjoint *adj, const void *w, const void *w_in,
                         const uint8_t *inputs, const void *targets, double *loss,
                         int64_t *n_spikes, void *stream);
int bspk_adjoint_backward(bspk_adjoint *adj, void *dw, void *dw_in, void *stream);
/* Element counts of the gradient operands (nnz recurrent weights, n * n_in
 * input weights) and the precision (32 / 64) of a handle. */
int bspk_adjoint_sizes(const bspk_adjoint *adj, int64_t *nnz, int64_t *n_w_in, int *precision);
/* How an FP32 handle forms the weight gradients.  1 (the default when the
 * buffers fit): the backward stores the input adjoint of every (step, trial,
 * neuron) and the recompute the previous step's spikes, and dL/dw, dL/dw_in
 * are dense contractions over (step, trial) on the tensor cores
 * (tcgen05.mma on bf16 parts that restate the FP32 operands, FP32
 * accumulation) followed by a gather of the edges (partial sums added in a
 * fixed order: deterministic).  0: per-trial
 * read-modify-writes in time order, summed over trials in trial order (the
 * only mode of FP64 handles, bit-exact with the float64 restatement).
 * Setting 1 on an FP64 handle, or on one whose buffers could not be
 * allocated, is BSPK_ERR_UNSUPPORTED. */
int bspk_adjoint_set_contraction(bspk_adjoint *adj, int on);
int bspk_adjoint_contraction(const bspk_adjoint *adj);
/* Synchronise the device and report (then clear) the handle's device error
 * flag: BSPK_ERR_TIMEOUT if a bounded wait of the tensor-core contraction
 * ran out since the last call. */
int bspk_adjoint_status(bspk_adjoint *adj);

/* No-allocation entry point (no counterpart in the reference).  For callers
 * that cannot call cudaMalloc -- code running inside another framework's
 * memory pool or allocation hooks, or a plugin host that forbids device
 * allocations -- this runs the deterministic FP64 network step for ONE
 * iaf_psc_alpha population without a plan and allocates nothing: every input
 * and output is a caller-owned device buffer, and the kernel's scratch
 * (parameter tables, Poisson CDF, spike-history words, barrier counter,
 * error flag, spike counter) lives in one fixed-size device array inside
 * the library, held by every GPU that loads it until the process exits.
 *
 * Network: a Poisson drive (rate, weight, delay, seed; created first), then
 * one recurrent projection given as in-edges per post neuron:
 * in_indptr[n+1], in_edges[E] = pre | (delay_steps + 1) << 24 in ascending
 * pre order (pre < n and min_delay_steps <= delay_steps <= max_delay_steps
 * for every edge; the kernel does not check them), per-edge weights in_w[E]
 * or NULL with w_const; in_edges must not be NULL, even for E = 0.
 * Reference Simulator timing (a spike of step m arrives at m + D + 1).
 * state: [6][n] doubles (V_m, I_syn_ex, dI_syn_ex, I_syn_in, dI_syn_in, y0),
 * refr: [n] refractory counters, both read and written.  Outputs, all device
 * memory: spikes as (step within this call, neuron) pairs; *spike_count is
 * the number of spikes of the call, which may exceed spike_cap: only the
 * first min(*spike_count, spike_cap) pairs are written, and *status is then
 * BSPK_DEV_ERR_OVERFLOW (2).  *status is 0 when the call completed, else a
 * device error code (1 = a bounded wait ran out).
 *
 * Limits: n <= 65536 neurons (the scratch array) and no more than the
 * cooperative launch can keep resident, 256 neurons per SM on a B200
 * (37 888 neurons on 148 SMs; larger networks return BSPK_ERR_UNSUPPORTED
 * with the limit in bspk_last_error()); delays <= 61 steps; drive CDF <=
 * 4096 entries (BSPK_ERR_ARG beyond).  Each call starts with an empty spike
 * history (spikes of earlier calls are not delivered) and restarts the
 * drive's random stream at step 0, so calls that continue a run need a new
 * drive_seed each.  All calls on a device share the scratch array, so calls
 * that overlap on the GPU race; serialise them.  The first call on a device
 * looks up the scratch array's device address (once per device, with that
 * device current).  Every call copies its small tables (coefficients, drive,
 * CDF, projection descriptor) from host memory with cudaMemcpyAsync, so no
 * call may be made on a stream that is being captured into a CUDA graph. */
int bspk_iaf_exact_run_noalloc(double dt, const double *params, int n_params, int n,
                               const int64_t *in_indptr, const uint32_t *in_edges,
                               const double *in_w, double w_const, int min_delay_steps,
                               int max_delay_steps, double drive_rate_hz, double drive_weight,
                               int drive_delay_steps, uint32_t drive_seed, double *state,
                               int32_t *refr, int64_t n_steps, int64_t *spike_step,
                               int32_t *spike_gid, int64_t spike_cap, int64_t *spike_count,
                               int *status, void *stream);

#ifdef __cplusplus
}
#endif
#endif
