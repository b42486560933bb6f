// plan.cpp -- host side of libbspk: the C ABI declared in include/bspk.h.
//
// A plan is built on the host (populations, projections, drives), uploaded
// once, then advanced by bspk_run.  All float64 preprocessing (propagators,
// Poisson CDF tables, connectivity sampling, CSR/CSC layouts) happens here;
// the kernels only see packed device structures.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/bspk.h"
#include "aeif_args.h"
#include "coef_cast.h"
#include "device_types.h"
#include "host_rng.h"
#include "jax_rng.h"
#include "lif_args.h"
#include "stdp_args.h"
#include "plan_internal.h"

using namespace bspk;

namespace bspk {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

}  // namespace bspk

namespace {

template <typename T>
int dalloc(bspk_plan *p, T **ptr, size_t count) {
    void *raw = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&raw, sizeof(T) * count);
    if (e != cudaSuccess)
        return fail(BSPK_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    p->allocs.push_back(raw);
    *ptr = static_cast<T *>(raw);
    return BSPK_OK;
}

}  // namespace

int bspk::dalloc_bytes(bspk_plan *p, void **ptr, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess)
        return fail(BSPK_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    p->allocs.push_back(*ptr);
    return BSPK_OK;
}

namespace {

template <typename T>
int upload_vec(bspk_plan *p, T **ptr, const std::vector<T> &v) {
    int rc = dalloc(p, ptr, v.size());
    if (rc) return rc;
    if (!v.empty()) BSPK_CUDA(cudaMemcpy(*ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return BSPK_OK;
}

const char *kStateNames[6][9] = {
    {"V_m", "I_syn_ex", "dI_syn_ex", "I_syn_in", "dI_syn_in", "y0", "", "", ""},
    {"V_m", "i_syn_ex", "i_syn_in", "i_0", "i_1", "", "", "", ""},
    {"V_m", "dg_ex", "g_ex", "dg_in", "g_in", "w", "h", "I_stim", ""},
    {"V_m", "g_ex", "g_in", "h", "I_stim", "", "", "", ""},
    {"V_m", "dg_ex", "g_ex", "dg_in", "g_in", "h", "I_stim", "", ""},
    {"V_m", "i_const", "i_syn_0", "i_syn_1", "i_syn_2", "i_syn_3", "", "", ""},
};

int state_slot(int model, const char *name) {
    if (!strcmp(name, "r") || !strcmp(name, "refractory_step_count")) return 100;
    for (int i = 0; i < 9; ++i)
        if (kStateNames[model][i][0] && !strcmp(kStateNames[model][i], name)) return i;
    return -1;
}

int n_state_slots(int model) { return model_n_slots(model); }

// Float64 propagators and thresholds, following the reference formulas
// (_nest_neuron/iaf_psc_alpha.py:451-556, iaf_psc_exp.py:492-512,
// _nest_base/utils.py:126-229).
void alpha_p31_p32(double tau_syn, double tau_m, double c_m, double h, double *p31, double *p32) {
    const double beta = tau_syn * tau_m / (tau_m - tau_syn);
    const double gamma = beta / c_m;
    const double inv_beta = (tau_m - tau_syn) / (tau_syn * tau_m);
    const double exp_h_tau_syn = std::exp(-h / tau_syn);
    const double expm1_h_tau = std::expm1(h * inv_beta);
    const double p32_raw = gamma * exp_h_tau_syn * expm1_h_tau;
    const double exp_h_tau_m = std::exp(-h / tau_m);
    const double p32_singular = h / c_m * exp_h_tau_m;
    const bool reg32 = std::isfinite(p32_raw) && std::fabs(p32_raw) >= 2.2250738585072014e-308 &&
                       p32_raw > 0.0;
    *p32 = reg32 ? p32_raw : p32_singular;
    const double h_min_regular = 1e-7 * tau_m * tau_m / std::fabs(tau_m - tau_syn);
    const bool reg31 = std::isfinite(h_min_regular) && (h > h_min_regular);
    const double p31_regular = gamma * exp_h_tau_syn * (beta * expm1_h_tau - h);
    const double p31_singular = 0.5 * h * h / c_m * exp_h_tau_m;
    *p31 = reg31 ? p31_regular : p31_singular;
}

double propagator_exp(double tau_syn, double tau_m, double c_m, double h) {
    const double beta = tau_syn * tau_m / (tau_m - tau_syn);
    const double gamma = beta / c_m;
    const double inv_beta = (tau_m - tau_syn) / (tau_syn * tau_m);
    const double exp_h_tau_syn = std::exp(-h / tau_syn);
    const double expm1_h_tau = std::expm1(h * inv_beta);
    const double p32_raw = gamma * exp_h_tau_syn * expm1_h_tau;
    const bool reg = std::isfinite(p32_raw) && std::fabs(p32_raw) >= 2.2250738585072014e-308 &&
                     p32_raw > 0.0;
    return reg ? p32_raw : h / c_m * std::exp(-h / tau_m);
}

constexpr double kE = 2.718281828459045;

// Reciprocals of the conductance models' divisors, in FP64, for the RKF45
// stages.  A zero Delta_T leaves the exponential term at zero whatever its
// argument, so its scale is then 1.
void set_cond_reciprocals(PopCoef<double> *c) {
    c->inv_C_m = 1.0 / c->C_m;
    c->inv_tau_syn_ex = 1.0 / c->tau_syn_ex;
    c->inv_tau_syn_in = 1.0 / c->tau_syn_in;
    c->inv_tau_w = c->tau_w > 0.0 ? 1.0 / c->tau_w : 0.0;
    c->inv_Delta_T = c->Delta_T == 0.0 ? 1.0 : 1.0 / c->Delta_T;
    c->inv_atol = 1.0 / c->atol;
}

int make_coef(int model, const std::vector<double> &p, double h, PopCoef<double> *c) {
    memset(c, 0, sizeof(*c));
    if (model == BSPK_IAF_PSC_ALPHA || model == BSPK_IAF_PSC_EXP) {
        const size_t need = model == BSPK_IAF_PSC_ALPHA ? 10 : 9;
        if (p.size() < need) return fail(BSPK_ERR_ARG, "too few parameters");
        const double E_L = p[0], C_m = p[1], tau_m = p[2], t_ref = p[3], V_th = p[4],
                     V_reset = p[5], tex = p[6], tin = p[7], I_e = p[8];
        // parameter validation (iaf_psc_alpha.py:385-410)
        if (!(C_m > 0)) return fail(BSPK_ERR_ARG, "Capacitance must be > 0.");
        if (!(tau_m > 0)) return fail(BSPK_ERR_ARG, "Membrane time constant must be > 0.");
        if (!(tex > 0) || !(tin > 0))
            return fail(BSPK_ERR_ARG, "All synaptic time constants must be > 0.");
        if (t_ref < 0) return fail(BSPK_ERR_ARG, "The refractory time t_ref can't be negative.");
        if (!(V_reset < V_th)) return fail(BSPK_ERR_ARG, "Reset potential must be smaller than threshold.");
        c->E_L = E_L;
        c->I_e = I_e;
        c->theta = V_th - E_L;
        c->vreset = V_reset - E_L;
        c->lower = model == BSPK_IAF_PSC_ALPHA ? p[9] - E_L : -INFINITY;
        c->ref_count = static_cast<int>(std::ceil(t_ref / h));
        c->P11ex = std::exp(-h / tex);
        c->P22ex = c->P11ex;
        c->P21ex = h * c->P11ex;
        c->P11in = std::exp(-h / tin);
        c->P22in = c->P11in;
        c->P21in = h * c->P11in;
        c->expm1_tm = std::expm1(-h / tau_m);
        c->P30 = -tau_m / C_m * c->expm1_tm;
        alpha_p31_p32(tex, tau_m, C_m, h, &c->P31ex, &c->P32ex);
        alpha_p31_p32(tin, tau_m, C_m, h, &c->P31in, &c->P32in);
        c->epsc = kE / tex;
        c->ipsc = kE / tin;
        c->eP11ex = std::exp(-h / tex);
        c->eP11in = std::exp(-h / tin);
        c->eP22 = std::exp(-h / tau_m);
        c->eP21ex = propagator_exp(tex, tau_m, C_m, h);
        c->eP21in = propagator_exp(tin, tau_m, C_m, h);
        c->eP20 = tau_m / C_m * (1.0 - std::exp(-h / tau_m));
        c->one_m_eP11ex = 1.0 - c->eP11ex;
        return BSPK_OK;
    }
    if (model == BSPK_AEIF_COND_ALPHA) {
        if (p.size() < 17) return fail(BSPK_ERR_ARG, "too few parameters");
        c->V_peak = p[0];
        c->V_reset = p[1];
        const double t_ref = p[2];
        c->g_L = p[3];
        c->C_m = p[4];
        c->E_ex = p[5];
        c->E_in = p[6];
        c->E_L = p[7];
        c->Delta_T = p[8];
        c->tau_w = p[9];
        c->a = p[10];
        c->b = p[11];
        c->V_th = p[12];
        c->tau_syn_ex = p[13];
        c->tau_syn_in = p[14];
        c->I_e = p[15];
        c->atol = p[16];
        // validation (aeif_cond_alpha.py:_validate_parameters, utils.py:85-119)
        if (!(c->V_peak >= c->V_th)) return fail(BSPK_ERR_ARG, "V_peak >= V_th required.");
        if (c->Delta_T < 0) return fail(BSPK_ERR_ARG, "Delta_T must be positive.");
        if (!(c->C_m > 0)) return fail(BSPK_ERR_ARG, "Capacitance must be strictly positive.");
        if (t_ref < 0) return fail(BSPK_ERR_ARG, "Refractory time cannot be negative.");
        if (!(c->tau_syn_ex > 0) || !(c->tau_syn_in > 0) || !(c->tau_w > 0))
            return fail(BSPK_ERR_ARG, "All time constants must be strictly positive.");
        if (!(c->atol > 0)) return fail(BSPK_ERR_ARG, "The gsl_error_tol must be strictly positive.");
        if (c->Delta_T > 0) {
            const double max_exp_arg = std::log(1.7976931348623157e308 / 1e20);
            if ((c->V_peak - c->V_th) / c->Delta_T >= max_exp_arg)
                return fail(BSPK_ERR_ARG, "The current combination of V_peak, V_th and Delta_T will "
                                          "lead to numerical overflow at spike time.");
        }
        c->ref_count = static_cast<int>(std::ceil(t_ref / h));
        c->pscon_ex = kE / c->tau_syn_ex;
        c->pscon_in = kE / c->tau_syn_in;
        c->v_peak_detect = c->Delta_T > 0.0 ? c->V_peak : c->V_th;
        set_cond_reciprocals(c);
        return BSPK_OK;
    }
    if (model == BSPK_IAF_COND_EXP || model == BSPK_IAF_COND_ALPHA) {
        if (p.size() < 12) return fail(BSPK_ERR_ARG, "too few parameters");
        c->E_L = p[0];
        c->C_m = p[1];
        const double t_ref = p[2];
        c->V_th = p[3];
        c->V_reset = p[4];
        c->E_ex = p[5];
        c->E_in = p[6];
        c->g_L = p[7];
        c->tau_syn_ex = p[8];
        c->tau_syn_in = p[9];
        c->I_e = p[10];
        c->atol = p[11];
        // validation (iaf_cond_exp.py:360-379, iaf_cond_alpha.py:368-385)
        if (!(c->V_reset < c->V_th)) return fail(BSPK_ERR_ARG, "Reset potential must be smaller than threshold.");
        if (!(c->C_m > 0)) return fail(BSPK_ERR_ARG, "Capacitance must be strictly positive.");
        if (t_ref < 0) return fail(BSPK_ERR_ARG, "Refractory time cannot be negative.");
        if (!(c->tau_syn_ex > 0) || !(c->tau_syn_in > 0))
            return fail(BSPK_ERR_ARG, model == BSPK_IAF_COND_EXP
                                          ? "All synaptic time constants must be strictly positive."
                                          : "All time constants must be strictly positive.");
        if (model == BSPK_IAF_COND_EXP && !(c->atol > 0))
            return fail(BSPK_ERR_ARG, "The gsl_error_tol must be strictly positive.");
        c->ref_count = static_cast<int>(std::ceil(t_ref / h));
        // jumps after integration: g += w (exp), dg += e / tau * w (alpha)
        c->pscon_ex = model == BSPK_IAF_COND_ALPHA ? kE / c->tau_syn_ex : 1.0;
        c->pscon_in = model == BSPK_IAF_COND_ALPHA ? kE / c->tau_syn_in : 1.0;
        c->V_peak = c->V_th;
        c->v_peak_detect = c->V_th;
        set_cond_reciprocals(c);
        return BSPK_OK;
    }
    if (model == BSPK_IAF_PSC_EXP_MULTISYNAPSE) {
        if (p.size() < 9) return fail(BSPK_ERR_ARG, "too few parameters");
        const double E_L = p[0], C_m = p[1], tau_m = p[2], t_ref = p[3], V_th = p[4],
                     V_reset = p[5], I_e = p[6];
        const int nrec = static_cast<int>(p[7]);
        if (nrec < 1 || nrec > kMaxReceptors || static_cast<double>(nrec) != p[7])
            return fail(BSPK_ERR_UNSUPPORTED, "n_receptors must be 1..4");
        if (p.size() < static_cast<size_t>(8 + nrec)) return fail(BSPK_ERR_ARG, "too few parameters");
        // validation (iaf_psc_exp_multisynapse.py:463-477)
        if (!(V_reset < V_th)) return fail(BSPK_ERR_ARG, "Reset potential must be smaller than threshold.");
        if (!(C_m > 0)) return fail(BSPK_ERR_ARG, "Capacitance must be > 0.");
        if (!(tau_m > 0)) return fail(BSPK_ERR_ARG, "Membrane time constant must be strictly positive.");
        for (int k = 0; k < nrec; ++k)
            if (!(p[8 + k] > 0))
                return fail(BSPK_ERR_ARG, "All synaptic time constants must be strictly positive.");
        for (int k = 0; k < nrec; ++k)  // numpy isclose: |a - b| <= 1e-8 + 1e-5 |b|
            if (std::fabs(p[8 + k] - tau_m) <= 1e-8 + 1e-5 * std::fabs(tau_m))
                return fail(BSPK_ERR_ARG, "Membrane and synapse time constants must differ.");
        if (t_ref < 0) return fail(BSPK_ERR_ARG, "Refractory time must not be negative.");
        // propagators (iaf_psc_exp_multisynapse.py:523-552)
        c->E_L = E_L;
        c->I_e = I_e;
        c->theta = V_th - E_L;
        c->vreset = V_reset - E_L;
        c->ref_count = static_cast<int>(std::ceil(t_ref / h));
        c->eP22 = std::exp(-h / tau_m);
        c->eP20 = tau_m / C_m * (1.0 - c->eP22);
        c->nrec = nrec;
        for (int k = 0; k < nrec; ++k) {
            c->msP11[k] = std::exp(-h / p[8 + k]);
            c->msP21[k] = propagator_exp(p[8 + k], tau_m, C_m, h);
        }
        return BSPK_OK;
    }
    return fail(BSPK_ERR_ARG, "unknown model");
}


// CDF table of Poisson(lam): F[0] = exp(-lam), p_k = p_{k-1} * lam / k,
// F[k] = F[k-1] + p_k, until F stops growing.  The count for a uniform u is
// the smallest k with u <= F[k] (table length if none).
std::vector<double> poisson_cdf(double lam) {
    std::vector<double> F;
    double p = std::exp(-lam), Fk = p;
    F.push_back(Fk);
    for (int k = 1; k < 4096; ++k) {
        p = p * lam;
        p = p / static_cast<double>(k);
        const double Fn = Fk + p;
        if (!(Fn > Fk)) break;
        Fk = Fn;
        F.push_back(Fk);
    }
    return F;
}

int lag_of(const bspk_plan *p, int delay_steps) {
    return p->cfg.semantics == BSPK_LEGACY ? delay_steps + 1 : delay_steps;
}

}  // namespace

// Host helpers shared with other translation units.
int bspk::host_make_coef(int model, const std::vector<double> &params, double h,
                         PopCoef<double> *c) {
    return make_coef(model, params, h, c);
}

std::vector<uint64_t> bspk::host_poisson_thresholds(double lam) {
    std::vector<uint64_t> t;
    for (double F : poisson_cdf(lam)) t.push_back(static_cast<uint64_t>(std::floor(std::ldexp(F, 53))));
    return t;
}

// =================================================================== C ABI

namespace {
// Receptor ports: 0 for the iaf_psc models (all inputs summed), 0/1 (g_ex /
// g_in) for the conductance models, 0..n_receptors-1 of the post population
// for iaf_psc_exp_multisynapse.
int check_receptor(const bspk_plan *p, int post_pop, int receptor) {
    const int model = p->cfg.model;
    if (p->ports_sep) {
        if (receptor < 0 || receptor > 1) return fail(BSPK_ERR_ARG, "receptor must be 0 ('ex') or 1 ('in_')");
        return BSPK_OK;
    }
    if (model == BSPK_IAF_PSC_EXP_MULTISYNAPSE) {
        const int n = p->pops[post_pop].c.nrec;
        if (receptor < 0 || receptor >= n)
            return fail(BSPK_ERR_ARG, "receptor must be below the population's n_receptors (" +
                                          std::to_string(n) + ")");
        return BSPK_OK;
    }
    if (receptor < 0 || receptor > 1) return fail(BSPK_ERR_ARG, "receptor must be 0 or 1");
    if (receptor != 0 && !model_is_cond(model))
        return fail(BSPK_ERR_ARG, "receptor ports are for conductance models; current models sum all inputs");
    return BSPK_OK;
}
}  // namespace

extern "C" {

const char *bspk_version(void) { return "bspk 0.1 (sm_100a)"; }
const char *bspk_last_error(void) { return g_err.c_str(); }

int bspk_plan_create(const bspk_config *cfg, bspk_plan **out) {
    if (!cfg || !out) return fail(BSPK_ERR_ARG, "null argument");
    if (!(cfg->dt > 0)) return fail(BSPK_ERR_ARG, "dt must be > 0");
    if (cfg->precision != 32 && cfg->precision != 64)
        return fail(BSPK_ERR_ARG, "precision must be 32 or 64");
    if (cfg->model < 0 || cfg->model > 5) return fail(BSPK_ERR_ARG, "unknown model");
    if (cfg->semantics != BSPK_LEGACY && cfg->semantics != BSPK_RING)
        return fail(BSPK_ERR_ARG, "unknown delivery semantics");
    if (cfg->deterministic && (cfg->precision != 64 || cfg->semantics != BSPK_LEGACY ||
                               model_per_step(cfg->model)))
        return fail(BSPK_ERR_UNSUPPORTED,
                    "deterministic mode needs precision 64, LEGACY semantics and an iaf model");
    bspk_plan *p = new bspk_plan();
    p->cfg = *cfg;
    if (p->cfg.spike_capacity <= 0) p->cfg.spike_capacity = 1 << 22;
    p->elt = cfg->precision == 64 ? 8 : 4;
    *out = p;
    return BSPK_OK;
}

int bspk_plan_destroy(bspk_plan *p) {
    if (!p) return BSPK_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    if (p->uploaded) cudaSetDevice(p->cfg.device);
    for (void *a : p->allocs) cudaFree(a);
    if (p->h_stage) cudaFreeHost(p->h_stage);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->ev_side) cudaEventDestroy(p->ev_side);
    if (p->ev_main) cudaEventDestroy(p->ev_main);
    if (p->side) cudaStreamDestroy(p->side);
    cudaSetDevice(dev);
    delete p;
    return BSPK_OK;
}

int bspk_pop_add(bspk_plan *p, int n, const double *params, int n_params, int *pop_id) {
    if (!p || n < 0 || !params) return fail(BSPK_ERR_ARG, "bad population");
    if (p->uploaded) return fail(BSPK_ERR_STATE, "plan already uploaded");
    if (static_cast<int>(p->pops.size()) >= kMaxPops) return fail(BSPK_ERR_ARG, "too many populations");
    Pop P;
    P.n = n;
    P.off = p->N;
    P.p.assign(params, params + n_params);
    int rc = make_coef(p->cfg.model, P.p, p->cfg.dt, &P.c);
    if (rc) return rc;
    P.c.off = P.off;
    P.c.n = n;
    p->pops.push_back(P);
    p->N += n;
    if (pop_id) *pop_id = static_cast<int>(p->pops.size()) - 1;
    return BSPK_OK;
}

int bspk_proj_add_csr(bspk_plan *p, int pre_pop, int post_pop, int64_t n_edges,
                      const int64_t *indptr, const int32_t *post_local, const double *w,
                      const int32_t *delay_steps, int receptor, int *proj_id) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (p->uploaded) return fail(BSPK_ERR_STATE, "plan already uploaded");
    const int npop = static_cast<int>(p->pops.size());
    if (pre_pop < 0 || pre_pop >= npop || post_pop < 0 || post_pop >= npop)
        return fail(BSPK_ERR_ARG, "population index out of range");
    if (n_edges < 0 || (n_edges > 0 && (!post_local || !w || !delay_steps)) || !indptr)
        return fail(BSPK_ERR_ARG, "bad edge arrays");
    const int rc0 = check_receptor(p, post_pop, receptor);
    if (rc0) return rc0;
    if (static_cast<int>(p->input_kind.size()) >= kMaxInputs) return fail(BSPK_ERR_ARG, "too many inputs");
    const int npre = p->pops[pre_pop].n, npost = p->pops[post_pop].n;
    if (npost >= (1 << kEdgeDelayShift) || npre >= (1 << kEdgeDelayShift))
        return fail(BSPK_ERR_UNSUPPORTED, "population larger than 2^24 neurons");
    Proj J;
    J.pre = pre_pop;
    J.post = post_pop;
    J.receptor = receptor;
    J.indptr.assign(indptr, indptr + npre + 1);
    if (J.indptr[0] != 0 || J.indptr[npre] != n_edges) return fail(BSPK_ERR_ARG, "indptr does not span the edges");
    for (int i = 0; i < npre; ++i)
        if (J.indptr[i + 1] < J.indptr[i]) return fail(BSPK_ERR_ARG, "indptr not monotone");
    J.post_local.assign(post_local, post_local + n_edges);
    J.delay.assign(delay_steps, delay_steps + n_edges);
    J.w.assign(w, w + n_edges);
    for (int64_t e = 0; e < n_edges; ++e) {
        if (J.post_local[e] < 0 || J.post_local[e] >= npost) return fail(BSPK_ERR_ARG, "post index out of range");
        const int lag = lag_of(p, J.delay[e]);
        if (lag < 1 || lag > 250) return fail(BSPK_ERR_ARG, "delay out of range (1..250 steps of arrival lag)");
        if (!std::isfinite(J.w[e])) return fail(BSPK_ERR_ARG, "non-finite weight");
    }
    J.homogeneous = n_edges > 0;
    for (int64_t e = 1; e < n_edges; ++e)
        if (J.w[e] != J.w[0]) { J.homogeneous = false; break; }
    J.w0 = n_edges > 0 ? J.w[0] : 0.0;
    J.input_order = static_cast<int>(p->input_kind.size());
    p->projs.push_back(std::move(J));
    const int id = static_cast<int>(p->projs.size()) - 1;
    p->input_kind.push_back(id);
    if (proj_id) *proj_id = id;
    return BSPK_OK;
}

int bspk_proj_add_fixed_indegree(bspk_plan *p, int pre_pop, int post_pop, int K, int64_t seed,
                                 int allow_autapses, int nbits, double weight,
                                 const int32_t *delay_steps, int delay_const, int receptor,
                                 int *proj_id) {
    return bspk_proj_add_fixed_indegree_w(p, pre_pop, post_pop, K, seed, allow_autapses, nbits,
                                          weight, nullptr, delay_steps, delay_const, receptor,
                                          proj_id);
}

int bspk_proj_add_fixed_indegree_w(bspk_plan *p, int pre_pop, int post_pop, int K, int64_t seed,
                                   int allow_autapses, int nbits, double weight,
                                   const double *w_draw, const int32_t *delay_steps,
                                   int delay_const, int receptor, int *proj_id) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    const int npop = static_cast<int>(p->pops.size());
    if (pre_pop < 0 || pre_pop >= npop || post_pop < 0 || post_pop >= npop)
        return fail(BSPK_ERR_ARG, "population index out of range");
    if (K < 0) return fail(BSPK_ERR_ARG, "K must be >= 0");
    if (nbits != 32 && nbits != 64) return fail(BSPK_ERR_ARG, "nbits must be 32 or 64");
    const int npre = p->pops[pre_pop].n, npost = p->pops[post_pop].n;
    const bool pre_is_post = pre_pop == post_pop;
    std::vector<int32_t> pre(static_cast<size_t>(npost) * K), post(pre.size());
    int rc = host_fixed_indegree(seed, npre, npost, K, pre_is_post, allow_autapses != 0, nbits,
                                 pre.data(), post.data());
    if (rc) return fail(BSPK_ERR_ARG, "fixed_indegree: a target has no available source");
    const int64_t E = static_cast<int64_t>(pre.size());
    std::vector<int64_t> order(E), indptr(npre + 1);
    std::vector<int32_t> indices(E);
    host_csr_structure(pre.data(), post.data(), E, npre, order.data(), indices.data(), indptr.data());
    std::vector<int32_t> dl(E);
    for (int64_t e = 0; e < E; ++e) dl[e] = delay_steps ? delay_steps[order[e]] : delay_const;
    std::vector<double> w(E, weight);
    if (w_draw)
        for (int64_t e = 0; e < E; ++e) w[e] = w_draw[order[e]];
    return bspk_proj_add_csr(p, pre_pop, post_pop, E, indptr.data(), indices.data(), w.data(),
                             dl.data(), receptor, proj_id);
}

int bspk_drive_add_poisson(bspk_plan *p, int post_pop, double rate_hz, double weight,
                           int delay_steps, uint32_t seed, int64_t t_min_step,
                           int64_t t_max_step, int receptor, int *drive_id) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (p->uploaded) return fail(BSPK_ERR_STATE, "plan already uploaded");
    if (post_pop < 0 || post_pop >= static_cast<int>(p->pops.size()))
        return fail(BSPK_ERR_ARG, "population index out of range");
    if (static_cast<int>(p->input_kind.size()) >= kMaxInputs) return fail(BSPK_ERR_ARG, "too many inputs");
    const int rc0 = check_receptor(p, post_pop, receptor);
    if (rc0) return rc0;
    const double lam = rate_hz * p->cfg.dt / 1000.0;
    if (!(lam >= 0) || lam > 700.0) return fail(BSPK_ERR_ARG, "rate*dt/1000 must be in [0, 700]");
    const int lag = lag_of(p, delay_steps);
    if (lag < 0 || delay_steps < 0) return fail(BSPK_ERR_ARG, "negative delay");
    Drive D;
    D.post = post_pop;
    D.lag = lag;
    D.delay = delay_steps;
    D.receptor = receptor;
    D.rate = rate_hz;
    D.weight = weight;
    D.seed = seed;
    D.tmin = t_min_step;
    D.tmax = rate_hz > 0 ? t_max_step : t_min_step;  // rate <= 0: never active
    D.cdf = poisson_cdf(lam);
    D.input_order = static_cast<int>(p->input_kind.size());
    p->drives.push_back(std::move(D));
    const int id = static_cast<int>(p->drives.size()) - 1;
    p->input_kind.push_back(-(id + 1));
    if (drive_id) *drive_id = id;
    return BSPK_OK;
}

int bspk_drive_add_poisson_keyed(bspk_plan *p, int post_pop, double rate_hz, double weight,
                                 int delay_steps, const uint32_t *obj_key, int64_t unit_off,
                                 int64_t t_min_step, int64_t t_max_step, int receptor,
                                 int *drive_id) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (!obj_key) return fail(BSPK_ERR_ARG, "null key");
    if (unit_off < 0 || unit_off > 0xFFFFFFFFll)
        return fail(BSPK_ERR_ARG, "unit offset out of range");
    const float lam = kernel_poisson_lam(rate_hz, p->cfg.dt);
    if (!(lam >= 0.0f) || lam >= 10.0f)
        return fail(BSPK_ERR_UNSUPPORTED,
                    "the kernel stream's CDF inversion needs rate*dt/1000 < 10 (larger means use "
                    "jax.random.poisson, which is not restated)");
    int id = -1;
    const int rc = bspk_drive_add_poisson(p, post_pop, rate_hz, weight, delay_steps, 0u, t_min_step,
                                          t_max_step, receptor, &id);
    if (rc) return rc;
    if (unit_off + p->pops[post_pop].n - 1 > 0xFFFFFFFFll) {
        p->drives.pop_back();
        p->input_kind.pop_back();
        return fail(BSPK_ERR_ARG, "units beyond 2^32");
    }
    Drive &D = p->drives[id];
    D.kind = 1;
    D.key0 = obj_key[0];
    D.key1 = obj_key[1];
    D.unit_off = unit_off;
    D.thr = kernel_poisson_table(lam);
    if (drive_id) *drive_id = id;
    return BSPK_OK;
}

int bspk_proj_csr_get(bspk_plan *p, int proj_id, int64_t *indptr, int32_t *post_local,
                      int32_t *delay_steps, double *w) {
    if (!p || proj_id < 0 || proj_id >= static_cast<int>(p->projs.size()))
        return fail(BSPK_ERR_ARG, "bad projection");
    const Proj &J = p->projs[proj_id];
    if (indptr) std::copy(J.indptr.begin(), J.indptr.end(), indptr);
    if (post_local) std::copy(J.post_local.begin(), J.post_local.end(), post_local);
    if (delay_steps) std::copy(J.delay.begin(), J.delay.end(), delay_steps);
    if (w) std::copy(J.w.begin(), J.w.end(), w);
    return BSPK_OK;
}

}  // extern "C"

namespace {
// Checks shared by the plastic rules: an existing CSR projection of a plan
// that is not uploaded, one homogeneous delay (the substrate's InputDelay).
int plastic_checks(bspk_plan *p, int proj_id) {
    if (p->uploaded) return fail(BSPK_ERR_STATE, "plan already uploaded");
    if (proj_id < 0 || proj_id >= static_cast<int>(p->projs.size())) return fail(BSPK_ERR_ARG, "bad projection");
    if (p->cfg.deterministic) return fail(BSPK_ERR_UNSUPPORTED, "STDP is not available in deterministic mode");
    const Proj &J = p->projs[proj_id];
    for (size_t e = 1; e < J.delay.size(); ++e)
        if (J.delay[e] != J.delay[0])
            return fail(BSPK_ERR_UNSUPPORTED, "a plastic projection needs one homogeneous delay");
    return BSPK_OK;
}
}  // namespace

extern "C" {

int bspk_proj_set_weights(bspk_plan *p, int proj_id, int64_t n_edges, const double *w) {
    if (!p || !w) return fail(BSPK_ERR_ARG, "null argument");
    if (p->uploaded) return fail(BSPK_ERR_STATE, "plan already uploaded");
    if (proj_id < 0 || proj_id >= static_cast<int>(p->projs.size())) return fail(BSPK_ERR_ARG, "bad projection");
    Proj &J = p->projs[proj_id];
    if (n_edges != static_cast<int64_t>(J.post_local.size()))
        return fail(BSPK_ERR_ARG, "weights must cover every edge of the projection");
    if (J.plastic) return fail(BSPK_ERR_STATE, "set the weights before making the projection plastic");
    J.w.assign(w, w + n_edges);
    J.homogeneous = false;
    return BSPK_OK;
}

int bspk_stdp_attach(bspk_plan *p, int proj_id, const bspk_stdp_params *sp) {
    if (!p || !sp) return fail(BSPK_ERR_ARG, "null argument");
    if (!(sp->tau_plus > 0)) return fail(BSPK_ERR_ARG, "'tau_plus' must be > 0.");
    if (!(sp->tau_minus > 0)) return fail(BSPK_ERR_ARG, "'tau_minus' must be > 0.");
    int rc = plastic_checks(p, proj_id);
    if (rc) return rc;
    Proj &J = p->projs[proj_id];
    for (double w : J.w)
        if ((w > 0) != (sp->Wmax > 0) && w != 0.0)
            return fail(BSPK_ERR_ARG, "Weight and Wmax must have same sign.");
    J.plastic = true;
    J.homogeneous = false;
    J.rule = 0;
    J.stdp = *sp;
    return BSPK_OK;
}

int bspk_stdp_triplet_attach(bspk_plan *p, int proj_id, const bspk_stdp_triplet_params *tp) {
    if (!p || !tp) return fail(BSPK_ERR_ARG, "null argument");
    // stdp_triplet_synapse.py:152-155
    const double taus[4] = {tp->tau_plus, tp->tau_plus_triplet, tp->tau_minus, tp->tau_minus_triplet};
    const char *names[4] = {"tau_plus", "tau_plus_triplet", "tau_minus", "tau_minus_triplet"};
    for (int i = 0; i < 4; ++i)
        if (!(taus[i] > 0)) return fail(BSPK_ERR_ARG, std::string("'") + names[i] + "' must be > 0.");
    int rc = plastic_checks(p, proj_id);
    if (rc) return rc;
    Proj &J = p->projs[proj_id];
    J.plastic = true;
    J.homogeneous = false;
    J.rule = 1;
    J.trip = *tp;
    return BSPK_OK;
}

int bspk_kernel_fixed_indegree(uint32_t seed, uint32_t proj_hi, uint32_t proj_lo, int n_parts,
                               const uint32_t *part_hi, const uint32_t *part_lo,
                               const int64_t *part_len, const int64_t *post_local,
                               const int64_t *self_pos, int64_t n_pre, int K, int32_t *src_pos) {
    if (n_parts < 0 || K < 0 || n_pre < 0 || (n_parts > 0 && (!part_hi || !part_lo || !part_len)))
        return fail(BSPK_ERR_ARG, "bad arguments");
    int64_t n_post = 0;
    for (int q = 0; q < n_parts; ++q) {
        if (part_len[q] < 0) return fail(BSPK_ERR_ARG, "negative part length");
        n_post += part_len[q];
    }
    if (n_post == 0 || K == 0) return BSPK_OK;
    if (!post_local || !src_pos) return fail(BSPK_ERR_ARG, "null arrays");
    for (int64_t j = 0; j < n_post; ++j) {
        if (post_local[j] < 0 || (post_local[j] >> 10) > 0xFFFFFFFFll)
            return fail(BSPK_ERR_ARG, "post ids must be non-negative and their blocks < 2^32");
        const int64_t sp = self_pos ? self_pos[j] : -1;
        if (sp >= n_pre) return fail(BSPK_ERR_ARG, "self position outside the pre view");
        if (n_pre - (sp >= 0 ? 1 : 0) <= 0)
            return fail(BSPK_ERR_ARG, "fixed_indegree: a target has no available source");
    }
    // object key: fold_in(fold_in(PRNGKey(seed), hi), lo) of the projection name
    const JaxKey obj = jax_fold(jax_fold(jax_key(static_cast<int64_t>(seed)), proj_hi), proj_lo);
    std::vector<int64_t> first(n_parts + 1, 0);
    for (int q = 0; q < n_parts; ++q) first[q + 1] = first[q] + part_len[q];
    unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n_post * K < 200000) nth = 1;
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < nth; ++t) {
        ts.emplace_back([=, &first]() {
            std::vector<int64_t> idx(K);
            for (int q = 0; q < n_parts; ++q) {
                const JaxKey pk = jax_fold(jax_fold(obj, part_hi[q]), part_lo[q]);
                for (int64_t j = first[q] + t; j < first[q + 1]; j += nth) {
                    const uint64_t l = static_cast<uint64_t>(post_local[j]);
                    const JaxKey kj = jax_fold(jax_fold(jax_fold(pk, static_cast<uint32_t>(l >> 10)),
                                                        0xFFFFFFFFu),
                                               static_cast<uint32_t>(l & 1023u));
                    const int64_t sp = self_pos ? self_pos[j] : -1;
                    const uint64_t avail = static_cast<uint64_t>(n_pre - (sp >= 0 ? 1 : 0));
                    jax_randint_span(kj, K, avail, 32, idx.data());
                    for (int k = 0; k < K; ++k) {
                        int64_t c = idx[k];
                        if (sp >= 0 && c >= sp) c += 1;  // skip the post neuron itself
                        src_pos[j * K + k] = static_cast<int32_t>(c);
                    }
                }
            }
        });
    }
    for (auto &th : ts) th.join();
    return BSPK_OK;
}

int bspk_plan_set_ports(bspk_plan *p, int separate) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (p->uploaded || !p->input_kind.empty())
        return fail(BSPK_ERR_STATE, "set the ports before adding inputs");
    if (separate && p->cfg.model != BSPK_IAF_PSC_ALPHA && p->cfg.model != BSPK_IAF_PSC_EXP)
        return fail(BSPK_ERR_UNSUPPORTED, "separate ports are for the iaf_psc models");
    if (separate && p->cfg.deterministic)
        return fail(BSPK_ERR_UNSUPPORTED, "separate ports are not available in deterministic mode");
    p->ports_sep = separate ? 1 : 0;
    return BSPK_OK;
}

int bspk_debug_withhold_record(bspk_plan *p, int cta, int window) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (!p->uploaded) return fail(BSPK_ERR_STATE, "plan not uploaded");
    if (!p->tiled) return fail(BSPK_ERR_UNSUPPORTED, "the record hook needs a plan on the tiled path");
    if (cta < 0 || cta >= p->grid || window < 0)
        return fail(BSPK_ERR_ARG, "cta must be in [0, grid) and window >= 0");
    p->hold_cta = cta;
    p->hold_win = window;
    return BSPK_OK;
}

int bspk_record_v(bspk_plan *p, int n, const int32_t *gids) {
    if (!p || n < 0 || (n > 0 && !gids)) return fail(BSPK_ERR_ARG, "bad record list");
    for (int i = 0; i < n; ++i)
        if (gids[i] < 0 || gids[i] >= p->N) return fail(BSPK_ERR_ARG, "record gid out of range");
    p->rec_v.assign(gids, gids + n);
    if (p->uploaded) {
        std::vector<int32_t> slot(p->N, -1);
        for (int i = 0; i < n; ++i) slot[gids[i]] = i;
        BSPK_CUDA(cudaSetDevice(p->cfg.device));
        BSPK_CUDA(cudaMemcpy(p->d_rec_slot, slot.data(), sizeof(int32_t) * p->N, cudaMemcpyHostToDevice));
    }
    return BSPK_OK;
}

int bspk_record_spikes_of(bspk_plan *p, int n, const int32_t *gids) {
    if (!p || n < 0 || (n > 0 && !gids)) return fail(BSPK_ERR_ARG, "bad record list");
    p->spk_flag.assign(p->N, 0);
    for (int i = 0; i < n; ++i) {
        if (gids[i] < 0 || gids[i] >= p->N) return fail(BSPK_ERR_ARG, "record gid out of range");
        p->spk_flag[gids[i]] = 1;
    }
    p->has_spk_flag = true;
    if (p->uploaded) {
        BSPK_CUDA(cudaSetDevice(p->cfg.device));
        if (!p->d_spk_flag) {
            int rc = dalloc(p, &p->d_spk_flag, p->N);
            if (rc) return rc;
        }
        BSPK_CUDA(cudaMemcpy(p->d_spk_flag, p->spk_flag.data(), p->N, cudaMemcpyHostToDevice));
    }
    return BSPK_OK;
}

}  // extern "C"

// --------------------------------------------------------------- upload

namespace {

template <typename Real>
int upload_projs(bspk_plan *p) {
    const bool exact = p->cfg.deterministic != 0;
    std::vector<ProjDev<Real>> pd;
    for (Proj &J : p->projs) {
        const int npre = p->pops[J.pre].n, npost = p->pops[J.post].n;
        const int64_t E = static_cast<int64_t>(J.post_local.size());
        std::vector<uint32_t> edges(E);
        for (int64_t e = 0; e < E; ++e)
            edges[e] = static_cast<uint32_t>(J.post_local[e]) |
                       (static_cast<uint32_t>(lag_of(p, J.delay[e])) << kEdgeDelayShift);
        {
            J.max_out = 0;
            for (int i = 0; i < npre; ++i)
                J.max_out = std::max<int64_t>(J.max_out, J.indptr[i + 1] - J.indptr[i]);
            std::vector<int64_t> indeg(npost, 0);
            for (int64_t e = 0; e < E; ++e) indeg[J.post_local[e]]++;
            J.max_in = 0;
            for (int64_t d : indeg) J.max_in = std::max(J.max_in, d);
        }
        int rc = upload_vec(p, &J.d_indptr, J.indptr);
        if (!rc) rc = upload_vec(p, &J.d_edges, edges);
        if (rc) return rc;
        if (!J.homogeneous) {
            std::vector<Real> w(E);
            for (int64_t e = 0; e < E; ++e) w[e] = static_cast<Real>(J.w[e]);
            Real *dw = nullptr;
            rc = upload_vec(p, &dw, w);
            if (rc) return rc;
            J.d_w = dw;
        }
        if (J.plastic) {
            rc = upload_vec(p, &J.d_wplastic, J.w);
            if (rc) return rc;
        }
        if (exact || J.plastic) {
            // CSC by post, stable in CSR order (so ascending pre for each post)
            std::vector<int64_t> cptr(npost + 1, 0);
            for (int64_t e = 0; e < E; ++e) cptr[J.post_local[e] + 1]++;
            for (int i = 0; i < npost; ++i) cptr[i + 1] += cptr[i];
            std::vector<int64_t> fill(cptr.begin(), cptr.end() - 1), perm(E);
            std::vector<uint32_t> ced(E);
            std::vector<double> cw(E);
            for (int i = 0; i < npre; ++i)
                for (int64_t e = J.indptr[i]; e < J.indptr[i + 1]; ++e) {
                    const int64_t q = fill[J.post_local[e]]++;
                    ced[q] = static_cast<uint32_t>(i) |
                             (static_cast<uint32_t>(lag_of(p, J.delay[e])) << kEdgeDelayShift);
                    cw[q] = J.w[e];
                    perm[q] = e;
                }
            rc = upload_vec(p, &J.d_cindptr, cptr);
            if (!rc) rc = upload_vec(p, &J.d_cedges, ced);
            if (!rc && !J.homogeneous) rc = upload_vec(p, &J.d_cw, cw);
            if (!rc && J.plastic) rc = upload_vec(p, &J.d_cperm, perm);
            if (rc) return rc;
        }
        if (J.plastic) {
            void *t1 = nullptr, *t2 = nullptr;
            const size_t cols = static_cast<size_t>(J.trace_cols());
            int rc2 = dalloc_bytes(p, &t1, sizeof(double) * npre * cols);
            if (!rc2) rc2 = dalloc_bytes(p, &t2, sizeof(double) * npost * cols);
            if (!rc2) rc2 = dalloc(p, &J.d_pre_list, npre);
            if (!rc2) rc2 = dalloc(p, &J.d_post_list, npost);
            if (rc2) return rc2;
            BSPK_CUDA(cudaMemset(t1, 0, sizeof(double) * npre * cols));
            BSPK_CUDA(cudaMemset(t2, 0, sizeof(double) * npost * cols));
            J.d_pre_trace = t1;
            J.d_post_trace = t2;
        }
        ProjDev<Real> d{};
        d.pre_pop = J.pre;
        d.post_pop = J.post;
        d.post_off = p->pops[J.post].off;
        d.receptor = J.receptor;
        d.homogeneous = J.homogeneous ? 1 : 0;
        d.w0 = static_cast<Real>(J.w0);
        d.indptr = J.d_indptr;
        d.edges = J.d_edges;
        d.w = static_cast<const Real *>(J.d_w);
        d.cindptr = J.d_cindptr;
        d.cedges = J.d_cedges;
        d.cw = J.d_cw;
        pd.push_back(d);
    }
    ProjDev<Real> *dp = nullptr;
    int rc = upload_vec(p, &dp, pd);
    p->d_projs = dp;
    if (rc) return rc;
    std::vector<int> plastic;
    int n_plastic = 0;
    for (auto &J : p->projs) {
        plastic.push_back(J.plastic ? 1 : 0);
        n_plastic += J.plastic ? 1 : 0;
    }
    rc = upload_vec(p, &p->d_proj_plastic, plastic);
    p->n_step_counters = 2 + 2 * n_plastic;
    if (!rc) rc = dalloc(p, &p->d_step_counters, p->n_step_counters);
    if (!rc) rc = dalloc(p, &p->d_step_ptr, 1);
    return rc;
}

template <typename Real>
int upload_coef(bspk_plan *p) {
    std::vector<PopCoef<Real>> c;
    for (auto &P : p->pops) c.push_back(cast_coef<Real>(P.c));
    PopCoef<Real> *dc = nullptr;
    int rc = upload_vec(p, &dc, c);
    p->d_coef = dc;
    return rc;
}

// Per-CTA CSR of the edges that target each tile, for the tiled kernel:
// ptr[c * (N + 1) + pre] .. ptr[c * (N + 1) + pre + 1] into `edges`, edge
// word post_in_tile | lag << 16 | projection << 24, weights in the same
// order when any projection is heterogeneous.  Rows of a CTA are all pre
// neurons, so the bounds of a spike's segment are one shared-memory read.
int build_tiled(bspk_plan *p) {
    const int G = p->grid, tile = p->tile, N = p->N;
    const size_t rows = static_cast<size_t>(G) * (N + 1);
    std::vector<int> ptr(rows + 1, 0);
    bool hetero = false;
    int64_t total = 0;
    for (auto &J : p->projs) {
        hetero |= !J.homogeneous;
        const int pre_off = p->pops[J.pre].off, post_off = p->pops[J.post].off;
        for (int i = 0; i < p->pops[J.pre].n; ++i)
            for (int64_t e = J.indptr[i]; e < J.indptr[i + 1]; ++e) {
                const int c = (post_off + J.post_local[e]) / tile;
                ptr[static_cast<size_t>(c) * (N + 1) + pre_off + i + 1]++;
            }
        total += static_cast<int64_t>(J.post_local.size());
    }
    if (total >= (int64_t(1) << 31)) return fail(BSPK_ERR_UNSUPPORTED, "more than 2^31 edges");
    for (size_t i = 0; i < rows; ++i) ptr[i + 1] += ptr[i];
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    std::vector<uint32_t> edges(total);
    std::vector<double> w(hetero ? total : 0);
    for (size_t j = 0; j < p->projs.size(); ++j) {
        const Proj &J = p->projs[j];
        const int pre_off = p->pops[J.pre].off, post_off = p->pops[J.post].off;
        for (int i = 0; i < p->pops[J.pre].n; ++i)
            for (int64_t e = J.indptr[i]; e < J.indptr[i + 1]; ++e) {
                const int post = post_off + J.post_local[e];
                const int c = post / tile;
                const int q = fill[static_cast<size_t>(c) * (N + 1) + pre_off + i]++;
                edges[q] = static_cast<uint32_t>(post - c * tile) |
                           (static_cast<uint32_t>(lag_of(p, J.delay[e])) << 16) |
                           (static_cast<uint32_t>(j) << 24) |
                           (p->ports_tiled && J.receptor == 1 ? 1u << 15 : 0u);
                if (hetero) w[q] = J.w[e];
            }
    }
    ptr.pop_back();
    int rc = upload_vec(p, &p->d_tptr, ptr);
    if (!rc) rc = upload_vec(p, &p->d_tedges, edges);
    if (rc) return rc;
    // fixed-point scale 2^k of the ring: an edge adds at most once per arrival
    // step, so no slot exceeds the largest per-neuron sum of |w| over in-edges
    std::vector<double> wsum(N, 0.0);
    for (auto &J : p->projs) {
        const int post_off = p->pops[J.post].off;
        for (size_t e = 0; e < J.post_local.size(); ++e)
            wsum[post_off + J.post_local[e]] += std::fabs(J.w[e]);
    }
    const double wmax = *std::max_element(wsum.begin(), wsum.end());
    const double limit = p->elt == 8 ? 4.0e18 : 2.0e9;  // below 2^62 / 2^31
    int k = 40;
    if (wmax > 0.0) k = static_cast<int>(std::floor(std::log2(limit / wmax)));
    k = std::max(-60, std::min(k, p->elt == 8 ? 100 : 60));
    const double scale = std::ldexp(1.0, k);
    p->tinv_scale = std::ldexp(1.0, -k);
    std::vector<int64_t> wproj(std::max<size_t>(p->projs.size(), 1), 0);
    for (size_t j = 0; j < p->projs.size(); ++j) wproj[j] = std::llrint(p->projs[j].w0 * scale);
    if (p->elt == 8) {
        std::vector<long long> f(wproj.begin(), wproj.end());
        long long *d = nullptr;
        rc = upload_vec(p, &d, f);
        p->d_twproj = d;
    } else {
        std::vector<int32_t> f(wproj.begin(), wproj.end());
        int32_t *d = nullptr;
        rc = upload_vec(p, &d, f);
        p->d_twproj = d;
    }
    if (rc) return rc;
    if (hetero) {
        if (p->elt == 8) {
            std::vector<long long> f(w.size());
            for (size_t q = 0; q < w.size(); ++q) f[q] = std::llrint(w[q] * scale);
            long long *dw = nullptr;
            rc = upload_vec(p, &dw, f);
            p->d_tw = dw;
        } else {
            std::vector<int32_t> f(w.size());
            for (size_t q = 0; q < w.size(); ++q) f[q] = static_cast<int32_t>(std::llrint(w[q] * scale));
            int32_t *dw = nullptr;
            rc = upload_vec(p, &dw, f);
            p->d_tw = dw;
        }
        if (rc) return rc;
    }
    p->list_cap = tile * p->tW;
    p->tlist_words = static_cast<size_t>(kRecBufs) * G * kRecWords;
    rc = dalloc(p, &p->d_tlist, p->tlist_words);
    if (!rc) rc = dalloc(p, &p->d_tovf, static_cast<size_t>(kRecBufs) * G * p->list_cap);
    if (!rc) rc = dalloc(p, &p->d_trec, static_cast<size_t>(G));
    if (rc) return rc;
    BSPK_CUDA(cudaMemset(p->d_trec, 0, sizeof(long long) * G));
    return BSPK_OK;
}

// Frees one of the plan's device buffers.
template <typename T>
void dfree(bspk_plan *p, T *&ptr) {
    if (!ptr) return;
    cudaFree(ptr);
    void *raw = static_cast<void *>(ptr);
    p->allocs.erase(std::remove(p->allocs.begin(), p->allocs.end(), raw), p->allocs.end());
    ptr = nullptr;
}

// dynamic shared memory budget of the tiled kernel: 227 KB minus its ~34 KB
// of static arrays
constexpr size_t kTiledBudget = 190 * 1024;

// Whether G CTAs can run the tiled kernel on this plan (tile per CTA within
// the kernel's limits and its shared memory budget).
bool tiled_fits(const bspk_plan *p, int G) {
    if (G < 1 || G > 160 || G > p->sm_count) return false;
    const int tile = (p->N + G - 1) / G;
    return tile <= 256 &&
           lif_tiled_smem(tile, p->L, p->tW, p->N, static_cast<int>(p->pops.size()),
                          static_cast<int>(p->projs.size()), p->elt == 8, false,
                          p->ports_tiled != 0) <= kTiledBudget;
}

// The tiled path's per-CTA structures rebuilt for G CTAs.
int retile(bspk_plan *p, int G) {
    dfree(p, p->d_tptr);
    dfree(p, p->d_tedges);
    dfree(p, p->d_tw);
    dfree(p, p->d_twproj);
    dfree(p, p->d_tlist);
    dfree(p, p->d_tovf);
    dfree(p, p->d_trec);
    p->grid = G;
    p->tile = (p->N + G - 1) / G;
    const int rc = build_tiled(p);
    if (rc) return rc;
    p->smem_ptr = lif_tiled_smem(p->tile, p->L, p->tW, p->N, static_cast<int>(p->pops.size()),
                                 static_cast<int>(p->projs.size()), p->elt == 8, true,
                                 p->ports_tiled != 0) <= kTiledBudget;
    p->cspk_valid = false;
    p->pref_step0 = -1;
    return BSPK_OK;
}

}  // namespace

// Buffers of the windowed engine (see WinDev).
static int alloc_window(bspk_plan *p) {
    const Proj *J = nullptr;
    for (const auto &q : p->projs)
        if (q.plastic) J = &q;
    const size_t W = p->W;
    const size_t npre = J ? p->pops[J->pre].n : 1, npost = J ? p->pops[J->post].n : 1;
    const size_t E = J ? std::max<size_t>(J->post_local.size(), 1) : 1;
    const size_t cap = J ? p->win_cap : 1;
    int rc = dalloc(p, &p->d_win_kp, W * npre);
    if (!rc) rc = dalloc(p, &p->d_win_amask, npre);
    if (!rc) rc = dalloc(p, &p->d_win_arr, W * cap * npost);
    if (!rc) rc = dalloc(p, &p->d_win_cnt, W * npost);
    if (!rc) rc = dalloc(p, &p->d_win_spk, W * static_cast<size_t>(p->N));
    if (!rc) rc = dalloc(p, &p->d_win_pre, 2 * npre);
    if (!rc) rc = dalloc(p, &p->d_win_post, 2 * npost);
    if (!rc) rc = dalloc(p, &p->d_win_ctr, 4);
    if (rc) return rc;
    BSPK_CUDA(cudaMemset(p->d_win_amask, 0, sizeof(uint32_t) * npre));
    BSPK_CUDA(cudaMemset(p->d_win_cnt, 0, sizeof(int) * W * npost));
    return BSPK_OK;
}

extern "C" int bspk_plan_upload(bspk_plan *p, void *stream) {
    (void)stream;
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (p->uploaded) return fail(BSPK_ERR_STATE, "plan already uploaded");
    if (p->N == 0) return fail(BSPK_ERR_ARG, "plan has no neurons");
    BSPK_CUDA(cudaSetDevice(p->cfg.device));
    cudaDeviceProp prop;
    BSPK_CUDA(cudaGetDeviceProperties(&prop, p->cfg.device));
    p->sm_count = prop.multiProcessorCount;
    const bool dbl = p->cfg.precision == 64;
    const bool exact = p->cfg.deterministic != 0;
    bool plastic = false;
    for (auto &J : p->projs) plastic |= J.plastic;
    // separate receptor ports of the iaf models run on the tiled kernel (one
    // ring per port) when it takes the network and every drive feeds 'ex';
    // otherwise on the per-step engine
    p->ports_tiled = 0;
    if (p->ports_sep && !model_per_step(p->cfg.model) && !exact && !plastic) {
        bool drives0 = true;
        for (auto &D : p->drives) drives0 &= D.receptor == 0;
        p->ports_tiled = drives0 ? 1 : 0;  // confirmed below once the geometry is known
    }

    // window and ring length
    int min_lag = 1 << 30, max_lag = 0;
    for (auto &J : p->projs)
        for (int32_t d : J.delay) {
            const int lag = lag_of(p, d);
            min_lag = std::min(min_lag, lag);
            max_lag = std::max(max_lag, lag);
        }
    if (p->projs.empty() || max_lag == 0) min_lag = kMaxWindow;
    p->max_lag = max_lag;
    p->W = std::max(1, std::min(min_lag, kMaxWindow));
    if (exact) {
        if (max_lag + 1 > 63) return fail(BSPK_ERR_UNSUPPORTED, "deterministic mode needs lags <= 62 steps");
        p->W = std::max(1, std::min(p->W, 64 - max_lag));
    }
    if (p->ports_tiled) {
        // the tiled geometry (as below) must fit, else the per-step engine
        const int grid = std::max(1, std::min(p->sm_count, (p->N + 31) / 32));
        const int tile = (p->N + grid - 1) / grid;
        const int L = p->W + max_lag + 1;
        if (!(tile <= 256 && grid <= 160 &&
              lif_tiled_smem(tile, L, p->W, p->N, static_cast<int>(p->pops.size()),
                             static_cast<int>(p->projs.size()), dbl, false, true) <= kTiledBudget))
            p->ports_tiled = 0;
    }
    const bool aeif = plan_per_step(p);  // per-step engine (RKF45, multisynapse, ports)
    p->win = false;
    if (aeif || plastic) {
        // windowed form when every lag allows W >= 2 steps per launch, the
        // window and the lags fit in the 64-step spike history, and at most
        // one pair-rule projection with one lag is plastic; its arrival
        // lists (W x max in-degree x posts) must stay within 16 GB
        int n_pl = 0;
        bool pl_ok = true;
        size_t arr_bytes = 0;
        const int Ww = std::min({min_lag, 32, 64 - max_lag});
        for (auto &J : p->projs) {
            if (!J.plastic) continue;
            ++n_pl;
            pl_ok = pl_ok && J.rule == 0 && J.post_local.size() < (size_t(1) << 32);
            for (int32_t d : J.delay) pl_ok = pl_ok && d == J.delay[0];
            std::vector<int64_t> indeg(p->pops[J.post].n, 0);
            for (int32_t q : J.post_local) indeg[q]++;
            const int64_t mx = indeg.empty() ? 0 : *std::max_element(indeg.begin(), indeg.end());
            arr_bytes = static_cast<size_t>(std::max(Ww, 1)) * std::max<int64_t>(mx, 1) *
                        p->pops[J.post].n * sizeof(WinArrival);
            p->win_cap = static_cast<int>(std::max<int64_t>(mx, 1));
        }
        p->win = p->win_ok = Ww >= 2 && n_pl <= 1 && pl_ok && arr_bytes <= (size_t(16) << 30);
        p->W = p->win ? Ww : 1;
    }
    p->L = p->W + max_lag + 1;

    // state
    const int ns = n_state_slots(p->cfg.model);
    for (int i = 0; i < 9; ++i) p->d_s[i] = nullptr;
    std::vector<double> init(p->N, 0.0);
    for (int i = 0; i < ns; ++i) {
        int rc = dalloc_bytes(p, &p->d_s[i], static_cast<size_t>(p->elt) * p->N);
        if (rc) return rc;
    }
    int rc = dalloc(p, &p->d_r, p->N);
    if (rc) return rc;
    BSPK_CUDA(cudaMemset(p->d_r, 0, sizeof(int) * p->N));
    for (int i = 0; i < ns; ++i) {
        for (auto &P : p->pops)
            for (int k = 0; k < P.n; ++k) {
                double v = 0.0;
                // V_m: E_L for the iaf and AdEx models; the iaf_cond models'
                // V_initializer is a constant -70 mV (iaf_cond_exp.py:310)
                if (i == 0) v = (p->cfg.model == BSPK_IAF_COND_EXP || p->cfg.model == BSPK_IAF_COND_ALPHA ||
                                 p->cfg.model == BSPK_IAF_PSC_EXP_MULTISYNAPSE)
                                    ? -70.0
                                    : P.c.E_L;
                if (model_is_cond(p->cfg.model) && i == cond_n_ode(p->cfg.model))
                    v = p->cfg.dt;  // integration_step = dt
                init[P.off + k] = v;
            }
        if (dbl) {
            BSPK_CUDA(cudaMemcpy(p->d_s[i], init.data(), 8 * p->N, cudaMemcpyHostToDevice));
        } else {
            std::vector<float> f(init.begin(), init.end());
            BSPK_CUDA(cudaMemcpy(p->d_s[i], f.data(), 4 * p->N, cudaMemcpyHostToDevice));
        }
    }
    // ring: [L][R][N], R = 2 for conductance models
    const int R = plan_n_receptors(p);
    const size_t ring_bytes = static_cast<size_t>(p->elt) * p->L * R * p->N;
    rc = dalloc_bytes(p, &p->d_ring, ring_bytes);
    if (rc) return rc;
    BSPK_CUDA(cudaMemset(p->d_ring, 0, ring_bytes));
    rc = dalloc(p, &p->d_hist, p->N);
    if (rc) return rc;
    BSPK_CUDA(cudaMemset(p->d_hist, 0, sizeof(uint64_t) * p->N));

    rc = dbl ? upload_coef<double>(p) : upload_coef<float>(p);
    if (!rc) rc = dbl ? upload_projs<double>(p) : upload_projs<float>(p);
    if (!rc && p->win) rc = alloc_window(p);
    if (rc) return rc;

    // drives and CDF tables
    std::vector<DriveDev> dd;
    // CDF tables as integer thresholds floor(F * 2^53): for a 53-bit uniform
    // b * 2^-53, u <= F[k] holds exactly when b <= floor(F[k] * 2^53).
    std::vector<uint64_t> cdf;
    for (auto &D : p->drives) {
        DriveDev d{};
        d.pop = D.post;
        d.lag = D.lag;
        d.seed = D.seed;
        d.cdf_off = static_cast<int>(cdf.size());
        d.receptor = D.receptor;
        d.weight = D.weight;
        d.tmin = D.tmin;
        d.tmax = D.tmax;
        d.kind = D.kind;
        d.key0 = D.key0;
        d.key1 = D.key1;
        d.unit_off = D.unit_off;
        d.trial = p->trial;
        if (D.kind == 1) {
            d.cdf_n = static_cast<int>(D.thr.size());
            cdf.insert(cdf.end(), D.thr.begin(), D.thr.end());
        } else {
            d.cdf_n = static_cast<int>(D.cdf.size());
            for (double F : D.cdf) cdf.push_back(static_cast<uint64_t>(std::floor(std::ldexp(F, 53))));
        }
        dd.push_back(d);
    }
    p->cdf_total = static_cast<int>(cdf.size());
    rc = upload_vec(p, &p->d_drives, dd);
    if (!rc) rc = upload_vec(p, &p->d_cdf, cdf);
    if (rc) return rc;
    // adjacency lists per population
    const int npop = static_cast<int>(p->pops.size());
    std::vector<int> out_ptr(npop + 1, 0), out_list, in_ptr(npop + 1, 0), in_list,
        dr_ptr(npop + 1, 0), dr_list;
    for (int q = 0; q < npop; ++q) {
        for (size_t j = 0; j < p->projs.size(); ++j)
            if (p->projs[j].pre == q && !p->projs[j].plastic) out_list.push_back(static_cast<int>(j));
        out_ptr[q + 1] = static_cast<int>(out_list.size());
        for (int id : p->input_kind) {
            const int post = id >= 0 ? p->projs[id].post : p->drives[-id - 1].post;
            if (post == q) in_list.push_back(id);
        }
        in_ptr[q + 1] = static_cast<int>(in_list.size());
        for (size_t j = 0; j < p->drives.size(); ++j)
            if (p->drives[j].post == q) dr_list.push_back(static_cast<int>(j));
        dr_ptr[q + 1] = static_cast<int>(dr_list.size());
    }
    rc = upload_vec(p, &p->d_pop_out_ptr, out_ptr);
    if (!rc) rc = upload_vec(p, &p->d_pop_out_list, out_list);
    if (!rc) rc = upload_vec(p, &p->d_pop_in_ptr, in_ptr);
    if (!rc) rc = upload_vec(p, &p->d_pop_in_list, in_list);
    if (!rc) rc = upload_vec(p, &p->d_pop_drive_ptr, dr_ptr);
    if (!rc) rc = upload_vec(p, &p->d_pop_drive_list, dr_list);
    if (rc) return rc;

    // recording
    rc = dalloc(p, &p->d_spk_step, p->cfg.spike_capacity);
    if (!rc) rc = dalloc(p, &p->d_spk_gid, p->cfg.spike_capacity);
    if (!rc) rc = dalloc(p, &p->d_spk_count, 1);
    if (!rc) rc = dalloc(p, &p->d_rec_slot, p->N);
    if (!rc) rc = dalloc(p, &p->d_barrier, 1);
    if (!rc) rc = dalloc(p, &p->d_err, 1);
    if (!rc) rc = dalloc(p, &p->d_step_spk, p->N);
    if (!rc) rc = dalloc(p, &p->d_step_nspk, 1);
    if (!rc) rc = dalloc(p, &p->d_rk_iters, 1);
    if (rc) return rc;
    BSPK_CUDA(cudaMemset(p->d_spk_count, 0, sizeof(unsigned long long)));
    BSPK_CUDA(cudaMemset(p->d_err, 0, sizeof(int)));
    BSPK_CUDA(cudaMemset(p->d_rk_iters, 0, sizeof(unsigned long long)));
    {
        std::vector<int32_t> slot(p->N, -1);
        for (size_t i = 0; i < p->rec_v.size(); ++i) slot[p->rec_v[i]] = static_cast<int32_t>(i);
        BSPK_CUDA(cudaMemcpy(p->d_rec_slot, slot.data(), sizeof(int32_t) * p->N, cudaMemcpyHostToDevice));
    }
    if (p->has_spk_flag) {
        rc = dalloc(p, &p->d_spk_flag, p->N);
        if (rc) return rc;
        BSPK_CUDA(cudaMemcpy(p->d_spk_flag, p->spk_flag.data(), p->N, cudaMemcpyHostToDevice));
    }
    BSPK_CUDA(cudaEventCreate(&p->ev0));
    BSPK_CUDA(cudaEventCreate(&p->ev1));

    // launch geometry of the persistent kernels: one CTA per SM when the
    // network is small, so every SM takes part in delivery.
    if (exact) {
        int block = ((p->N + p->sm_count - 1) / p->sm_count + 31) / 32 * 32;
        block = std::max(64, std::min(block, 256));
        p->block = block;
        p->grid = (p->N + block - 1) / block;
        p->tile = block;
    } else {
        // fast path: one 256-thread CTA per SM, a contiguous tile of neurons each
        p->block = 256;
        p->grid = std::max(1, std::min(p->sm_count, (p->N + 31) / 32));
        p->tile = (p->N + p->grid - 1) / p->grid;
        // (the per-step engine, windowed or not, keeps no tile in shared memory)
        if (!(aeif || plastic) && static_cast<size_t>(p->tile) * p->W * 4 > 160 * 1024)
            return fail(BSPK_ERR_UNSUPPORTED, "network too large for the persistent kernel tile");
    }
    for (auto &J : p->projs)
        if (J.post_local.size() >= (size_t(1) << 31))
            return fail(BSPK_ERR_UNSUPPORTED, "projection with >= 2^31 edges");
    // tiled (target-partitioned) path: state in registers, ring in shared memory
    // the tiled kernel delivers a window one iteration late when every lag is
    // at least 2 W (W is capped at kMaxWindow, so only long delays allow it);
    // halving W to get there costs more in per-window latency than it saves
    p->tiled = false;
    p->tW = p->W;
    p->tpipe = min_lag >= 2 * p->W ? 1 : 0;
    const int nproj_t = static_cast<int>(p->projs.size());
    const size_t tiled_budget = kTiledBudget;
    const bool two = p->ports_tiled != 0;
    if (!exact && !aeif && !plastic && p->tile <= 256 && p->grid <= 160 &&
        lif_tiled_smem(p->tile, p->L, p->tW, p->N, npop, nproj_t, dbl, false, two) <= tiled_budget) {
        rc = build_tiled(p);
        if (rc) return rc;
        p->tiled = true;
        p->smem_ptr =
            lif_tiled_smem(p->tile, p->L, p->tW, p->N, npop, nproj_t, dbl, true, two) <= tiled_budget;
    }
    if (two && !p->tiled) return fail(BSPK_ERR_CUDA, "separate ports: tiled geometry check differs");
    p->uploaded = true;
    p->step = 0;
    return BSPK_OK;
}

// ------------------------------------------------------------------ run

namespace {

template <typename Real>
LifArgs<Real> lif_args(bspk_plan *p, int64_t n_steps) {
    LifArgs<Real> a{};
    a.N = p->N;
    a.npop = static_cast<int>(p->pops.size());
    a.nproj = static_cast<int>(p->projs.size());
    a.ndrive = static_cast<int>(p->drives.size());
    a.coef = static_cast<const PopCoef<Real> *>(p->d_coef);
    for (int i = 0; i < 6; ++i) a.s[i] = static_cast<Real *>(p->d_s[i]);
    a.r = p->d_r;
    a.ring = static_cast<Real *>(p->d_ring);
    a.L = p->L;
    a.projs = static_cast<const ProjDev<Real> *>(p->d_projs);
    a.pop_out_ptr = p->d_pop_out_ptr;
    a.pop_out_list = p->d_pop_out_list;
    a.pop_in_ptr = p->d_pop_in_ptr;
    a.pop_in_list = p->d_pop_in_list;
    a.drives = p->d_drives;
    a.pop_drive_ptr = p->d_pop_drive_ptr;
    a.pop_drive_list = p->d_pop_drive_list;
    a.cdf = p->d_cdf;
    a.cdf_total = p->cdf_total;
    a.step0 = p->step;
    a.n_steps = n_steps;
    a.run_step0 = p->step;
    a.W = p->W;
    a.tile = p->tile;
    a.model = p->cfg.model;
    a.spk_step = p->d_spk_step;
    a.spk_gid = p->d_spk_gid;
    a.spk_count = p->d_spk_count;
    a.spk_cap = p->cfg.spike_capacity;
    a.spk_flag = p->has_spk_flag ? p->d_spk_flag : nullptr;
    a.rec_slot = p->rec_v.empty() ? nullptr : p->d_rec_slot;
    a.v_out = static_cast<Real *>(p->d_v);
    a.n_rec = static_cast<int>(p->rec_v.size());
    a.hist = p->d_hist;
    a.barrier = p->d_barrier;
    a.err = p->d_err;
    return a;
}


// Tiled path: the run in launches of at most kDriveBudget bytes of drive;
// each launch is a drive pass over (step, neuron) then the persistent kernel,
// with freshly zeroed records (window tags restart per launch).
constexpr size_t kDriveBudget = size_t(512) << 20;

template <typename Real>
int run_tiled(bspk_plan *p, int64_t n_steps, cudaStream_t st) {
    const size_t per_step = sizeof(Real) * static_cast<size_t>(p->N);
    int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_steps, kDriveBudget / per_step));
    if (p->drive_chunk > 0) chunk = std::min<int64_t>(chunk, p->drive_chunk);
    if (p->tdrive_steps < chunk) {
        for (void **b : {&p->d_tdrive, &p->d_tdrive2}) {
            if (*b) {
                cudaFree(*b);
                p->allocs.erase(std::remove(p->allocs.begin(), p->allocs.end(), *b), p->allocs.end());
                *b = nullptr;
            }
            int rc = dalloc_bytes(p, b, per_step * chunk);
            if (rc) return rc;
        }
        p->tdrive_steps = chunk;
        p->pref_step0 = -1;
    }
    if (p->drive_overlap && !p->side) {
        BSPK_CUDA(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
        BSPK_CUDA(cudaEventCreateWithFlags(&p->ev_side, cudaEventDisableTiming));
        BSPK_CUDA(cudaEventCreateWithFlags(&p->ev_main, cudaEventDisableTiming));
    }
    // the record area for the chosen copies and stride
    const size_t rec_words = static_cast<size_t>(kRecBufs) * p->rec_rep * p->grid * p->rec_stride;
    if (rec_words > p->tlist_words) {
        cudaFree(p->d_tlist);
        p->allocs.erase(std::remove(p->allocs.begin(), p->allocs.end(), p->d_tlist), p->allocs.end());
        p->d_tlist = nullptr;
        int rc = dalloc(p, &p->d_tlist, rec_words);
        if (rc) return rc;
        p->tlist_words = rec_words;
    }
    void *bufs[2] = {p->d_tdrive, p->d_tdrive2};
    // a prefill issued by the previous run may still be writing a buffer if
    // this run comes on another stream
    if (p->side) BSPK_CUDA(cudaStreamWaitEvent(st, p->ev_side, 0));
    const int64_t run0 = p->step;
    // a run from a restored checkpoint is likely to be repeated from there
    // (Runner.simulate): then the prefill after its last launch draws the
    // drive of that step again instead of the continuation's
    const bool restart = p->restart_step == run0;
    if (!restart) p->restart_step = -1;
    int64_t launches = 0;
    for (int64_t done = 0; done < n_steps; done += chunk) {
        const int64_t n = std::min<int64_t>(chunk, n_steps - done);
        LifArgs<Real> a = lif_args<Real>(p, n);
        a.step0 = run0 + done;
        a.run_step0 = run0;
        a.W = p->tW;
        a.pipe = p->tpipe;
        // this launch's drive: prefilled beside the previous launch, or now
        int cur = 0;
        if (p->drive_overlap && p->pref_step0 == a.step0 && p->pref_n >= n) {
            cur = p->pref_buf;
            BSPK_CUDA(cudaStreamWaitEvent(st, p->ev_side, 0));
        } else {
            cudaError_t e = launch_drive_fill<Real>(a, a.step0, static_cast<int>(n),
                                                    static_cast<Real *>(bufs[cur]), st);
            if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("drive launch: ") + cudaGetErrorString(e));
            ++launches;
        }
        p->pref_step0 = -1;
        BSPK_CUDA(cudaMemsetAsync(p->d_tlist, 0, sizeof(uint32_t) * rec_words, st));
        BSPK_CUDA(cudaMemsetAsync(p->d_tovf, 0,
                                  sizeof(uint32_t) * kRecBufs * static_cast<size_t>(p->grid) * p->list_cap, st));
        using Fix = typename FixOf<Real>::type;
        TiledArgs<Real> t2{p->d_tptr, p->d_tedges, static_cast<const Fix *>(p->d_tw),
                           static_cast<const Fix *>(p->d_twproj), static_cast<Real>(p->tinv_scale),
                           p->d_tlist, p->d_tovf, p->d_trec, p->list_cap, p->smem_ptr ? 1 : 0,
                           static_cast<const Real *>(bufs[cur]), a.step0,
                           done == 0 ? p->hold_cta : -1, done == 0 ? p->hold_win : -1,
                           p->ports_tiled, p->rec_rep, p->rec_stride, p->poll_pause};
        // ev_main marks the end of everything before this launch (the last
        // reader of the other buffer); the persistent kernel is submitted
        // first so that its CTAs take their SMs before the side blocks do
        if (p->drive_overlap) BSPK_CUDA(cudaEventRecord(p->ev_main, st));
        cudaError_t e = launch_lif_tiled<Real>(a, t2, p->grid, st);
        if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
        ++launches;
        if (p->drive_overlap) {
            // the drive of the steps after this launch (the next launch, or as
            // many steps after the run), into the other buffer, once every
            // launch enqueued so far (the last reader of that buffer) is done
            const bool last = done + n >= n_steps;
            const int64_t next0 = last && restart ? run0 : a.step0 + n;
            const int64_t nn = !last ? std::min<int64_t>(chunk, n_steps - done - n)
                                     : (restart ? std::min<int64_t>(chunk, n_steps) : n);
            if (next0 + nn < (int64_t(1) << 32)) {
                BSPK_CUDA(cudaStreamWaitEvent(p->side, p->ev_main, 0));
                LifArgs<Real> b = lif_args<Real>(p, nn);
                cudaError_t e = launch_drive_fill<Real>(b, next0, static_cast<int>(nn),
                                                        static_cast<Real *>(bufs[cur ^ 1]), p->side,
                                                        true);
                if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("drive launch: ") + cudaGetErrorString(e));
                BSPK_CUDA(cudaEventRecord(p->ev_side, p->side));
                p->pref_step0 = next0;
                p->pref_n = nn;
                p->pref_buf = cur ^ 1;
                ++launches;
            }
        }
    }
    // the side stream's last prefill completes within this run's stream order
    if (p->drive_overlap && p->pref_step0 >= 0) BSPK_CUDA(cudaStreamWaitEvent(st, p->ev_side, 0));
    p->hold_cta = p->hold_win = -1;  // the test hook covers one run
    p->last_launches = launches;
    return BSPK_OK;
}

}  // namespace

extern "C" int bspk_run(bspk_plan *p, int64_t n_steps, void *stream) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (!p->uploaded) return fail(BSPK_ERR_STATE, "plan not uploaded");
    if (n_steps < 0) return fail(BSPK_ERR_ARG, "n_steps must be >= 0");
    if (p->step + n_steps >= (int64_t(1) << 32))
        return fail(BSPK_ERR_UNSUPPORTED, "step counter beyond 2^32 (RNG counter width)");
    BSPK_CUDA(cudaSetDevice(p->cfg.device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // V recording buffer for this run
    const size_t vbytes = static_cast<size_t>(p->elt) * n_steps * p->rec_v.size();
    if (!p->rec_v.empty() && n_steps > p->v_steps_cap) {
        if (p->d_v) {
            cudaFree(p->d_v);
            p->allocs.erase(std::remove(p->allocs.begin(), p->allocs.end(), p->d_v), p->allocs.end());
            p->d_v = nullptr;
        }
        int rc = dalloc_bytes(p, &p->d_v, vbytes);
        if (rc) return rc;
        p->v_steps_cap = n_steps;
    }
    BSPK_CUDA(cudaMemsetAsync(p->d_spk_count, 0, sizeof(unsigned long long), st));
    BSPK_CUDA(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
    p->last_run_steps = n_steps;
    p->cspk_valid = false;
    if (n_steps == 0) return BSPK_OK;
    const bool dbl = p->cfg.precision == 64;
    BSPK_CUDA(cudaMemsetAsync(p->d_barrier, 0, sizeof(unsigned int), st));
    BSPK_CUDA(cudaEventRecord(p->ev0, st));
    cudaError_t e = cudaSuccess;
    bool per_step = plan_per_step(p);
    for (auto &J : p->projs) per_step |= J.plastic;
    if (p->tiled) BSPK_CUDA(cudaMemsetAsync(p->d_trec, 0, sizeof(long long) * p->grid, st));
    for (auto &J : p->projs) {
        if (!J.rec_w) continue;
        const int64_t need = n_steps * static_cast<int64_t>(J.post_local.size());
        if (need > J.wtrace_cap) {
            if (J.d_wtrace) {
                cudaFree(J.d_wtrace);
                p->allocs.erase(std::remove(p->allocs.begin(), p->allocs.end(), J.d_wtrace),
                                p->allocs.end());
                J.d_wtrace = nullptr;
            }
            int rc = dalloc(p, &J.d_wtrace, need);
            if (rc) return rc;
            J.wtrace_cap = need;
        }
        J.wtrace_steps = n_steps;
    }
    if (per_step) {
        int rc = run_per_step(p, n_steps, st);
        if (rc) return rc;
    } else if (p->cfg.deterministic) {
        LifArgs<double> a = lif_args<double>(p, n_steps);
        e = launch_lif_exact(a, p->grid, p->block, st);
        p->last_launches = 1;
    } else if (p->tiled) {
        int rc = dbl ? run_tiled<double>(p, n_steps, st) : run_tiled<float>(p, n_steps, st);
        if (rc) return rc;
    } else if (dbl) {
        LifArgs<double> a = lif_args<double>(p, n_steps);
        e = launch_lif_fast<double>(a, p->grid, p->block, st);
        p->last_launches = 1;
    } else {
        LifArgs<float> a = lif_args<float>(p, n_steps);
        e = launch_lif_fast<float>(a, p->grid, p->block, st);
        p->last_launches = 1;
    }
    if (e != cudaSuccess) return fail(BSPK_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    BSPK_CUDA(cudaEventRecord(p->ev1, st));
    p->step += n_steps;
    return BSPK_OK;
}

int bspk::plan_stage(bspk_plan *p, size_t bytes) {
    if (p->h_stage_bytes >= bytes) return BSPK_OK;
    if (p->h_stage) cudaFreeHost(p->h_stage);
    p->h_stage = nullptr;
    p->h_stage_bytes = 0;
    BSPK_CUDA(cudaMallocHost(&p->h_stage, bytes));
    p->h_stage_bytes = bytes;
    return BSPK_OK;
}

int bspk::sync_and_check(bspk_plan *p) {
    BSPK_CUDA(cudaSetDevice(p->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    int err = 0;
    BSPK_CUDA(cudaMemcpy(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err == BSPK_DEV_ERR_TIMEOUT) return fail(BSPK_ERR_TIMEOUT, "device barrier timed out");
    if (err == BSPK_DEV_ERR_UNSTABLE)
        return fail(BSPK_ERR_UNSTABLE, p->cfg.model == BSPK_IAF_COND_EXP
                                           ? "Numerical instability in iaf_cond_exp dynamics."
                                           : "Numerical instability in aeif_cond_alpha dynamics.");
    if (err == BSPK_DEV_ERR_RKCAP) return fail(BSPK_ERR_RKCAP, "RKF45 iteration cap reached");
    if (err == BSPK_DEV_ERR_BOUNDS) return fail(BSPK_ERR_ARG, "device bounds check failed");
    if (err == BSPK_DEV_ERR_OVERFLOW) return fail(BSPK_ERR_OVERFLOW, "device list overflow");
    if (err) return fail(BSPK_ERR_CUDA, "device error flag " + std::to_string(err));
    return BSPK_OK;
}


extern "C" {

int bspk_spikes_get(bspk_plan *p, int64_t cap, int64_t *steps, int32_t *gids, int64_t *n_out) {
    if (!p || !p->uploaded || !n_out) return fail(BSPK_ERR_ARG, "bad arguments");
    int rc = sync_and_check(p);
    if (rc) return rc;
    if (p->tiled) {
        // per-CTA regions of spike_capacity / G entries each
        const int G = p->grid;
        const int64_t region = p->cfg.spike_capacity / G;
        std::vector<long long> counts(G);
        BSPK_CUDA(cudaMemcpy(counts.data(), p->d_trec, sizeof(long long) * G, cudaMemcpyDeviceToHost));
        int64_t total = 0;
        for (int c = 0; c < G; ++c) {
            total += counts[c];
            if (counts[c] > region) {
                *n_out = total;
                return fail(BSPK_ERR_OVERFLOW, "spike record overflowed its device capacity");
            }
        }
        if (!p->cspk_valid) {
            if (!p->d_cspk_step) {
                int rc2 = dalloc(p, &p->d_cspk_step, static_cast<size_t>(p->cfg.spike_capacity));
                if (!rc2) rc2 = dalloc(p, &p->d_cspk_gid, static_cast<size_t>(p->cfg.spike_capacity));
                if (!rc2) rc2 = dalloc(p, &p->d_cspk_n, 1);
                if (rc2) return rc2;
            }
            BSPK_CUDA(cudaMemset(p->d_cspk_n, 0, sizeof(unsigned long long)));
            BSPK_CUDA(launch_compact_spikes(G, region, p->d_trec, p->d_spk_step, p->d_spk_gid,
                                            p->d_cspk_step, p->d_cspk_gid, p->d_cspk_n, nullptr));
            unsigned long long n = 0;
            BSPK_CUDA(cudaMemcpy(&n, p->d_cspk_n, sizeof(n), cudaMemcpyDeviceToHost));
            p->cspk_n = static_cast<int64_t>(n);
            p->cspk_valid = true;
        }
        const int64_t k = std::min<int64_t>(cap, p->cspk_n);
        if (k > 0 && steps && gids) {
            BSPK_CUDA(cudaMemcpy(steps, p->d_cspk_step, 8 * k, cudaMemcpyDeviceToHost));
            BSPK_CUDA(cudaMemcpy(gids, p->d_cspk_gid, 4 * k, cudaMemcpyDeviceToHost));
        }
        *n_out = p->cspk_n;
        return BSPK_OK;
    }
    unsigned long long cnt = 0;
    BSPK_CUDA(cudaMemcpy(&cnt, p->d_spk_count, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (static_cast<int64_t>(cnt) > p->cfg.spike_capacity) {
        *n_out = static_cast<int64_t>(cnt);
        return fail(BSPK_ERR_OVERFLOW, "spike record overflowed its device capacity");
    }
    const int64_t n = std::min<int64_t>(static_cast<int64_t>(cnt), cap);
    if (n > 0) {
        std::vector<int64_t> s(n);
        std::vector<int32_t> g(n);
        BSPK_CUDA(cudaMemcpy(s.data(), p->d_spk_step, 8 * n, cudaMemcpyDeviceToHost));
        BSPK_CUDA(cudaMemcpy(g.data(), p->d_spk_gid, 4 * n, cudaMemcpyDeviceToHost));
        int64_t m = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (g[i] < 0) continue;  // unrecorded neuron
            steps[m] = s[i];
            gids[m] = g[i];
            ++m;
        }
        *n_out = m;
    } else {
        *n_out = static_cast<int64_t>(cnt);
    }
    return BSPK_OK;
}

int bspk_v_get(bspk_plan *p, double *out) {
    if (!p || !p->uploaded || !out) return fail(BSPK_ERR_ARG, "bad arguments");
    int rc = sync_and_check(p);
    if (rc) return rc;
    const size_t n = static_cast<size_t>(p->last_run_steps) * p->rec_v.size();
    if (n == 0) return BSPK_OK;
    // the traces come through a pinned staging buffer kept by the plan: a
    // device-to-pinned copy runs at link speed, a copy into pageable memory
    // is staged by the CUDA driver in small pieces
    const size_t bytes = static_cast<size_t>(p->elt) * n;
    rc = plan_stage(p, bytes);
    if (rc) return rc;
    BSPK_CUDA(cudaMemcpy(p->h_stage, p->d_v, bytes, cudaMemcpyDeviceToHost));
    if (p->elt == 8) {
        memcpy(out, p->h_stage, bytes);
    } else {
        const float *f = static_cast<const float *>(p->h_stage);
        for (size_t i = 0; i < n; ++i) out[i] = f[i];
    }
    return BSPK_OK;
}

int bspk_v_get_f32(bspk_plan *p, float *out) {
    if (!p || !p->uploaded || !out) return fail(BSPK_ERR_ARG, "bad arguments");
    int rc = sync_and_check(p);
    if (rc) return rc;
    const size_t n = static_cast<size_t>(p->last_run_steps) * p->rec_v.size();
    if (n == 0) return BSPK_OK;
    if (p->elt == 4) {  // the traces are float32 on the device: one copy
        BSPK_CUDA(cudaMemcpy(out, p->d_v, 4 * n, cudaMemcpyDeviceToHost));
        return BSPK_OK;
    }
    rc = plan_stage(p, 8 * n);
    if (rc) return rc;
    BSPK_CUDA(cudaMemcpy(p->h_stage, p->d_v, 8 * n, cudaMemcpyDeviceToHost));
    const double *d = static_cast<const double *>(p->h_stage);
    for (size_t i = 0; i < n; ++i) out[i] = static_cast<float>(d[i]);
    return BSPK_OK;
}

int bspk_weights_get(bspk_plan *p, int proj_id, double *w) {
    if (!p || proj_id < 0 || proj_id >= static_cast<int>(p->projs.size()) || !w)
        return fail(BSPK_ERR_ARG, "bad arguments");
    Proj &J = p->projs[proj_id];
    const size_t E = J.post_local.size();
    if (!p->uploaded || !J.plastic) {
        std::copy(J.w.begin(), J.w.end(), w);
        return BSPK_OK;
    }
    int rc = sync_and_check(p);
    if (rc) return rc;
    if (E) BSPK_CUDA(cudaMemcpy(w, J.d_wplastic, 8 * E, cudaMemcpyDeviceToHost));
    return BSPK_OK;
}

int bspk_state_get(bspk_plan *p, int pop, const char *name, double *values) {
    if (!p || !name || !values || pop < 0 || pop >= static_cast<int>(p->pops.size()))
        return fail(BSPK_ERR_ARG, "bad arguments");
    const int slot = state_slot(p->cfg.model, name);
    if (slot < 0) return fail(BSPK_ERR_ARG, std::string("unknown state ") + name);
    if (!p->uploaded) return fail(BSPK_ERR_STATE, "plan not uploaded");
    int rc = sync_and_check(p);
    if (rc) return rc;
    const Pop &P = p->pops[pop];
    if (slot == 100) {
        std::vector<int> r(P.n);
        BSPK_CUDA(cudaMemcpy(r.data(), p->d_r + P.off, 4 * P.n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < P.n; ++i) values[i] = r[i];
        return BSPK_OK;
    }
    const char *base = static_cast<const char *>(p->d_s[slot]) + static_cast<size_t>(p->elt) * P.off;
    if (p->elt == 8) {
        BSPK_CUDA(cudaMemcpy(values, base, 8 * P.n, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> f(P.n);
        BSPK_CUDA(cudaMemcpy(f.data(), base, 4 * P.n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < P.n; ++i) values[i] = f[i];
    }
    return BSPK_OK;
}

int bspk_state_set(bspk_plan *p, int pop, const char *name, const double *values) {
    if (!p || !name || !values || pop < 0 || pop >= static_cast<int>(p->pops.size()))
        return fail(BSPK_ERR_ARG, "bad arguments");
    const int slot = state_slot(p->cfg.model, name);
    if (slot < 0) return fail(BSPK_ERR_ARG, std::string("unknown state ") + name);
    if (!p->uploaded) return fail(BSPK_ERR_STATE, "plan not uploaded");
    BSPK_CUDA(cudaSetDevice(p->cfg.device));
    BSPK_CUDA(cudaDeviceSynchronize());
    const Pop &P = p->pops[pop];
    if (slot == 100) {
        std::vector<int> r(P.n);
        for (int i = 0; i < P.n; ++i) r[i] = static_cast<int>(values[i]);
        BSPK_CUDA(cudaMemcpy(p->d_r + P.off, r.data(), 4 * P.n, cudaMemcpyHostToDevice));
        return BSPK_OK;
    }
    char *base = static_cast<char *>(p->d_s[slot]) + static_cast<size_t>(p->elt) * P.off;
    if (p->elt == 8) {
        BSPK_CUDA(cudaMemcpy(base, values, 8 * P.n, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(values, values + P.n);
        BSPK_CUDA(cudaMemcpy(base, f.data(), 4 * P.n, cudaMemcpyHostToDevice));
    }
    return BSPK_OK;
}

int64_t bspk_step_count(bspk_plan *p) { return p ? p->step : -1; }

int bspk_step_fused(bspk_plan *p, void *stream) { return bspk_run(p, 1, stream); }

int bspk_plan_set_tiled_options(bspk_plan *p, int record_copies, int poll_pause_ns,
                                int drive_overlap, int drive_chunk_steps, int record_stride_bytes) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (record_stride_bytes < 64 || record_stride_bytes > 65536 || record_stride_bytes % 64)
        return fail(BSPK_ERR_ARG, "record stride must be a multiple of 64 bytes in 64..65536");
    if (drive_chunk_steps < 0) return fail(BSPK_ERR_ARG, "drive chunk must be >= 0 steps");
    if (record_copies < 1 || record_copies > kRecRepMax)
        return fail(BSPK_ERR_ARG, "record copies must be in 1.." + std::to_string(kRecRepMax));
    if (poll_pause_ns < 0 || poll_pause_ns > 100000)
        return fail(BSPK_ERR_ARG, "poll pause must be in 0..100000 ns");
    p->rec_rep = record_copies;
    p->poll_pause = poll_pause_ns;
    p->drive_overlap = drive_overlap != 0;
    p->drive_chunk = drive_chunk_steps;
    p->rec_stride = record_stride_bytes / 4;
    p->pref_step0 = -1;
    return BSPK_OK;
}

int bspk_plan_tune_tiled(bspk_plan *p, int64_t pilot_steps, int *grid, int *poll_pause_ns,
                         double *pilot_ms) {
    if (!p || !p->uploaded || !p->tiled) return fail(BSPK_ERR_STATE, "tuning needs an uploaded plan on the tiled path");
    if (pilot_steps <= 0) return fail(BSPK_ERR_ARG, "pilot_steps must be > 0");
    BSPK_CUDA(cudaSetDevice(p->cfg.device));
    int64_t bytes = 0;
    int rc = bspk_checkpoint_size(p, &bytes);
    if (rc) return rc;
    std::vector<char> snap(static_cast<size_t>(bytes));
    rc = bspk_checkpoint_save(p, snap.data(), bytes);
    if (rc) return rc;
    const int g0 = p->grid, pause0 = p->poll_pause;
    std::vector<int> cands;
    for (int G : {g0, g0 * 3 / 4, g0 / 2})
        if (tiled_fits(p, G) && std::find(cands.begin(), cands.end(), G) == cands.end()) cands.push_back(G);
    if (cands.empty()) cands.push_back(g0);
    double best = 1e300;
    int best_g = g0, best_pause = pause0;
    for (int G : cands) {
        if (G != p->grid) {
            rc = retile(p, G);
            if (rc) break;
        }
        for (int pause : {200, 400, 700}) {
            p->poll_pause = pause;
            // the faster of two pilots (one pilot's noise is of the order of
            // the differences between pauses)
            double ms = 1e300;
            for (int rep = 0; rep < 2 && !rc; ++rep) {
                double t = 0.0;
                rc = bspk_run(p, pilot_steps, nullptr);
                if (!rc) rc = sync_and_check(p);
                if (!rc) rc = bspk_last_kernel_time(p, &t, nullptr);
                if (!rc) rc = bspk_checkpoint_restore(p, snap.data(), bytes);
                ms = std::min(ms, t);
            }
            if (rc) break;
            if (ms < best) {
                best = ms;
                best_g = G;
                best_pause = pause;
            }
        }
        if (rc) break;
    }
    // the best shape, and the state as it was
    int rc2 = best_g != p->grid ? retile(p, best_g) : BSPK_OK;
    p->poll_pause = rc ? pause0 : best_pause;
    if (!rc2) rc2 = bspk_checkpoint_restore(p, snap.data(), bytes);
    if (rc) return rc;
    if (rc2) return rc2;
    if (grid) *grid = best_g;
    if (poll_pause_ns) *poll_pause_ns = best_pause;
    if (pilot_ms) *pilot_ms = best;
    return BSPK_OK;
}

int bspk_plan_get_tiled_options(bspk_plan *p, int *record_copies, int *poll_pause_ns,
                                int *drive_overlap, int *drive_chunk_steps,
                                int *record_stride_bytes) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (record_stride_bytes) *record_stride_bytes = p->rec_stride * 4;
    if (drive_chunk_steps) *drive_chunk_steps = p->drive_chunk;
    if (record_copies) *record_copies = p->rec_rep;
    if (poll_pause_ns) *poll_pause_ns = p->poll_pause;
    if (drive_overlap) *drive_overlap = p->drive_overlap ? 1 : 0;
    return BSPK_OK;
}

int bspk_record_weights(bspk_plan *p, int proj_id, int on) {
    if (!p || proj_id < 0 || proj_id >= static_cast<int>(p->projs.size()))
        return fail(BSPK_ERR_ARG, "bad projection");
    if (!p->projs[proj_id].plastic)
        return fail(BSPK_ERR_ARG, "record_weights needs a plastic projection");
    p->projs[proj_id].rec_w = on != 0;
    return BSPK_OK;
}

int bspk_weight_trace_get(bspk_plan *p, int proj_id, int64_t *n_steps, double *out) {
    if (!p || proj_id < 0 || proj_id >= static_cast<int>(p->projs.size()))
        return fail(BSPK_ERR_ARG, "bad projection");
    Proj &J = p->projs[proj_id];
    if (!J.rec_w || !J.d_wtrace) return fail(BSPK_ERR_STATE, "no weight trajectory recorded");
    if (n_steps) *n_steps = J.wtrace_steps;
    if (!out) return BSPK_OK;
    int rc = sync_and_check(p);
    if (rc) return rc;
    BSPK_CUDA(cudaMemcpy(out, J.d_wtrace,
                         sizeof(double) * J.wtrace_steps * static_cast<int64_t>(J.post_local.size()),
                         cudaMemcpyDeviceToHost));
    return BSPK_OK;
}

int bspk_plan_ring_fraction_bits(bspk_plan *p, int *bits) {
    if (!p || !bits) return fail(BSPK_ERR_ARG, "null argument");
    if (!p->uploaded || !p->tiled) return fail(BSPK_ERR_STATE, "not an uploaded plan on the tiled path");
    *bits = static_cast<int>(std::lround(-std::log2(p->tinv_scale)));
    return BSPK_OK;
}

int bspk_plan_set_trial(bspk_plan *p, uint32_t trial) {
    if (!p) return fail(BSPK_ERR_ARG, "null plan");
    if (p->uploaded) return fail(BSPK_ERR_STATE, "the trial is set before upload");
    p->trial = trial;
    return BSPK_OK;
}

int bspk_plan_set_windowed(bspk_plan *p, int on) {
    if (!p || !p->uploaded) return fail(BSPK_ERR_STATE, "plan not uploaded");
    if (on && !p->win_ok) return fail(BSPK_ERR_UNSUPPORTED, "this plan cannot run windowed");
    p->win = on != 0;
    return BSPK_OK;
}

const char *bspk_plan_engine(bspk_plan *p) {
    if (!p || !p->uploaded) return "";
    bool per_step = plan_per_step(p);
    for (auto &J : p->projs) per_step |= J.plastic;
    if (per_step) return p->win ? "windowed" : "per_step";
    if (p->cfg.deterministic) return "exact";
    if (p->tiled) return "tiled";
    return "global_ring";
}

int bspk_last_kernel_time(bspk_plan *p, double *ms, int64_t *launches) {
    if (!p || !p->uploaded) return fail(BSPK_ERR_ARG, "bad arguments");
    BSPK_CUDA(cudaEventSynchronize(p->ev1));
    float f = 0.f;
    BSPK_CUDA(cudaEventElapsedTime(&f, p->ev0, p->ev1));
    if (ms) *ms = f;
    if (launches) *launches = p->last_launches;
    return BSPK_OK;
}

int bspk_rk_substeps(bspk_plan *p, int64_t *total) {
    if (!p || !total || !p->uploaded) return fail(BSPK_ERR_ARG, "bad arguments");
    const int rc = sync_and_check(p);
    if (rc) return rc;
    unsigned long long v = 0;
    BSPK_CUDA(cudaMemcpy(&v, p->d_rk_iters, sizeof(v), cudaMemcpyDeviceToHost));
    *total = static_cast<int64_t>(v);
    return BSPK_OK;
}

}  // extern "C"
