/* bspk_oracle_bptt.c -- float64 CPU restatement of surrogate-gradient BPTT
 * through a recurrent iaf_psc_exp network (TEST INFRASTRUCTURE ONLY: the
 * checker of the GPU adjoint, never part of the product path).
 *
 * Forward (hard): the NEST iaf_psc_exp step of _nest_neuron/iaf_psc_exp.py:
 * 552-682 (no current injector), the summed input sign-split into the two
 * synaptic currents (iaf_psc_exp.py:641-643); a spike is allowed only when
 * the neuron was not refractory at the start of the step (the refractory
 * mask of _kernel/spiking.py SpikeRule.check, :364-420).
 * Backward: count_ste (_kernel/spiking.py:65-88): the spike's gradient is the
 * surrogate derivative of the margin V - V_th; the reset carries the soft
 * gradient d_spike * (V_reset - V) unless detach_reset (SpikeRule._jump,
 * :449-466).  Relaxed forward (_check_relaxed, :422-447): spikes are the
 * surrogate primitive, the reset is applied softly, refractoriness keeps the
 * hard condition.
 * Surrogate: fast sigmoid of slope beta as a smooth step,
 *     sigma(m) = 0.5 * (1 + beta m / (1 + beta |m|)),
 *     sigma'(m) = 0.5 beta / (1 + beta |m|)^2.
 * Readout and loss: z_t = alpha z_{t-1} + c s_t for neurons 0..R-1,
 * alpha = exp(-dt/tau_r), c = (1 - alpha) * 1000 / dt (Hz), loss = mean over
 * (trial, step, readout) of (z - y)^2 (rate_mse, _kernel/learn/bptt.py:142-214).
 * Recurrent spikes of step t reach the network at step t + 1; input counts
 * of step t act in step t.
 *
 * Arithmetic order (the GPU kernels follow it operation for operation):
 *   x  = sum over in-edges (row order) of w * s_prev, then + w_in * u over the
 *        active inputs in ascending order;
 *   ls = (readout ? c * g : 0) + sum over out-edges (pre-major, stable) of w * lx_next;
 *   per trial dW accumulates over descending t; trials are summed in order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "bspk_oracle.h"

static double sur_grad(double m, double halfbeta, double beta) {
    double q = 1.0 + beta * fabs(m);
    return halfbeta / (q * q);
}

static double sur_fun(double m, double beta) {
    double q = 1.0 + beta * fabs(m);
    return 0.5 * (1.0 + (beta * m) / q);
}

int bo_lif_bptt(const bo_bptt_cfg *c, const int64_t *row_ptr, const int32_t *col, int64_t nnz,
                const double *w, const double *w_in, const uint8_t *inputs, const double *targets,
                double *loss, double *dw, double *dw_in, int64_t *n_spikes) {
    const int N = c->n, NI = c->n_in, B = c->batch, T = c->n_steps, R = c->n_readout;
    if (N <= 0 || B <= 0 || T <= 0 || R < 0 || R > N || NI < 0) return -1;
    const double h = c->dt;
    const double E_L = c->params[0], C_m = c->params[1], tau_m = c->params[2],
                 t_ref = c->params[3], V_th = c->params[4], V_reset = c->params[5],
                 tex = c->params[6], tin = c->params[7], I_e = c->params[8];
    const double eP22 = exp(-h / tau_m), eP11ex = exp(-h / tex), eP11in = exp(-h / tin);
    const double eP21ex = bo_propagator_exp(tex, tau_m, C_m, h);
    const double eP21in = bo_propagator_exp(tin, tau_m, C_m, h);
    const double eP20 = tau_m / C_m * (1.0 - exp(-h / tau_m));
    const double theta = V_th - E_L, vr = V_reset - E_L;
    const int ref = (int)ceil(t_ref / h);
    const double alpha = exp(-h / c->readout_tau);
    const double cz = (1.0 - alpha) * 1000.0 / h;
    const double denom = (double)B * (double)T * (double)R;
    const double inv = 2.0 / denom;
    const double beta = c->slope, halfbeta = 0.5 * c->slope;
    const int grad = dw != NULL;

    /* out-edge lists: stable counting sort of the in-edge list by pre */
    int64_t *optr = (int64_t *)calloc((size_t)N + 1, sizeof(int64_t));
    int64_t *oeid = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
    int32_t *opost = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    for (int64_t e = 0; e < nnz; ++e) optr[col[e] + 1]++;
    for (int i = 0; i < N; ++i) optr[i + 1] += optr[i];
    {
        int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)N);
        for (int i = 0; i < N; ++i) fill[i] = optr[i];
        for (int i = 0; i < N; ++i)
            for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
                int64_t q = fill[col[e]]++;
                oeid[q] = e;
                opost[q] = i;
            }
        free(fill);
    }
    const size_t TN = (size_t)T * (size_t)N;
    double *X = (double *)malloc(sizeof(double) * TN);
    double *VT = (double *)malloc(sizeof(double) * TN);
    double *S = (double *)malloc(sizeof(double) * TN);
    uint8_t *A = (uint8_t *)malloc(TN);
    double *Z = (double *)malloc(sizeof(double) * (size_t)T * (size_t)(R > 0 ? R : 1));
    double *V = (double *)malloc(sizeof(double) * (size_t)N);
    double *Ie = (double *)malloc(sizeof(double) * (size_t)N);
    double *Ii = (double *)malloc(sizeof(double) * (size_t)N);
    int *rr = (int *)malloc(sizeof(int) * (size_t)N);
    double *zz = (double *)malloc(sizeof(double) * (size_t)(R > 0 ? R : 1));
    double *acc = (double *)malloc(sizeof(double) * (size_t)(R > 0 ? R : 1));
    double *lV = (double *)malloc(sizeof(double) * (size_t)N);
    double *lIe = (double *)malloc(sizeof(double) * (size_t)N);
    double *lIi = (double *)malloc(sizeof(double) * (size_t)N);
    double *lxn = (double *)malloc(sizeof(double) * (size_t)N);
    double *lxc = (double *)malloc(sizeof(double) * (size_t)N);
    double *ls = (double *)malloc(sizeof(double) * (size_t)N);
    double *g = (double *)malloc(sizeof(double) * (size_t)(R > 0 ? R : 1));
    double *dwb = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    double *dwib = (double *)malloc(sizeof(double) * (size_t)N * (size_t)(NI > 0 ? NI : 1));
    if (grad) {
        memset(dw, 0, sizeof(double) * (size_t)nnz);
        if (dw_in) memset(dw_in, 0, sizeof(double) * (size_t)N * (size_t)NI);
    }
    double total = 0.0;
    int64_t nsp = 0;
    for (int b = 0; b < B; ++b) {
        for (int i = 0; i < N; ++i) {
            V[i] = 0.0;
            Ie[i] = 0.0;
            Ii[i] = 0.0;
            rr[i] = 0;
        }
        for (int j = 0; j < R; ++j) {
            zz[j] = 0.0;
            acc[j] = 0.0;
        }
        /* ---- forward, whole trajectory kept */
        for (int t = 0; t < T; ++t) {
            const uint8_t *u = inputs + ((size_t)t * B + b) * (size_t)NI;
            const double *sp = t > 0 ? S + (size_t)(t - 1) * N : NULL;
            double *st = S + (size_t)t * N;
            for (int i = 0; i < N; ++i) {
                double x = 0.0;
                if (sp)
                    for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) x = x + w[e] * sp[col[e]];
                for (int k = 0; k < NI; ++k)
                    if (u[k]) x = x + w_in[(size_t)i * NI + k] * (double)u[k];
                const int a = rr[i] == 0;
                double Vt = V[i];
                if (a) Vt = V[i] * eP22 + Ie[i] * eP21ex + Ii[i] * eP21in + I_e * eP20;
                else rr[i] = rr[i] - 1;
                double ie = Ie[i] * eP11ex, ii = Ii[i] * eP11in;
                const double wex = x > 0.0 ? x : 0.0, win = x < 0.0 ? x : 0.0;
                Ie[i] = ie + wex;
                Ii[i] = ii + win;
                const int hard = a && Vt >= theta;
                double s;
                if (c->relaxed) {
                    s = a ? sur_fun(Vt - theta, beta) : 0.0;
                    V[i] = Vt + s * (vr - Vt);
                } else {
                    s = hard ? 1.0 : 0.0;
                    V[i] = hard ? vr : Vt;
                }
                if (hard) {
                    rr[i] = ref;
                    nsp++;
                }
                X[(size_t)t * N + i] = x;
                VT[(size_t)t * N + i] = Vt;
                A[(size_t)t * N + i] = (uint8_t)a;
                st[i] = s;
            }
            const double *y = targets + ((size_t)t * B + b) * (size_t)R;
            for (int j = 0; j < R; ++j) {
                zz[j] = zz[j] * alpha + cz * st[j];
                const double d = zz[j] - y[j];
                acc[j] = acc[j] + d * d;
                Z[(size_t)t * R + j] = zz[j];
            }
        }
        double lb = 0.0;
        for (int j = 0; j < R; ++j) lb = lb + acc[j];
        total = total + lb;
        if (!grad) continue;
        /* ---- backward */
        for (int i = 0; i < N; ++i) {
            lV[i] = 0.0;
            lIe[i] = 0.0;
            lIi[i] = 0.0;
            lxn[i] = 0.0;
        }
        for (int j = 0; j < R; ++j) g[j] = 0.0;
        memset(dwb, 0, sizeof(double) * (size_t)nnz);
        memset(dwib, 0, sizeof(double) * (size_t)N * (size_t)NI);
        for (int t = T - 1; t >= 0; --t) {
            const double *y = targets + ((size_t)t * B + b) * (size_t)R;
            for (int j = 0; j < R; ++j) g[j] = (Z[(size_t)t * R + j] - y[j]) * inv + alpha * g[j];
            for (int p = 0; p < N; ++p) {
                double l = p < R ? cz * g[p] : 0.0;
                for (int64_t q = optr[p]; q < optr[p + 1]; ++q) l = l + w[oeid[q]] * lxn[opost[q]];
                ls[p] = l;
            }
            const uint8_t *u = inputs + ((size_t)t * B + b) * (size_t)NI;
            const double *sp = t > 0 ? S + (size_t)(t - 1) * N : NULL;
            for (int i = 0; i < N; ++i) {
                const size_t o = (size_t)t * N + i;
                const int a = A[o];
                const double Vt = VT[o], s = S[o];
                const double m = Vt - theta;
                const double sg = a ? sur_grad(m, halfbeta, beta) : 0.0;
                const double cross = c->detach_reset ? 0.0 : lV[i] * (vr - Vt);
                const double lVt = lV[i] * (1.0 - s) + (ls[i] + cross) * sg;
                const double lx = X[o] >= 0.0 ? lIe[i] : lIi[i];
                lIe[i] = lIe[i] * eP11ex + (a ? lVt * eP21ex : 0.0);
                lIi[i] = lIi[i] * eP11in + (a ? lVt * eP21in : 0.0);
                lV[i] = a ? lVt * eP22 : lVt;
                lxc[i] = lx;
                if (sp)
                    for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e)
                        if (sp[col[e]] != 0.0) dwb[e] = dwb[e] + lx * sp[col[e]];
                for (int k = 0; k < NI; ++k)
                    if (u[k]) dwib[(size_t)i * NI + k] = dwib[(size_t)i * NI + k] + lx * (double)u[k];
            }
            double *tmp = lxn;
            lxn = lxc;
            lxc = tmp;
        }
        for (int64_t e = 0; e < nnz; ++e) dw[e] = dw[e] + dwb[e];
        if (dw_in)
            for (size_t q = 0; q < (size_t)N * NI; ++q) dw_in[q] = dw_in[q] + dwib[q];
    }
    *loss = total / denom;
    if (n_spikes) *n_spikes = nsp;
    free(optr); free(oeid); free(opost); free(X); free(VT); free(S); free(A); free(Z);
    free(V); free(Ie); free(Ii); free(rr); free(zz); free(acc); free(lV); free(lIe); free(lIi);
    free(lxn); free(lxc); free(ls); free(g); free(dwb); free(dwib);
    return 0;
}
