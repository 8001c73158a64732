/*
 * pmcmc_oracle.c -- TEST INFRASTRUCTURE ONLY (see pmcmc_oracle.h).
 *
 * FP64 CPU restatement of the reference's DEER hot path.  Every function cites
 * the reference file:line it follows (paths relative to the ParallelMCMC.jl
 * project root).  Compiled with -ffp-contract=off so that the FP32 tape
 * generator rounds exactly like the device generator (explicit fmaf only).
 */
#include "pmcmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ========================================================================= */
/* Tape generator: Philox4x32-10 (Salmon et al., SC'11) + Box-Muller.          */
/* This is the project's tape specification (the reference draws its tape from */
/* Julia's MersenneTwister, interface.jl:334-358, which cannot be reproduced). */
/* ========================================================================= */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u
enum { TAG_XI = 1, TAG_U = 2, TAG_Z = 3 };

void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += PHILOX_W0;
            k1 += PHILOX_W1;
        }
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* (2k+1) * 2^-24 with k = top 23 bits: exact in FP32, strictly inside (0,1). */
float orc_u01(uint32_t bits) {
    uint32_t k = bits >> 9;
    return (float)(2u * k + 1u) * 0x1p-24f;
}

static float f_from_bits(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static uint32_t f_bits(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }

/* Natural log for x in [2^-24, 1]: x = m 2^e, m in [sqrt(1/2), sqrt(2)),
 * ln m = 2 atanh(s), s = (m-1)/(m+1), atanh series to s^11 (|s| <= 0.1716). */
float orc_logf(float x) {
    uint32_t b = f_bits(x);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = f_from_bits((b & 0x7fffffu) | 0x3f800000u);
    if (m > 0x1.6a09e6p+0f) { m = m * 0.5f; e += 1; }
    float num = m - 1.0f;
    float den = m + 1.0f;
    float s = num / den;
    float s2 = s * s;
    float p = 0x1.745d18p-4f;
    p = fmaf(p, s2, 0x1.c71c72p-4f);
    p = fmaf(p, s2, 0x1.24924ap-3f);
    p = fmaf(p, s2, 0x1.99999ap-3f);
    p = fmaf(p, s2, 0x1.555556p-2f);
    float t = 2.0f * s;
    float ts2 = t * s2;
    float lnm = fmaf(ts2, p, t);
    return fmaf((float)e, 0x1.62e430p-1f, lnm);
}

/* sin and cos of 2*pi*u for u in (0,1): quadrant k = rint(4u), phi = (4u-k)*pi/2
 * in [-pi/4, pi/4], Taylor polynomials (sin to phi^9, cos to phi^10). */
void orc_sincos2pi(float u, float* s_out, float* c_out) {
    float q4 = u * 4.0f;
    float k = rintf(q4);
    float f = q4 - k;
    float phi = f * 0x1.921fb6p+0f;
    float p2 = phi * phi;
    float sp = 0x1.71de3ap-19f;
    sp = fmaf(sp, p2, -0x1.a01a02p-13f);
    sp = fmaf(sp, p2, 0x1.111112p-7f);
    sp = fmaf(sp, p2, -0x1.555556p-3f);
    float pp = phi * p2;
    float sn = fmaf(pp, sp, phi);
    float cp = -0x1.27e4fcp-22f;
    cp = fmaf(cp, p2, 0x1.a01a02p-16f);
    cp = fmaf(cp, p2, -0x1.6c16c2p-10f);
    cp = fmaf(cp, p2, 0x1.555556p-5f);
    cp = fmaf(cp, p2, -0.5f);
    float cs = fmaf(p2, cp, 1.0f);
    int ki = ((int)k) & 3;
    float s, c;
    switch (ki) {
        case 0: s = sn; c = cs; break;
        case 1: s = cs; c = -sn; break;
        case 2: s = -sn; c = -cs; break;
        default: s = -cs; c = sn; break;
    }
    *s_out = s;
    *c_out = c;
}

static void box_muller(uint32_t b1, uint32_t b2, float* n0, float* n1) {
    float u1 = orc_u01(b1), u2 = orc_u01(b2);
    float L = orc_logf(u1);
    float r = sqrtf(-2.0f * L);
    float s, c;
    orc_sincos2pi(u2, &s, &c);
    *n0 = r * c;
    *n1 = r * s;
}

/* Tape block (xi_t ~ N(0,I_D) and u_t ~ U(0,1) for t = 0..T-1): the counter-based
 * counterpart of _make_mala_tape_block (interface.jl:334-358). */
void orc_tape(uint64_t seed, uint64_t block, int64_t D, int64_t T, float* Xi, float* u) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    int64_t nq = (D + 3) / 4;
    for (int64_t t = 0; t < T; ++t) {
        for (int64_t j = 0; j < nq; ++j) {
            uint32_t ctr[4] = {(uint32_t)j, (uint32_t)t, (uint32_t)block, TAG_XI}, o[4];
            orc_philox4x32_10(ctr, key, o);
            float n[4];
            box_muller(o[0], o[1], &n[0], &n[1]);
            box_muller(o[2], o[3], &n[2], &n[3]);
            for (int i = 0; i < 4; ++i) {
                int64_t d = 4 * j + i;
                if (d < D && Xi) Xi[t * D + d] = n[i];
            }
        }
        if (u) {
            uint32_t ctr[4] = {0u, (uint32_t)t, (uint32_t)block, TAG_U}, o[4];
            orc_philox4x32_10(ctr, key, o);
            u[t] = orc_u01(o[0]);
        }
    }
}

/* Rademacher probe Z (D x T) for Newton iteration `iter`, probe `probe`:
 * counter-based replacement of _rademacher! (DEER.jl:298-325). */
void orc_probe(uint64_t seed, uint64_t block, int32_t iter, int32_t probe, int64_t D,
               int64_t T, double* Z) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t tag = TAG_Z | ((uint32_t)probe << 4) | ((uint32_t)iter << 12);
    for (int64_t t = 0; t < T; ++t) {
        for (int64_t j = 0; j * 128 < D; ++j) {
            uint32_t ctr[4] = {(uint32_t)j, (uint32_t)t, (uint32_t)block, tag}, o[4];
            orc_philox4x32_10(ctr, key, o);
            for (int64_t d = j * 128; d < D && d < (j + 1) * 128; ++d) {
                uint32_t w = o[(d >> 5) & 3];
                Z[t * D + d] = ((w >> (d & 31)) & 1u) ? 1.0 : -1.0;
            }
        }
    }
}

/* ========================================================================= */
/* Targets.                                                                   */
/* ========================================================================= */
static double softplus(double z) { return (z > 0 ? z : 0.0) + log1p(exp(-fabs(z))); }
static double sigm(double l) { return 1.0 / (1.0 + exp(-l)); }

/* logits l = X * theta (bayes_logreg.jl:38, mul!(logits, X, beta)) */
static void logits(const orc_target* tg, const double* th, double* l) {
    int64_t N = tg->N, D = tg->D;
    for (int64_t n = 0; n < N; ++n) l[n] = 0.0;
    for (int64_t i = 0; i < D; ++i) {
        const double* col = tg->X + i * N;
        double ti = th[i];
        for (int64_t n = 0; n < N; ++n) l[n] += col[n] * ti;
    }
}

static double mu(const orc_target* tg, int64_t i) { return tg->mean ? tg->mean[i] : 0.0; }

/* logp: diag/dense Gaussian; logistic = bayes_logreg.jl:37-46 with the stable
 * softplus of docs/src/15-gpu.md:91-97 and prior precision tau. */
double orc_logp(const orc_target* tg, const double* x) {
    int64_t D = tg->D;
    if (tg->kind == ORC_DIAG_GAUSS) {
        double s = 0;
        for (int64_t i = 0; i < D; ++i) {
            double r = x[i] - mu(tg, i);
            s += tg->prec[i] * r * r;
        }
        return -0.5 * s;
    } else if (tg->kind == ORC_DENSE_GAUSS) {
        double s = 0;
        for (int64_t j = 0; j < D; ++j) {
            double rj = x[j] - mu(tg, j), acc = 0;
            for (int64_t i = 0; i < D; ++i) acc += tg->prec[j * D + i] * (x[i] - mu(tg, i));
            s += rj * acc;
        }
        return -0.5 * s;
    } else {
        int64_t N = tg->N;
        double* l = (double*)malloc(sizeof(double) * N);
        logits(tg, x, l);
        double s = 0;
        for (int64_t n = 0; n < N; ++n)
            s += tg->y[n] * (-softplus(-l[n])) + (1.0 - tg->y[n]) * (-softplus(l[n]));
        free(l);
        double q = 0;
        for (int64_t i = 0; i < D; ++i) q += x[i] * x[i];
        return s - 0.5 * tg->prior_prec * q;
    }
}

/* grad: logistic = bayes_logreg.jl:48-58 (X'(y - sigma(X beta)) - tau beta). */
void orc_grad(const orc_target* tg, const double* x, double* g) {
    int64_t D = tg->D;
    if (tg->kind == ORC_DIAG_GAUSS) {
        for (int64_t i = 0; i < D; ++i) g[i] = -tg->prec[i] * (x[i] - mu(tg, i));
    } else if (tg->kind == ORC_DENSE_GAUSS) {
        for (int64_t i = 0; i < D; ++i) g[i] = 0.0;
        for (int64_t j = 0; j < D; ++j) {
            double rj = x[j] - mu(tg, j);
            for (int64_t i = 0; i < D; ++i) g[i] -= tg->prec[j * D + i] * rj;
        }
    } else {
        int64_t N = tg->N;
        double* l = (double*)malloc(sizeof(double) * N);
        logits(tg, x, l);
        for (int64_t n = 0; n < N; ++n) l[n] = tg->y[n] - sigm(l[n]);
        for (int64_t i = 0; i < D; ++i) {
            const double* col = tg->X + i * N;
            double s = 0;
            for (int64_t n = 0; n < N; ++n) s += col[n] * l[n];
            g[i] = s - tg->prior_prec * x[i];
        }
        free(l);
    }
}

/* hvp: logistic = bayes_logreg.jl:76-83 (-X'(w .* Xv) - tau v, w = p(1-p)). */
void orc_hvp(const orc_target* tg, const double* x, const double* v, double* out) {
    int64_t D = tg->D;
    if (tg->kind == ORC_DIAG_GAUSS) {
        for (int64_t i = 0; i < D; ++i) out[i] = -tg->prec[i] * v[i];
    } else if (tg->kind == ORC_DENSE_GAUSS) {
        for (int64_t i = 0; i < D; ++i) out[i] = 0.0;
        for (int64_t j = 0; j < D; ++j)
            for (int64_t i = 0; i < D; ++i) out[i] -= tg->prec[j * D + i] * v[j];
    } else {
        int64_t N = tg->N;
        double* l = (double*)malloc(sizeof(double) * N);
        double* xv = (double*)malloc(sizeof(double) * N);
        logits(tg, x, l);
        logits(tg, v, xv);
        for (int64_t n = 0; n < N; ++n) {
            double p = sigm(l[n]);
            xv[n] *= p * (1.0 - p);
        }
        for (int64_t i = 0; i < D; ++i) {
            const double* col = tg->X + i * N;
            double s = 0;
            for (int64_t n = 0; n < N; ++n) s += col[n] * xv[n];
            out[i] = -s - tg->prior_prec * v[i];
        }
        free(l);
        free(xv);
    }
}

/* ========================================================================= */
/* MALA (identity mass matrix).                                               */
/* ========================================================================= */

/* logq_mala! (MALA.jl:172-193): -0.5 |y - x - eps g_x|^2 / (2 eps) - (D/2) log(4 pi eps). */
double orc_logq(const orc_target* tg, const double* y, const double* x, const double* gx,
                double eps) {
    int64_t D = tg->D;
    double s = 0;
    for (int64_t i = 0; i < D; ++i) {
        double mu_i = x[i] + eps * gx[i];
        double r = y[i] - mu_i;
        s += r * r;
    }
    return -0.5 * s / (2 * eps) - ((double)D / 2) * log(4 * M_PI * eps);
}

typedef struct {
    double *gx, *gy, *y, *hvx, *hvy, *w, *r, *dr;
} mala_ws;

static void ws_alloc(mala_ws* w, int64_t D) {
    double* m = (double*)malloc(sizeof(double) * 8 * D);
    w->gx = m; w->gy = m + D; w->y = m + 2 * D; w->hvx = m + 3 * D;
    w->hvy = m + 4 * D; w->w = m + 5 * D; w->r = m + 6 * D; w->dr = m + 7 * D;
}
static void ws_free(mala_ws* w) { free(w->gx); }

/* Forward half shared by mala_step_with_logalpha! (MALA.jl:377-411) and the
 * fused fwd+JVP (MALA.jl:732-797): proposal (MALA.jl:221-222), logalpha (:402). */
static double mala_forward(const orc_target* tg, double eps, const double* x, const double* xi,
                           mala_ws* w) {
    int64_t D = tg->D;
    orc_grad(tg, x, w->gx);
    double s2e = sqrt(2 * eps);
    for (int64_t i = 0; i < D; ++i) w->y[i] = x[i] + eps * w->gx[i] + s2e * xi[i];
    double lpx = orc_logp(tg, x);
    double lpy = orc_logp(tg, w->y);
    orc_grad(tg, w->y, w->gy);
    double lq_yx = orc_logq(tg, w->y, x, w->gx, eps);
    double lq_xy = orc_logq(tg, x, w->y, w->gy, eps);
    return (lpy + lq_xy) - (lpx + lq_yx);
}

double orc_mala_step(const orc_target* tg, double eps, const double* x, const double* xi,
                     double u, double* x_next, int32_t* accepted) {
    mala_ws w;
    ws_alloc(&w, tg->D);
    double la = mala_forward(tg, eps, x, xi, &w);
    int acc = log(u) < la; /* strict, MALA.jl:404 */
    memcpy(x_next, acc ? w.y : x, sizeof(double) * tg->D);
    if (accepted) *accepted = acc;
    ws_free(&w);
    return la;
}

/* run_mala_sequential_taped (MALA.jl:322-346); S column t = x_{t+1}. */
void orc_mala_sequential(const orc_target* tg, double eps, const double* x0, const double* Xi,
                         const double* u, int64_t T, double* S, int32_t* accepted,
                         double* logalpha) {
    int64_t D = tg->D;
    const double* x = x0;
    for (int64_t t = 0; t < T; ++t) {
        int32_t a;
        double la = orc_mala_step(tg, eps, x, Xi + t * D, u[t], S + t * D, &a);
        if (accepted) accepted[t] = a;
        if (logalpha) logalpha[t] = la;
        x = S + t * D;
    }
}

/* lp(th) and g(th) of the logistic target, with the arithmetic of orc_logp and
 * orc_grad (bayes_logreg.jl:37-58): every logit sums over i in order, every
 * gradient entry over n in order, and the log-likelihood terms are added in
 * row order.  Threads split the rows (logits, terms) and the coordinates
 * (gradient), which leaves each sum's order, and so its rounding, unchanged. */
static double logistic_lp_grad(const orc_target* tg, const double* th, double* l, double* term,
                               double* g, int nth) {
    const int64_t N = tg->N, D = tg->D;
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
    {
        int me = 0, nt = 1;
#ifdef _OPENMP
        me = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        const int64_t n0 = N * me / nt, n1 = N * (me + 1) / nt;
        for (int64_t n = n0; n < n1; ++n) l[n] = 0.0;
        for (int64_t i = 0; i < D; ++i) {
            const double* col = tg->X + i * N;
            const double ti = th[i];
            for (int64_t n = n0; n < n1; ++n) l[n] += col[n] * ti;
        }
        for (int64_t n = n0; n < n1; ++n) {
            term[n] = tg->y[n] * (-softplus(-l[n])) + (1.0 - tg->y[n]) * (-softplus(l[n]));
            l[n] = tg->y[n] - sigm(l[n]);
        }
#ifdef _OPENMP
#pragma omp barrier
#pragma omp for schedule(static)
#endif
        for (int64_t i = 0; i < D; ++i) {
            const double* col = tg->X + i * N;
            double s = 0;
            for (int64_t n = 0; n < N; ++n) s += col[n] * l[n];
            g[i] = s - tg->prior_prec * th[i];
        }
    }
    double s = 0;
    for (int64_t n = 0; n < N; ++n) s += term[n];
    double q = 0;
    for (int64_t i = 0; i < D; ++i) q += th[i] * th[i];
    return s - 0.5 * tg->prior_prec * q;
}

/* orc_mala_sequential for the logistic target, with the log density and the
 * gradient of an accepted proposal carried to the next step (they are the
 * values at the new state) and the target's sums split over threads as in
 * logistic_lp_grad: the same results as orc_mala_sequential, bit for bit, in
 * a time that makes full-size chains (N = 10000, D = 256, T = 65536) a test. */
void orc_mala_sequential_logistic(const orc_target* tg, double eps, const double* x0,
                                  const double* Xi, const double* u, int64_t T, double* S,
                                  int32_t* accepted, double* logalpha, int32_t nthreads) {
    const int64_t N = tg->N, D = tg->D;
    int nth = 1;
#ifdef _OPENMP
    nth = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    (void)nthreads;
    double* buf = (double*)malloc(sizeof(double) * (2 * N + 4 * D));
    double *l = buf, *term = buf + N, *x = buf + 2 * N, *gx = x + D, *y = gx + D, *gy = y + D;
    memcpy(x, x0, sizeof(double) * D);
    double lpx = logistic_lp_grad(tg, x, l, term, gx, nth);
    const double s2e = sqrt(2 * eps);
    for (int64_t t = 0; t < T; ++t) {
        const double* xi = Xi + t * D;
        for (int64_t i = 0; i < D; ++i) y[i] = x[i] + eps * gx[i] + s2e * xi[i];
        const double lpy = logistic_lp_grad(tg, y, l, term, gy, nth);
        const double lq_yx = orc_logq(tg, y, x, gx, eps);
        const double lq_xy = orc_logq(tg, x, y, gy, eps);
        const double la = (lpy + lq_xy) - (lpx + lq_yx);
        const int acc = log(u[t]) < la; /* strict, MALA.jl:404 */
        if (acc) {
            memcpy(x, y, sizeof(double) * D);
            memcpy(gx, gy, sizeof(double) * D);
            lpx = lpy;
        }
        memcpy(S + t * D, x, sizeof(double) * D);
        if (accepted) accepted[t] = acc;
        if (logalpha) logalpha[t] = la;
    }
    free(buf);
}

/* Mass-matrix MALA with M = L L^T (cholM of the reference), L lower triangular,
 * D x D column-major: _apply_M! (MALA.jl:29-35), _apply_L! (:37-38), _quad_Minv!
 * (:40-44), _logdet_M (:46-47), the proposal (:207-229), logq_mala! (:160-193) and
 * the strict accept test of mala_step_with_logalpha! (:377-411).  S column t = x_{t+1}. */
static void lower_mv(int64_t D, const double* L, const double* v, double* out) {
    for (int64_t i = 0; i < D; ++i) out[i] = 0.0;
    for (int64_t k = 0; k < D; ++k)
        for (int64_t i = k; i < D; ++i) out[i] += L[k * D + i] * v[k];
}
static void lower_t_mv(int64_t D, const double* L, const double* v, double* out) {
    for (int64_t k = 0; k < D; ++k) {
        double s = 0.0;
        for (int64_t i = k; i < D; ++i) s += L[k * D + i] * v[i];
        out[k] = s;
    }
}
/* |L^-1 r|^2 by forward substitution (ldiv! with the lower factor) */
static double quad_minv(int64_t D, const double* L, const double* r, double* tmp) {
    double q = 0.0;
    for (int64_t i = 0; i < D; ++i) {
        double s = r[i];
        for (int64_t k = 0; k < i; ++k) s -= L[k * D + i] * tmp[k];
        tmp[i] = s / L[i * D + i];
        q += tmp[i] * tmp[i];
    }
    return q;
}

void orc_mala_sequential_mass(const orc_target* tg, double eps, const double* L, const double* x0,
                              const double* Xi, const double* u, int64_t T, double* S,
                              int32_t* accepted, double* logalpha) {
    const int64_t D = tg->D;
    double* b = (double*)malloc(sizeof(double) * 9 * D);
    double *x = b, *gx = b + D, *y = b + 2 * D, *gy = b + 3 * D, *mg = b + 4 * D,
           *lx = b + 5 * D, *tmp = b + 6 * D, *r = b + 7 * D, *t2 = b + 8 * D;
    double logdet = 0.0;
    for (int64_t i = 0; i < D; ++i) logdet += 2.0 * log(L[i * D + i]);
    const double c = (double)D / 2 * log(4 * M_PI * eps);
    const double s2e = sqrt(2 * eps);
    memcpy(x, x0, sizeof(double) * D);
    for (int64_t t = 0; t < T; ++t) {
        orc_grad(tg, x, gx);
        lower_t_mv(D, L, gx, tmp);
        lower_mv(D, L, tmp, mg);           /* M g_x */
        lower_mv(D, L, Xi + t * D, lx);    /* L xi */
        for (int64_t i = 0; i < D; ++i) y[i] = x[i] + eps * mg[i] + s2e * lx[i];
        orc_grad(tg, y, gy);
        for (int64_t i = 0; i < D; ++i) r[i] = y[i] - (x[i] + eps * mg[i]);
        const double lq_yx = -0.5 * quad_minv(D, L, r, t2) / (2 * eps) - c - 0.5 * logdet;
        lower_t_mv(D, L, gy, tmp);
        lower_mv(D, L, tmp, mg);           /* M g_y */
        for (int64_t i = 0; i < D; ++i) r[i] = x[i] - (y[i] + eps * mg[i]);
        const double lq_xy = -0.5 * quad_minv(D, L, r, t2) / (2 * eps) - c - 0.5 * logdet;
        const double la = (orc_logp(tg, y) + lq_xy) - (orc_logp(tg, x) + lq_yx);
        const int acc = log(u[t]) < la;
        if (acc) memcpy(x, y, sizeof(double) * D);
        memcpy(S + t * D, x, sizeof(double) * D);
        if (accepted) accepted[t] = acc;
        if (logalpha) logalpha[t] = la;
    }
    free(b);
}

/* Per-column fused forward + surrogate JVP in the batched operation order of
 * mala_step_batched_fwd_and_jvp! (MALA.jl:577-626), identity mass matrix. */
static void fwd_jvp_col(const orc_target* tg, double eps, const double* x, const double* xi,
                        double u, const double* z, double* f, double* jv, mala_ws* w) {
    int64_t D = tg->D;
    double la = mala_forward(tg, eps, x, xi, w);
    double logu = log(u);
    double g = 1.0 / (1.0 + exp(-(la - logu)));
    int acc = logu < la;
    for (int64_t i = 0; i < D; ++i) f[i] = acc ? w->y[i] : x[i];
    orc_hvp(tg, x, z, w->hvx);
    for (int64_t i = 0; i < D; ++i) w->w[i] = z[i] + eps * w->hvx[i];
    orc_hvp(tg, w->y, w->w, w->hvy);
    for (int64_t i = 0; i < D; ++i) {
        w->r[i] = x[i] - w->y[i] - eps * w->gy[i];
        w->dr[i] = z[i] - w->w[i] - eps * w->hvy[i];
    }
    double dot1 = 0, dot2 = 0, dot3 = 0;
    for (int64_t i = 0; i < D; ++i) dot3 += w->r[i] * w->dr[i];
    for (int64_t i = 0; i < D; ++i) dot1 += w->gy[i] * w->w[i];
    for (int64_t i = 0; i < D; ++i) dot2 += w->gx[i] * z[i];
    double dla = dot1 - dot2 - (1.0 / (2 * eps)) * dot3;
    double dg = g * (1.0 - g) * dla;
    for (int64_t i = 0; i < D; ++i) jv[i] = (acc ? w->w[i] : z[i]) + (w->y[i] - x[i]) * dg;
}

/* mala_step_taped_and_jvp! (MALA.jl:732-797) */
void orc_fwd_and_jvp(const orc_target* tg, double eps, const double* x, const double* xi,
                     double u, const double* v, double* f, double* jv) {
    mala_ws w;
    ws_alloc(&w, tg->D);
    fwd_jvp_col(tg, eps, x, xi, u, v, f, jv, &w);
    ws_free(&w);
}

/* mala_step_batched_fwd_and_jvp! (MALA.jl:556-628) over T columns. */
void orc_fwd_and_jvp_batched(const orc_target* tg, double eps, int64_t T, const double* X,
                             const double* Xi, const double* u, const double* Z, double* FT,
                             double* Jt, int32_t nthreads) {
    int64_t D = tg->D;
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
    {
        mala_ws w;
        ws_alloc(&w, D);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t t = 0; t < T; ++t)
            fwd_jvp_col(tg, eps, X + t * D, Xi + t * D, u[t], Z + t * D, FT + t * D,
                        Jt + t * D, &w);
        ws_free(&w);
    }
    (void)nthreads;
}

/* Dense surrogate Jacobian (new: the reference rejects :full, DEER.jl:465-466):
 * J = a (I + eps H_x) + (1-a) I + g(1-g) (y - x) grad(logalpha)^T with
 * grad(logalpha) = (I+eps H_x) g_y - g_x - (1/2eps)[r - (I+eps H_x)(I+eps H_y) r],
 * the matrix whose action is the JVP of MALA.jl:768-795. J is D x D column-major. */
void orc_jac_full(const orc_target* tg, double eps, const double* x, const double* xi,
                  double u, double* f, double* J) {
    int64_t D = tg->D;
    mala_ws w;
    ws_alloc(&w, D);
    double la = mala_forward(tg, eps, x, xi, &w);
    double logu = log(u);
    double g = 1.0 / (1.0 + exp(-(la - logu)));
    int acc = logu < la;
    for (int64_t i = 0; i < D; ++i) f[i] = acc ? w.y[i] : x[i];
    double* gl = (double*)malloc(sizeof(double) * 4 * D);
    double *q = gl + D, *tmp = gl + 2 * D, *e = gl + 3 * D;
    for (int64_t i = 0; i < D; ++i) w.r[i] = x[i] - w.y[i] - eps * w.gy[i];
    orc_hvp(tg, x, w.gy, tmp);
    for (int64_t i = 0; i < D; ++i) gl[i] = w.gy[i] + eps * tmp[i] - w.gx[i];
    orc_hvp(tg, w.y, w.r, tmp);
    for (int64_t i = 0; i < D; ++i) q[i] = w.r[i] + eps * tmp[i];
    orc_hvp(tg, x, q, tmp);
    for (int64_t i = 0; i < D; ++i) gl[i] -= (1.0 / (2 * eps)) * (w.r[i] - (q[i] + eps * tmp[i]));
    double c = g * (1.0 - g);
    for (int64_t j = 0; j < D; ++j) {
        for (int64_t i = 0; i < D; ++i) e[i] = (i == j) ? 1.0 : 0.0;
        orc_hvp(tg, x, e, tmp);
        for (int64_t i = 0; i < D; ++i) {
            double base = (acc ? (e[i] + eps * tmp[i]) : e[i]);
            J[j * D + i] = base + (w.y[i] - x[i]) * c * gl[j];
        }
    }
    free(gl);
    ws_free(&w);
}

/* ========================================================================= */
/* Affine scans (DEERScan.jl).                                                */
/* ========================================================================= */

/* solve_affine_seq! (DEERScan.jl:51-68) */
void orc_scan_seq(int64_t D, int64_t T, const double* A, const double* B, const double* s0,
                  double* S) {
    if (T == 0) return;
    for (int64_t i = 0; i < D; ++i) S[i] = A[i] * s0[i] + B[i];
    for (int64_t t = 1; t < T; ++t)
        for (int64_t i = 0; i < D; ++i)
            S[t * D + i] = A[t * D + i] * S[(t - 1) * D + i] + B[t * D + i];
}

/* solve_affine_scan_diag! (DEERScan.jl:102-173): Hillis-Steele doubling with
 * ping-pong buffers; ws holds 4*D*T doubles. */
void orc_scan_doubling(int64_t D, int64_t T, const double* A, const double* B,
                       const double* s0, double* S, double* ws) {
    if (T == 0) return;
    int64_t n = D * T;
    double *al = ws, *be = ws + n, *aln = ws + 2 * n, *ben = ws + 3 * n;
    memcpy(al, A, sizeof(double) * n);
    memcpy(be, B, sizeof(double) * n);
    int64_t off = 1;
    while (off < T) {
        int last = (off << 1) >= T;
        if (!last) {
            memcpy(aln, al, sizeof(double) * D * off);
            memcpy(ben, be, sizeof(double) * D * off);
        }
        for (int64_t t = off; t < T; ++t)
            for (int64_t i = 0; i < D; ++i) {
                double a2 = al[t * D + i];
                aln[t * D + i] = a2 * al[(t - off) * D + i];
                ben[t * D + i] = a2 * be[(t - off) * D + i] + be[t * D + i];
            }
        if (last) {
            for (int64_t t = 0; t < off; ++t)
                for (int64_t i = 0; i < D; ++i)
                    S[t * D + i] = al[t * D + i] * s0[i] + be[t * D + i];
            for (int64_t t = off; t < T; ++t)
                for (int64_t i = 0; i < D; ++i)
                    S[t * D + i] = aln[t * D + i] * s0[i] + ben[t * D + i];
            return;
        }
        double* tp = al; al = aln; aln = tp;
        tp = be; be = ben; ben = tp;
        off <<= 1;
    }
    for (int64_t t = 0; t < T; ++t)
        for (int64_t i = 0; i < D; ++i) S[t * D + i] = al[t * D + i] * s0[i] + be[t * D + i];
}

/* affine_scan_residual (DEERScan.jl:203-219) */
double orc_scan_residual(int64_t D, int64_t T, const double* S, const double* A,
                         const double* B, const double* s0) {
    double r = 0;
    for (int64_t t = 0; t < T; ++t)
        for (int64_t i = 0; i < D; ++i) {
            double prev = t == 0 ? s0[i] : S[(t - 1) * D + i];
            double e = fabs(S[t * D + i] - (A[t * D + i] * prev + B[t * D + i]));
            if (e > r) r = e;
        }
    return r;
}

/* Dense counterpart (new): s_t = J_t s_{t-1} + b_t, J_t D x D column-major. */
void orc_scan_dense_seq(int64_t D, int64_t T, const double* J, const double* B,
                        const double* s0, double* S) {
    for (int64_t t = 0; t < T; ++t) {
        const double* prev = t == 0 ? s0 : S + (t - 1) * D;
        const double* Jt = J + t * D * D;
        for (int64_t i = 0; i < D; ++i) S[t * D + i] = B[t * D + i];
        for (int64_t j = 0; j < D; ++j)
            for (int64_t i = 0; i < D; ++i) S[t * D + i] += Jt[j * D + i] * prev[j];
    }
}

/* ========================================================================= */
/* DEER.                                                                      */
/* ========================================================================= */

/* One DEER update (DEER.jl:375-475) over columns [t_lo, t_hi) of the trajectory:
 * x_bar = [s_lo, S_in[:, t_lo:t_hi-2]], Jacobian estimate, scan from s_lo, damping.
 * A_out/B_out (D x (t_hi-t_lo)) may be NULL. */
static int deer_update_range(const orc_target* tg, const orc_deer_params* p, int64_t T,
                             int64_t t_lo, int64_t t_hi, const double* s_lo,
                             const double* S_in, const double* Xi, const double* u,
                             uint64_t seed, uint64_t block, int32_t iter, double* S_out,
                             double* A_out, double* B_out) {
    int64_t D = tg->D, W = t_hi - t_lo;
    if (!(p->damping > 0 && p->damping <= 1)) return 1;
    if (p->probes < 1) return 1;
    double* Xbar = (double*)malloc(sizeof(double) * D * W);
    double* A = A_out ? A_out : (double*)malloc(sizeof(double) * D * W);
    double* B = B_out ? B_out : (double*)malloc(sizeof(double) * D * W);
    memcpy(Xbar, s_lo, sizeof(double) * D);
    if (W > 1) memcpy(Xbar + D, S_in + t_lo * D, sizeof(double) * D * (W - 1));
    const double* XiW = Xi + t_lo * D;
    const double* uW = u + t_lo;
    int nt = p->nthreads;
    (void)nt;
    int rc = 0;
    if (p->jacobian == ORC_JAC_STOCH_DIAG) {
        /* batched branch (DEER.jl:398-419); the per-t branch (:433-455) is the same
         * arithmetic column by column, so one code path serves both. */
        double* Zfull = (double*)malloc(sizeof(double) * D * T);
        double* FT = (double*)malloc(sizeof(double) * D * W);
        double* Jt = (double*)malloc(sizeof(double) * D * W);
        for (int32_t k = 0; k < p->probes; ++k) {
            orc_probe(seed, block, iter, k, D, T, Zfull);
            const double* Z = Zfull + t_lo * D;
            orc_fwd_and_jvp_batched(tg, p->eps, W, Xbar, XiW, uW, Z, FT, Jt, p->nthreads);
            for (int64_t e = 0; e < D * W; ++e) {
                if (k == 0) A[e] = Z[e] * Jt[e];
                else A[e] += Z[e] * Jt[e];
            }
        }
        if (p->probes > 1)
            for (int64_t e = 0; e < D * W; ++e) A[e] *= 1.0 / p->probes;
        for (int64_t e = 0; e < D * W; ++e) B[e] = FT[e] - A[e] * Xbar[e];
        free(Zfull); free(FT); free(Jt);
        if (p->scan_doubling) {
            double* ws = (double*)malloc(sizeof(double) * 4 * D * W);
            orc_scan_doubling(D, W, A, B, s_lo, S_out + t_lo * D, ws);
            free(ws);
        } else {
            orc_scan_seq(D, W, A, B, s_lo, S_out + t_lo * D);
        }
    } else if (p->jacobian == ORC_JAC_DIAG) {
        /* per-t branch with jac_diag_via_jvps (DEER.jl:456-462, 327-342): D JVPs
         * with basis vectors per column. */
#ifdef _OPENMP
        int nth = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nth)
#endif
        {
            double* ei = (double*)malloc(sizeof(double) * D);
            double* jv = (double*)malloc(sizeof(double) * D);
            double* ft = (double*)malloc(sizeof(double) * D);
            double* fd = (double*)malloc(sizeof(double) * D);
            mala_ws w;
            ws_alloc(&w, D);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (int64_t t = 0; t < W; ++t) {
                const double* xb = Xbar + t * D;
                int32_t acc;
                orc_mala_step(tg, p->eps, xb, XiW + t * D, uW[t], ft, &acc);
                for (int64_t i = 0; i < D; ++i) ei[i] = 0.0;
                for (int64_t i = 0; i < D; ++i) {
                    ei[i] = 1.0;
                    fwd_jvp_col(tg, p->eps, xb, XiW + t * D, uW[t], ei, fd, jv, &w);
                    A[t * D + i] = jv[i];
                    ei[i] = 0.0;
                }
                for (int64_t i = 0; i < D; ++i) B[t * D + i] = ft[i] - A[t * D + i] * xb[i];
            }
            ws_free(&w);
            free(ei); free(jv); free(ft); free(fd);
        }
        if (p->scan_doubling) {
            double* ws = (double*)malloc(sizeof(double) * 4 * D * W);
            orc_scan_doubling(D, W, A, B, s_lo, S_out + t_lo * D, ws);
            free(ws);
        } else {
            orc_scan_seq(D, W, A, B, s_lo, S_out + t_lo * D);
        }
    } else if (p->jacobian == ORC_JAC_FULL) {
        double* J = (double*)malloc(sizeof(double) * D * D * W);
        double* ft = (double*)malloc(sizeof(double) * D * W);
#ifdef _OPENMP
        int nth = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel for num_threads(nth) schedule(static)
#endif
        for (int64_t t = 0; t < W; ++t) {
            const double* xb = Xbar + t * D;
            orc_jac_full(tg, p->eps, xb, XiW + t * D, uW[t], ft + t * D, J + t * D * D);
            double* Bt = B + t * D;
            for (int64_t i = 0; i < D; ++i) Bt[i] = ft[t * D + i];
            for (int64_t j = 0; j < D; ++j)
                for (int64_t i = 0; i < D; ++i) Bt[i] -= J[t * D * D + j * D + i] * xb[j];
            for (int64_t i = 0; i < D; ++i) A[t * D + i] = J[t * D * D + i * D + i];
        }
        orc_scan_dense_seq(D, W, J, B, s_lo, S_out + t_lo * D);
        free(J); free(ft);
    } else {
        rc = 1;
    }
    if (rc == 0 && p->damping != 1.0) {
        for (int64_t e = t_lo * D; e < t_hi * D; ++e)
            S_out[e] = (1 - p->damping) * S_in[e] + p->damping * S_out[e];
    }
    free(Xbar);
    if (!A_out) free(A);
    if (!B_out) free(B);
    return rc;
}

int orc_deer_update(const orc_target* tg, const orc_deer_params* p, int64_t T,
                    const double* s0, const double* S_in, const double* Xi, const double* u,
                    uint64_t seed, uint64_t block, int32_t iter, double* S_out,
                    double* A_out, double* B_out) {
    return deer_update_range(tg, p, T, 0, T, s0, S_in, Xi, u, seed, block, iter, S_out,
                             A_out, B_out);
}

/* DEER.solve (DEER.jl:506-595).  With window > 0 (new; the reference only names
 * the sliding window, README.md:30) each sweep updates columns [t_lo, t_lo+W)
 * from s_{t_lo-1}; t_lo advances to the first column whose change exceeds the
 * tolerance scale.  window = 0 is exactly the reference loop. */
int orc_deer_solve(const orc_target* tg, const orc_deer_params* p, int64_t T,
                   const double* s0, const double* Xi, const double* u, uint64_t seed,
                   uint64_t block, double* S_out, orc_deer_info* info) {
    int64_t D = tg->D;
    if (p->maxiter < 1 || p->tol_abs < 0 || p->tol_rel < 0) return 1;
    if (!(p->damping > 0 && p->damping <= 1)) return 1;
    double* S = (double*)malloc(sizeof(double) * D * T);
    double* Sn = (double*)malloc(sizeof(double) * D * T);
    for (int64_t t = 0; t < T; ++t) memcpy(S + t * D, s0, sizeof(double) * D);
    memcpy(Sn, S, sizeof(double) * D * T);
    int converged = 0, iters = 0;
    double last = INFINITY;
    int64_t t_lo = 0;
    int64_t W = (p->window > 0 && p->window < T) ? p->window : T;
    int rc = 0;
    for (int32_t it = 0; it < p->maxiter; ++it) {
        iters = it + 1;
        int64_t t_hi = t_lo + W < T ? t_lo + W : T;
        const double* slo = t_lo == 0 ? s0 : S + (t_lo - 1) * D;
        memcpy(Sn, S, sizeof(double) * D * T);
        rc = deer_update_range(tg, p, T, t_lo, t_hi, slo, S, Xi, u, seed, block, it, Sn, NULL,
                               NULL);
        if (rc) break;
        double dmax = 0, smax = 0;
        for (int64_t e = t_lo * D; e < t_hi * D; ++e) {
            double d = fabs(Sn[e] - S[e]);
            if (d > dmax) dmax = d;
            double a = fabs(Sn[e]);
            if (a > smax) smax = a;
        }
        double scale = p->tol_abs + p->tol_rel * smax;
        double metric = dmax / scale;
        last = metric;
        double* tp = S; S = Sn; Sn = tp;
        if (W == T) {
            if (metric <= 1) { converged = 1; break; }
        } else {
            int64_t first_bad = t_hi;
            for (int64_t t = t_lo; t < t_hi && first_bad == t_hi; ++t)
                for (int64_t i = 0; i < D; ++i)
                    if (fabs(S[t * D + i] - Sn[t * D + i]) > scale) { first_bad = t; break; }
            t_lo = first_bad;
            if (t_lo >= T) { converged = 1; break; }
        }
    }
    memcpy(S_out, S, sizeof(double) * D * T);
    free(S); free(Sn);
    if (info) { info->iters = iters; info->converged = converged; info->metric = last; }
    return rc;
}
