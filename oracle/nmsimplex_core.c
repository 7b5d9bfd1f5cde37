/*
 * TEST INFRASTRUCTURE ONLY — FP64 restatement of the Nelder-Mead simplex
 * minimiser the reference's MLEwG fitter uses (GSL 1.16
 * gsl_multimin_fminimizer_nmsimplex2, reference source/Localization.cpp:
 * 657-724; GSL's source is not in the reference tree). Restated from the
 * published algorithm of that minimiser: the simplex starts at x and x + step
 * along each axis; each iteration reflects the worst corner through the
 * centroid of the others, expands (factor 2) if that is the new best, keeps the
 * reflection if it beats the second worst, otherwise contracts the worst
 * corner half-way (after accepting the reflection if it improved on the worst)
 * and, if that fails too, shrinks every corner half-way to the best one. The
 * simplex centre and its squared RMS size (the convergence measure) are
 * updated incrementally with each moved corner and recomputed after a shrink.
 * Vector kernels follow the reference BLAS definitions (dnrm2 by scaled sum of
 * squares, ddot and daxpy as plain loops).
 */
#include "nmsimplex_core.h"

#include <math.h>
#include <string.h>

double nm_dnrm2(const double *x, int n)
{
    if (n <= 0) return 0.0;
    if (n == 1) return fabs(x[0]);
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; i++) {
        if (x[i] != 0.0) {
            const double ax = fabs(x[i]);
            if (scale < ax) {
                ssq = 1.0 + ssq * (scale / ax) * (scale / ax);
                scale = ax;
            } else {
                ssq += (ax / scale) * (ax / scale);
            }
        }
    }
    return scale * sqrt(ssq);
}

static double ddot(const double *x, const double *y, int n)
{
    double r = 0.0;
    for (int i = 0; i < n; i++) r += x[i] * y[i];
    return r;
}

static void daxpy(double a, const double *x, double *y, int n)
{
    for (int i = 0; i < n; i++) y[i] += a * x[i];
}

static void compute_center(nm_state *s)
{
    const int n = s->n, P = n + 1;
    for (int j = 0; j < n; j++) s->center[j] = 0.0;
    for (int i = 0; i < P; i++) daxpy(1.0, s->x1 + i * n, s->center, n);
    const double alpha = 1.0 / P;
    for (int j = 0; j < n; j++) s->center[j] *= alpha;
}

static double compute_size(nm_state *s)
{
    const int n = s->n, P = n + 1;
    double ss = 0.0;
    for (int i = 0; i < P; i++) {
        for (int j = 0; j < n; j++) s->ws1[j] = s->x1[i * n + j];
        daxpy(-1.0, s->center, s->ws1, n);
        const double t = nm_dnrm2(s->ws1, n);
        ss += t * t;
    }
    s->S2 = ss / P;
    return sqrt(ss / P);
}

static double try_corner_move(double coeff, nm_state *s, int corner, double *xc, nm_fn f, void *par)
{
    const int n = s->n, P = n + 1;
    const double alpha = (1 - coeff) * P / (P - 1.0);
    const double beta = (P * coeff - 1.0) / (P - 1.0);
    for (int j = 0; j < n; j++) xc[j] = s->center[j] * alpha;
    daxpy(beta, s->x1 + corner * n, xc, n);
    return f(xc, par);
}

static void update_point(nm_state *s, int i, const double *x, double val)
{
    const int n = s->n, P = n + 1;
    const double *xo = s->x1 + i * n;
    for (int j = 0; j < n; j++) s->delta[j] = x[j];
    daxpy(-1.0, xo, s->delta, n);
    for (int j = 0; j < n; j++) s->xmc[j] = xo[j];
    daxpy(-1.0, s->center, s->xmc, n);
    const double d = nm_dnrm2(s->delta, n);
    const double xmcd = ddot(s->xmc, s->delta, n);
    s->S2 += (2.0 / P) * xmcd + ((P - 1.0) / P) * (d * d / P);
    const double alpha = 1.0 / P;
    daxpy(-alpha, xo, s->center, n);
    daxpy(alpha, x, s->center, n);
    for (int j = 0; j < n; j++) s->x1[i * n + j] = x[j];
    s->y1[i] = val;
}

static int contract_by_best(nm_state *s, int best, double *xc, nm_fn f, void *par)
{
    const int n = s->n, P = n + 1;
    int status = 0;
    for (int i = 0; i < P; i++) {
        if (i == best) continue;
        for (int j = 0; j < n; j++) s->x1[i * n + j] = 0.5 * (s->x1[i * n + j] + s->x1[best * n + j]);
        for (int j = 0; j < n; j++) xc[j] = s->x1[i * n + j];
        const double v = f(xc, par);
        s->y1[i] = v;
        if (!isfinite(v)) status = NM_EBADFUNC;
    }
    compute_center(s);
    compute_size(s);
    return status;
}

int nm_set(nm_state *s, int n, nm_fn f, void *par, const double *x, const double *step, double *size)
{
    if (n < 1 || n > NM_NMAX) return NM_EINVAL;
    s->n = n;
    double v = f(x, par);
    if (!isfinite(v)) return NM_EBADFUNC;
    for (int j = 0; j < n; j++) s->x1[j] = x[j];
    s->y1[0] = v;
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) s->ws1[j] = x[j];
        s->ws1[i] = x[i] + step[i];
        v = f(s->ws1, par);
        if (!isfinite(v)) return NM_EBADFUNC;
        for (int j = 0; j < n; j++) s->x1[(i + 1) * n + j] = s->ws1[j];
        s->y1[i + 1] = v;
    }
    compute_center(s);
    *size = compute_size(s);
    return 0;
}

int nm_iterate(nm_state *s, nm_fn f, void *par, double *x, double *size, double *fval)
{
    const int n = s->n, P = n + 1;
    double *xc = s->ws1, *xc2 = s->ws2;
    int hi = 0, lo = 0, s_hi = 1;
    double dhi = s->y1[0], dlo = s->y1[0], ds_hi = s->y1[1];
    for (int i = 1; i < P; i++) {
        const double v = s->y1[i];
        if (v < dlo) {
            dlo = v;
            lo = i;
        } else if (v > dhi) {
            ds_hi = dhi;
            s_hi = hi;
            dhi = v;
            hi = i;
        } else if (v > ds_hi) {
            ds_hi = v;
            s_hi = i;
        }
    }
    const double val = try_corner_move(-1.0, s, hi, xc, f, par);
    if (isfinite(val) && val < s->y1[lo]) {
        const double val2 = try_corner_move(-2.0, s, hi, xc2, f, par);
        if (isfinite(val2) && val2 < s->y1[lo]) update_point(s, hi, xc2, val2);
        else update_point(s, hi, xc, val);
    } else if (!isfinite(val) || val > s->y1[s_hi]) {
        if (isfinite(val) && val <= s->y1[hi]) update_point(s, hi, xc, val);
        const double val2 = try_corner_move(0.5, s, hi, xc2, f, par);
        if (isfinite(val2) && val2 <= s->y1[hi]) {
            update_point(s, hi, xc2, val2);
        } else {
            if (contract_by_best(s, lo, xc, f, par) != 0) return NM_EFAILED;
        }
    } else {
        update_point(s, hi, xc, val);
    }
    /* lowest corner (first minimum) as the current point */
    lo = 0;
    for (int i = 1; i < P; i++)
        if (s->y1[i] < s->y1[lo]) lo = i;
    for (int j = 0; j < n; j++) x[j] = s->x1[lo * n + j];
    *fval = s->y1[lo];
    if (s->S2 > 0) *size = sqrt(s->S2);
    else *size = compute_size(s);
    return 0;
}
