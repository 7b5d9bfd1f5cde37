/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle (see lmsder_core.h for the rules and
 * the provenance of the algorithm). FP64 throughout; build without -ffast-math.
 *
 * Layout conventions: every matrix is row-major. J and the QR workspace r are
 * n x p with row stride p. After the pivoted QR, the upper triangle of the top
 * p x p block of r holds R, the Householder vectors sit below the diagonal and
 * perm[j] is the original column placed in position j, so J P = Q R.
 */
#include "lmsder_core.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define RR(i, j) r[(i) * p + (j)]

double lmc_enorm(const double *v, size_t n, size_t stride)
{
    double scale = 0.0, ssq = 1.0;
    if (n == 0) return 0.0;
    if (n == 1) return fabs(v[0]);
    for (size_t i = 0; i < n; i++) {
        double xi = v[i * stride];
        if (xi != 0.0) {
            double ax = fabs(xi);
            if (scale < ax) {
                double t = scale / ax;
                ssq = 1.0 + ssq * t * t;
                scale = ax;
            } else {
                double t = ax / scale;
                ssq += t * t;
            }
        }
    }
    return scale * sqrt(ssq);
}

static double scaled_enorm(const double *d, const double *x, size_t p)
{
    double tmp[16];
    for (size_t i = 0; i < p; i++) tmp[i] = d[i] * x[i];
    return lmc_enorm(tmp, p, 1);
}

/* Householder reflector for v[0..m-1] (stride s): on return v[0] = beta and
 * v[1..] holds the reflector with an implicit leading 1; returns tau. */
static double householder_make(double *v, size_t m, size_t s)
{
    if (m == 1) return 0.0;
    double xnorm = lmc_enorm(v + s, m - 1, s);
    if (xnorm == 0.0) return 0.0;
    double alpha = v[0];
    double beta = -(alpha >= 0.0 ? 1.0 : -1.0) * hypot(alpha, xnorm);
    double tau = (beta - alpha) / beta;
    double den = alpha - beta;
    if (fabs(den) > DBL_MIN) {
        double inv = 1.0 / den;
        for (size_t i = 1; i < m; i++) v[i * s] *= inv;
    } else {
        double a = DBL_EPSILON / den, b = 1.0 / DBL_EPSILON;
        for (size_t i = 1; i < m; i++) v[i * s] *= a;
        for (size_t i = 1; i < m; i++) v[i * s] *= b;
    }
    v[0] = beta;
    return tau;
}

/* Apply (I - tau v v^T) from the left to the m x c block M (row stride ld);
 * v has stride vs and an implicit v[0] = 1. */
static void householder_apply(double tau, const double *v, size_t vs, double *M,
                              size_t m, size_t c, size_t ld)
{
    if (tau == 0.0) return;
    for (size_t j = 0; j < c; j++) {
        double wj = M[j];
        for (size_t i = 1; i < m; i++) wj += M[i * ld + j] * v[i * vs];
        M[j] -= tau * wj;
        for (size_t i = 1; i < m; i++) M[i * ld + j] -= tau * v[i * vs] * wj;
    }
}

/* Column-pivoted Householder QR of the n x p row-major matrix A (in place). */
static void qrpt_decomp(double *A, size_t n, size_t p, double *tau, size_t *perm, double *norm)
{
    for (size_t j = 0; j < p; j++) {
        perm[j] = j;
        norm[j] = lmc_enorm(A + j, n, p);
    }
    size_t kmin = n < p ? n : p;
    for (size_t i = 0; i < kmin; i++) {
        double best = norm[i];
        size_t kmax = i;
        for (size_t j = i + 1; j < p; j++) {
            if (norm[j] > best) {
                best = norm[j];
                kmax = j;
            }
        }
        if (kmax != i) {
            for (size_t row = 0; row < n; row++) {
                double t = A[row * p + i];
                A[row * p + i] = A[row * p + kmax];
                A[row * p + kmax] = t;
            }
            size_t tp = perm[i]; perm[i] = perm[kmax]; perm[kmax] = tp;
            double tn = norm[i]; norm[i] = norm[kmax]; norm[kmax] = tn;
        }
        double *v = A + i * p + i;
        tau[i] = householder_make(v, n - i, p);
        if (i + 1 < p) householder_apply(tau[i], v, p, v + 1, n - i, p - (i + 1), p);
        if (i + 1 < n) {
            for (size_t j = i + 1; j < p; j++) {
                double xn = norm[j];
                if (xn > 0.0) {
                    double y;
                    double t = A[i * p + j] / xn;
                    if (fabs(t) >= 1.0) y = 0.0;
                    else y = xn * sqrt(1.0 - t * t);
                    if (fabs(y / xn) < sqrt(20.0) * sqrt(DBL_EPSILON))
                        y = lmc_enorm(A + (i + 1) * p + j, n - (i + 1), p);
                    norm[j] = y;
                }
            }
        }
    }
}

/* v <- Q^T v for the reflectors stored in A (n x p). */
static void qr_qtvec(const double *A, size_t n, size_t p, const double *tau, double *v)
{
    size_t kmin = n < p ? n : p;
    for (size_t i = 0; i < kmin; i++) {
        if (tau[i] == 0.0) continue;
        double wj = v[i];
        for (size_t k = i + 1; k < n; k++) wj += A[k * p + i] * v[k];
        v[i] -= tau[i] * wj;
        for (size_t k = i + 1; k < n; k++) v[k] -= tau[i] * A[k * p + i] * wj;
    }
}

static void compute_diag(const double *J, size_t n, size_t p, double *diag)
{
    for (size_t j = 0; j < p; j++) {
        double sum = 0.0;
        for (size_t i = 0; i < n; i++) sum += J[i * p + j] * J[i * p + j];
        if (sum == 0.0) sum = 1.0;
        diag[j] = sqrt(sum);
    }
}

static void update_diag(const double *J, size_t n, size_t p, double *diag)
{
    for (size_t j = 0; j < p; j++) {
        double sum = 0.0;
        for (size_t i = 0; i < n; i++) sum += J[i * p + j] * J[i * p + j];
        if (sum == 0.0) sum = 1.0;
        double cn = sqrt(sum);
        if (cn > diag[j]) diag[j] = cn;
    }
}

static size_t count_nsing(const double *r, size_t p)
{
    size_t i = 0;
    while (i < p && RR(i, i) != 0.0) i++;
    return i;
}

/* Gauss-Newton direction: least-squares solution of R P^T x = qtf. */
static void newton_direction(const double *r, size_t p, const size_t *perm,
                             const double *qtf, double *x, double *tmp)
{
    size_t nsing = count_nsing(r, p);
    for (size_t i = 0; i < p; i++) tmp[i] = (i < nsing) ? qtf[i] : 0.0;
    for (size_t jj = nsing; jj > 0; jj--) {
        size_t j = jj - 1;
        double t = tmp[j] / RR(j, j);
        tmp[j] = t;
        for (size_t i = 0; i < j; i++) tmp[i] -= RR(i, j) * t;
    }
    for (size_t i = 0; i < p; i++) x[perm[i]] = tmp[i];
}

/* w = R^-T (P^T D^2 x) / |D x|, or zero when R is singular. */
static void newton_bound(const double *r, size_t p, const double *x, double dxnorm,
                         const size_t *perm, const double *diag, double *w)
{
    if (count_nsing(r, p) < p) {
        for (size_t i = 0; i < p; i++) w[i] = 0.0;
        return;
    }
    for (size_t i = 0; i < p; i++) {
        size_t pi = perm[i];
        w[i] = diag[pi] * (diag[pi] * x[pi]) / dxnorm;
    }
    for (size_t j = 0; j < p; j++) {
        double sum = 0.0;
        for (size_t i = 0; i < j; i++) sum += RR(i, j) * w[i];
        w[j] = (w[j] - sum) / RR(j, j);
    }
}

/* g = D^-1 P R^T qtf, i.e. the scaled gradient J^T f / D in pivoted order. */
static void gradient_direction(const double *r, size_t p, const size_t *perm,
                               const double *qtf, const double *diag, double *g)
{
    for (size_t j = 0; j < p; j++) {
        double sum = 0.0;
        for (size_t i = 0; i <= j; i++) sum += RR(i, j) * qtf[i];
        g[j] = sum / diag[perm[j]];
    }
}

/* Same as newton_bound but through the factor S of the damped system, whose
 * strict upper triangle qrsolv left (transposed) below the diagonal of r. */
static void newton_correction(const double *r, size_t p, const double *sdiag,
                              const size_t *perm, const double *x, double dxnorm,
                              const double *diag, double *w)
{
    for (size_t i = 0; i < p; i++) {
        size_t pi = perm[i];
        w[i] = diag[pi] * (diag[pi] * x[pi] / dxnorm);
    }
    for (size_t j = 0; j < p; j++) {
        double t = w[j] / sdiag[j];
        w[j] = t;
        for (size_t i = j + 1; i < p; i++) w[i] -= RR(i, j) * t;
    }
}

/* Solve min |R P^T x - qtf|^2 + lambda^2 |D x|^2 by Givens rotations. */
static void qrsolv(double *r, size_t p, const size_t *perm, double lambda,
                   const double *diag, const double *qtb, double *x,
                   double *sdiag, double *wa)
{
    for (size_t j = 0; j < p; j++) {
        for (size_t i = j + 1; i < p; i++) RR(i, j) = RR(j, i);
        x[j] = RR(j, j);
        wa[j] = qtb[j];
    }
    for (size_t j = 0; j < p; j++) {
        double d = lambda * diag[perm[j]];
        if (d == 0.0) continue;
        sdiag[j] = d;
        for (size_t k = j + 1; k < p; k++) sdiag[k] = 0.0;
        double qtbpj = 0.0;
        for (size_t k = j; k < p; k++) {
            double sk = sdiag[k];
            if (sk == 0.0) continue;
            double rkk = RR(k, k), sn, cs;
            if (fabs(rkk) < fabs(sk)) {
                double cot = rkk / sk;
                sn = 0.5 / sqrt(0.25 + 0.25 * cot * cot);
                cs = sn * cot;
            } else {
                double tn = sk / rkk;
                cs = 0.5 / sqrt(0.25 + 0.25 * tn * tn);
                sn = cs * tn;
            }
            double wak = wa[k];
            RR(k, k) = cs * rkk + sn * sk;
            wa[k] = cs * wak + sn * qtbpj;
            qtbpj = -sn * wak + cs * qtbpj;
            for (size_t i = k + 1; i < p; i++) {
                double rik = RR(i, k), si = sdiag[i];
                RR(i, k) = cs * rik + sn * si;
                sdiag[i] = -sn * rik + cs * si;
            }
        }
        double rjj = RR(j, j);
        sdiag[j] = rjj;
        RR(j, j) = x[j];
    }
    size_t nsing = p;
    for (size_t j = 0; j < p; j++) {
        if (sdiag[j] == 0.0) {
            nsing = j;
            break;
        }
    }
    for (size_t j = nsing; j < p; j++) wa[j] = 0.0;
    for (size_t k = 0; k < nsing; k++) {
        size_t j = nsing - 1 - k;
        double sum = 0.0;
        for (size_t i = j + 1; i < nsing; i++) sum += RR(i, j) * wa[i];
        wa[j] = (wa[j] - sum) / sdiag[j];
    }
    for (size_t j = 0; j < p; j++) x[perm[j]] = wa[j];
}

/* Levenberg-Marquardt parameter for the trust-region radius delta. */
static void lmpar(lmc_state *s, double *x_out)
{
    const size_t p = s->p;
    double *r = s->r;
    const double delta = s->delta;
    double par = s->par;
    double dxnorm, gnorm, fp, fp_old, par_lower, par_upper, par_c;
    size_t iter = 0;

    newton_direction(r, p, s->perm, s->qtf, s->newton, s->work1);
    dxnorm = scaled_enorm(s->diag, s->newton, p);
    fp = dxnorm - delta;
    if (fp <= 0.1 * delta) {
        memcpy(x_out, s->newton, p * sizeof(double));
        s->par = 0.0;
        return;
    }
    newton_bound(r, p, s->newton, dxnorm, s->perm, s->diag, s->w);
    {
        double wnorm = lmc_enorm(s->w, p, 1);
        double phider = wnorm * wnorm;
        par_lower = (wnorm > 0.0) ? fp / (delta * phider) : 0.0;
    }
    gradient_direction(r, p, s->perm, s->qtf, s->diag, s->gradient);
    gnorm = lmc_enorm(s->gradient, p, 1);
    par_upper = gnorm / delta;
    if (par_upper == 0.0) par_upper = DBL_MIN / (delta < 0.1 ? delta : 0.1);
    if (par > par_upper) par = par_upper;
    else if (par < par_lower) par = par_lower;
    if (par == 0.0) par = gnorm / dxnorm;

    for (;;) {
        iter++;
        if (par == 0.0) par = (0.001 * par_upper > DBL_MIN) ? 0.001 * par_upper : DBL_MIN;
        qrsolv(r, p, s->perm, sqrt(par), s->diag, s->qtf, x_out, s->sdiag, s->work1);
        s->n_lambda_trials++;
        dxnorm = scaled_enorm(s->diag, x_out, p);
        fp_old = fp;
        fp = dxnorm - delta;
        if (fabs(fp) <= 0.1 * delta) break;
        if (par_lower == 0.0 && fp <= fp_old && fp_old < 0.0) break;
        if (iter == 10) break;
        newton_correction(r, p, s->sdiag, s->perm, x_out, dxnorm, s->diag, s->w);
        {
            double wnorm = lmc_enorm(s->w, p, 1);
            par_c = fp / (delta * wnorm * wnorm);
        }
        if (fp > 0.0) {
            if (par > par_lower) par_lower = par;
        } else if (fp < 0.0) {
            if (par < par_upper) par_upper = par;
        }
        par = (par_lower > par + par_c) ? par_lower : par + par_c;
    }
    s->par = par;
}

int lmc_alloc(lmc_state *s, size_t n, size_t p)
{
    memset(s, 0, sizeof(*s));
    if (p == 0 || p > 16 || n < p) return -1;
    s->n = n;
    s->p = p;
    size_t total = 3 * n * p + 4 * n + 16 * p;
    double *blk = (double *)calloc(total, sizeof(double));
    s->perm = (size_t *)calloc(p, sizeof(size_t));
    if (!blk || !s->perm) {
        free(blk);
        free(s->perm);
        return -1;
    }
    double *q = blk;
    s->J = q; q += n * p;
    s->r = q; q += n * p;
    q += n * p; /* spare */
    s->fvec = q; q += n;
    s->f_trial = q; q += n;
    s->qtf = q; q += n;
    q += n; /* spare */
    s->x = q; q += p;
    s->dx = q; q += p;
    s->tau = q; q += p;
    s->diag = q; q += p;
    s->newton = q; q += p;
    s->gradient = q; q += p;
    s->x_trial = q; q += p;
    s->sdiag = q; q += p;
    s->rptdx = q; q += p;
    s->w = q; q += p;
    s->work1 = q; q += p;
    return 0;
}

void lmc_free(lmc_state *s)
{
    free(s->J);
    free(s->perm);
    memset(s, 0, sizeof(*s));
}

int lmc_set(lmc_state *s, lmc_f_fn f, lmc_df_fn df, void *params, const double *x0)
{
    const size_t n = s->n, p = s->p;
    s->f = f;
    s->df = df;
    s->params = params;
    memcpy(s->x, x0, p * sizeof(double));
    int status = f(s->x, params, s->fvec);
    if (status == 0) status = df(s->x, params, s->J);
    s->n_df_evals++;
    if (status) return status;
    s->par = 0.0;
    s->iter = 1;
    s->fnorm = lmc_enorm(s->fvec, n, 1);
    for (size_t i = 0; i < p; i++) s->dx[i] = 0.0;
    compute_diag(s->J, n, p, s->diag);
    s->xnorm = scaled_enorm(s->diag, s->x, p);
    s->delta = (s->xnorm > 0.0) ? 100.0 * s->xnorm : 100.0;
    memcpy(s->r, s->J, n * p * sizeof(double));
    qrpt_decomp(s->r, n, p, s->tau, s->perm, s->work1);
    for (size_t i = 0; i < p; i++) s->rptdx[i] = s->w[i] = 0.0;
    for (size_t i = 0; i < n; i++) s->f_trial[i] = 0.0;
    return 0;
}

int lmc_iterate(lmc_state *s)
{
    const size_t n = s->n, p = s->p;
    double *r = s->r;
    const double p1 = 0.1, p25 = 0.25, p5 = 0.5, p75 = 0.75, p0001 = 0.0001;
    double gnorm;
    int inner = 0;

    if (s->fnorm == 0.0) return LMC_SUCCESS;

    memcpy(s->qtf, s->fvec, n * sizeof(double));
    qr_qtvec(r, n, p, s->tau, s->qtf);
    gradient_direction(r, p, s->perm, s->qtf, s->diag, s->gradient);
    {
        size_t imax = 0;
        double best = fabs(s->gradient[0]);
        for (size_t i = 1; i < p; i++) {
            if (fabs(s->gradient[i]) > best) {
                best = fabs(s->gradient[i]);
                imax = i;
            }
        }
        gnorm = fabs(s->gradient[imax] / s->fnorm);
    }

    for (;;) {
        inner++;
        lmpar(s, s->dx);
        s->n_inner_trials++;
        for (size_t i = 0; i < p; i++) s->dx[i] = -s->dx[i];
        for (size_t i = 0; i < p; i++) s->x_trial[i] = s->x[i] + s->dx[i];
        double pnorm = scaled_enorm(s->diag, s->dx, p);
        if (s->iter == 1 && pnorm < s->delta) s->delta = pnorm;

        int status = s->f(s->x_trial, s->params, s->f_trial);
        s->n_f_evals++;
        if (status) return LMC_EBADFUNC;
        double fnorm1 = lmc_enorm(s->f_trial, n, 1);

        double actred = -1.0;
        if (p1 * fnorm1 < s->fnorm) {
            double u = fnorm1 / s->fnorm;
            actred = 1.0 - u * u;
        }

        for (size_t i = 0; i < p; i++) {
            double sum = 0.0;
            for (size_t j = i; j < p; j++) sum += RR(i, j) * s->dx[s->perm[j]];
            s->rptdx[i] = sum;
        }
        double fnorm1p = lmc_enorm(s->rptdx, p, 1);
        double t1 = fnorm1p / s->fnorm;
        double t2 = (sqrt(s->par) * pnorm) / s->fnorm;
        double prered = t1 * t1 + t2 * t2 / p5;
        double dirder = -(t1 * t1 + t2 * t2);
        double ratio = (prered > 0.0) ? actred / prered : 0.0;

        if (ratio > p25) {
            if (s->par == 0.0 || ratio >= p75) {
                s->delta = pnorm / p5;
                s->par *= p5;
            }
        } else {
            double temp = (actred >= 0.0) ? p5 : p5 * dirder / (dirder + p5 * actred);
            if (p1 * fnorm1 >= s->fnorm || temp < p1) temp = p1;
            double lim = pnorm / p1;
            s->delta = temp * (s->delta < lim ? s->delta : lim);
            s->par /= temp;
        }

        if (ratio >= p0001) {
            memcpy(s->x, s->x_trial, p * sizeof(double));
            memcpy(s->fvec, s->f_trial, n * sizeof(double));
            status = s->df(s->x_trial, s->params, s->J);
            s->n_df_evals++;
            if (status) return LMC_EBADFUNC;
            s->xnorm = scaled_enorm(s->diag, s->x, p);
            s->fnorm = fnorm1;
            s->iter++;
            update_diag(s->J, n, p, s->diag);
            memcpy(r, s->J, n * p * sizeof(double));
            qrpt_decomp(r, n, p, s->tau, s->perm, s->work1);
            return LMC_SUCCESS;
        } else if (fabs(actred) <= DBL_EPSILON && prered <= DBL_EPSILON && p5 * ratio <= 1.0) {
            return LMC_ETOLF;
        } else if (s->delta <= DBL_EPSILON * s->xnorm) {
            return LMC_ETOLX;
        } else if (gnorm <= DBL_EPSILON) {
            return LMC_ETOLG;
        } else if (inner < 10) {
            continue;
        }
        return LMC_ENOPROG;
    }
}

int lmc_test_delta(const double *dx, const double *x, size_t p, double epsabs, double epsrel)
{
    for (size_t i = 0; i < p; i++) {
        double tol = epsabs + epsrel * fabs(x[i]);
        if (!(fabs(dx[i]) < tol)) return LMC_CONTINUE;
    }
    return LMC_SUCCESS;
}

int lmc_covar(const double *J, size_t n, size_t p, size_t ldj, double epsrel, double *covar)
{
    if (p == 0 || p > 16 || n < p) return -1;
    double *r = (double *)malloc(n * p * sizeof(double));
    if (!r) return -1;
    double tau[16], norm[16];
    size_t perm[16];
    for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < p; j++) r[i * p + j] = J[i * ldj + j];
    qrpt_decomp(r, n, p, tau, perm, norm);

    double tolr = epsrel * fabs(RR(0, 0));
    size_t kmax = 0;
    for (size_t k = 0; k < p; k++) {
        double rkk = RR(k, k);
        if (fabs(rkk) <= tolr) break;
        RR(k, k) = 1.0 / rkk;
        for (size_t j = 0; j < k; j++) {
            double t = RR(j, k) / rkk;
            RR(j, k) = 0.0;
            for (size_t i = 0; i <= j; i++) RR(i, k) -= t * RR(i, j);
        }
        kmax = k;
    }
    for (size_t k = 0; k <= kmax; k++) {
        for (size_t j = 0; j < k; j++) {
            double rjk = RR(j, k);
            for (size_t i = 0; i <= j; i++) RR(i, j) += rjk * RR(i, k);
        }
        double t = RR(k, k);
        for (size_t i = 0; i <= k; i++) RR(i, k) *= t;
    }
    for (size_t j = 0; j < p; j++) {
        size_t pj = perm[j];
        for (size_t i = 0; i <= j; i++) {
            size_t pi = perm[i];
            double rij;
            if (j > kmax) {
                RR(i, j) = 0.0;
                rij = 0.0;
            } else {
                rij = RR(i, j);
            }
            if (pi > pj) RR(pi, pj) = rij;
            else if (pi < pj) RR(pj, pi) = rij;
        }
        covar[pj * p + pj] = RR(j, j);
    }
    for (size_t j = 0; j < p; j++) {
        for (size_t i = 0; i < j; i++) {
            double rji = RR(j, i);
            covar[j * p + i] = rji;
            covar[i * p + j] = rji;
        }
    }
    free(r);
    return 0;
}
