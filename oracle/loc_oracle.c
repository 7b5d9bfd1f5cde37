/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle of the Gaussian fitting path (see
 * loc_oracle.h). Every function cites the reference lines it restates.
 * Build without -ffast-math: this is the FP64 yardstick.
 */
#include "loc_oracle.h"
#include "lmsder_core.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* Defines.h:97-98 */
static const double REF_PI = 3.1415926535897932384626433;
static const double REF_SQRT2 = 1.4142135623730950488;

enum {
    FLAG_KEPT = 0,
    FLAG_EDGE = 1,
    FLAG_AMPLITUDE = 2,
    FLAG_OUT_OF_WINDOW = 3,
    FLAG_WIDTH_RANGE = 4,
    FLAG_DRIFT = 5,
    FLAG_EIGEN = 6,
    FLAG_NO_AXIS = 7,
    FLAG_SYMPSF_RATIO = 8,
    FLAG_SYMPSF_WIDTH = 9,
    FLAG_BAD_INPUT = 10
};

/* measured_data_Gauss_fits, Localization.h:195-205 */
typedef struct {
    const double *roi; /* size x size, x fastest */
    int size;
    double x_offset, y_offset, sigma, width;
} fit_data;

int oracle_ref_columns(int method)
{
    switch (method) {
    case 0: return 12; /* Storage.cpp:268-290 */
    case 1: return 10; /* Storage.cpp:405-425 */
    case 5:
    case 7: return 16; /* Storage.cpp:614-640 */
    default: return 0;
    }
}

static int n_params(int method)
{
    return method == 0 ? 5 : method == 1 ? 4 : 7;
}

/* FitFunction_SymmetricGaussian, Localization.cpp:1007-1048 */
static int sym_f(const double *p, void *ctx, double *f)
{
    const fit_data *d = (const fit_data *)ctx;
    double A = p[0], r = p[1], x0 = p[2], y0 = p[3], off = p[4];
    if (r == 0) return -1;
    double two_r2 = 2.0 * r * r;
    int k = 0;
    for (int j = 0; j < d->size; j++) {
        for (int i = 0; i < d->size; i++, k++) {
            double x = d->x_offset + (double)i, y = d->y_offset + (double)j;
            double q = -1.0 * ((x0 - x) * (x0 - x) + (y0 - y) * (y0 - y));
            f[k] = ((exp(q / two_r2) * A + off) - d->roi[k]) / d->sigma;
        }
    }
    return 0;
}

/* Jacobian_SymmetricGaussian, Localization.cpp:1128-1181; the width column
 * keeps the reference's 1/sqrt(2) scaling (cubeStdDev = 2 r^2 sqrt2 r). */
static int sym_jac_core(const double *p, const fit_data *d, double *J, int ld, int skip_width)
{
    double A = p[0], r = p[1], x0 = p[2], y0 = p[3];
    if (r == 0) return -1;
    double s = d->sigma;
    double sq = 2.0 * r * r;
    double cube = sq * REF_SQRT2 * r;
    double dfdoff = 1 / s;
    int k = 0;
    for (int j = 0; j < d->size; j++) {
        for (int i = 0; i < d->size; i++, k++) {
            double x = d->x_offset + (double)i, y = d->y_offset + (double)j;
            double xd = x0 - x, yd = y0 - y;
            double e = exp(-(xd * xd + yd * yd) / sq);
            double dA = e / s;
            double dr = ((2.0 * yd * yd + 2.0 * xd * xd) / cube) * e * A / s;
            double dx0 = (2.0 * (x - x0) * e * A) / (sq * s);
            double dy0 = (2.0 * (y - y0) * e * A) / (sq * s);
            double *row = J + (size_t)k * ld;
            if (skip_width) {
                row[0] = dA; row[1] = dx0; row[2] = dy0; row[3] = dfdoff;
            } else {
                row[0] = dA; row[1] = dr; row[2] = dx0; row[3] = dy0; row[4] = dfdoff;
            }
        }
    }
    return 0;
}

static int sym_df(const double *p, void *ctx, double *J)
{
    return sym_jac_core(p, (const fit_data *)ctx, J, 5, 0);
}

/* FitFunction_FixedWidthGaussian / Jacobian_FixedWidthGaussian,
 * Localization.cpp:1050-1076, 1183-1225: the symmetric model at width w0. */
static int fixed_f(const double *p, void *ctx, double *f)
{
    const fit_data *d = (const fit_data *)ctx;
    double q[5] = {p[0], d->width, p[1], p[2], p[3]};
    return sym_f(q, ctx, f);
}

static int fixed_df(const double *p, void *ctx, double *J)
{
    const fit_data *d = (const fit_data *)ctx;
    double q[5] = {p[0], d->width, p[1], p[2], p[3]};
    return sym_jac_core(q, d, J, 4, 1);
}

/* FitFunction_EllipsoidalGaussian, Localization.cpp:1078-1126 */
static int ell_f(const double *p, void *ctx, double *f)
{
    const fit_data *d = (const fit_data *)ctx;
    double A = p[0], sx = p[1], sy = p[2], x0 = p[3], y0 = p[4], rho = p[5], off = p[6];
    if (sx == 0 || sy == 0) return -1;
    double cct = -1.0 / (2.0 * (1 - rho * rho));
    double sx2 = sx * sx, sy2 = sy * sy;
    int k = 0;
    for (int j = 0; j < d->size; j++) {
        for (int i = 0; i < d->size; i++, k++) {
            double x = d->x_offset + (double)i, y = d->y_offset + (double)j;
            double xd = x - x0, yd = y - y0;
            double q = cct * (xd * xd / sx2 + yd * yd / sy2 - 2.0 * rho * xd * yd / sx / sy);
            f[k] = ((exp(q) * A + off) - d->roi[k]) / d->sigma;
        }
    }
    return 0;
}

/* Jacobian_EllipsoidalGaussian, Localization.cpp:1227-1295; the correlation
 * column keeps the reference expression (exact only when sx == sy). */
static int ell_df(const double *p, void *ctx, double *J)
{
    const fit_data *d = (const fit_data *)ctx;
    double A = p[0], sx = p[1], sy = p[2], x0 = p[3], y0 = p[4], rho = p[5];
    if (sx == 0 || sy == 0) return -1;
    double s = d->sigma;
    double den = 2.0 * (1.0 - rho * rho) * s;
    double dfdoff = 1.0 / s;
    double cct = -1.0 / (2.0 * (1.0 - rho * rho));
    double omr = 1.0 - rho * rho;
    double sx2 = sx * sx, sy2 = sy * sy, sxsy = sx * sy;
    int k = 0;
    for (int j = 0; j < d->size; j++) {
        for (int i = 0; i < d->size; i++, k++) {
            double x = d->x_offset + (double)i, y = d->y_offset + (double)j;
            double xd = x - x0, yd = y - y0;
            double xd2 = xd * xd, yd2 = yd * yd;
            double e = exp(cct * (xd2 / sx2 + yd2 / sy2 - 2.0 * rho * xd * yd / sxsy));
            double *row = J + (size_t)k * 7;
            row[0] = e / s;
            row[1] = -A * (2.0 * rho * xd * yd / sx2 / sy - 2.0 * xd2 / (sx2 * sx)) * e / den;
            row[2] = -A * (2.0 * rho * xd * yd / sx / sy2 - 2.0 * yd2 / (sy2 * sy)) * e / den;
            row[3] = -A * (2.0 * rho * yd / sxsy - 2.0 * xd / sx2) * e / den;
            row[4] = -A * (2.0 * rho * xd / sxsy - 2.0 * yd / sy2) * e / den;
            row[5] = A * (xd * yd / omr / sxsy - rho * (-2.0 * rho * xd * yd + yd2 + xd2) / sxsy / omr / omr) * e / s;
            row[6] = dfdoff;
        }
    }
    return 0;
}

int oracle_model_jacobian(int method, const double *params, double w0, double sigma,
                          double x_offset, double y_offset, int r, const double *roi,
                          double *f, double *J)
{
    fit_data d = {roi, 2 * r + 1, x_offset, y_offset, sigma, w0};
    switch (method) {
    case 0:
        if (sym_f(params, &d, f)) return -1;
        return sym_df(params, &d, J);
    case 1:
        if (fixed_f(params, &d, f)) return -1;
        return fixed_df(params, &d, J);
    case 5:
    case 7:
        if (ell_f(params, &d, f)) return -1;
        return ell_df(params, &d, J);
    default:
        return -2;
    }
}

/* Eigen decomposition of the symmetric 2x2 [[a, b], [b, c]] with ascending
 * eigenvalues, as Eigen::SelfAdjointEigenSolver delivers them for the
 * ellipsoid axes (Localization.cpp:529-547). Returns theta = atan(v00/v10)
 * for the eigenvector v of the smaller eigenvalue (0 when v10 == 0). */
static int eig2_theta(double a, double b, double c, double *l0, double *l1, double *theta)
{
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) return -1;
    double half_tr = 0.5 * (a + c);
    double hd = 0.5 * (a - c);
    double rad = hypot(hd, b);
    *l0 = half_tr - rad;
    *l1 = half_tr + rad;
    double v0, v1;
    if (b == 0.0) {
        if (a <= c) { v0 = 1.0; v1 = 0.0; } else { v0 = 0.0; v1 = 1.0; }
    } else {
        /* (b, l0 - a) and (l0 - c, b) are both eigenvectors; take the larger. */
        double ua0 = b, ua1 = *l0 - a;
        double ub0 = *l0 - c, ub1 = b;
        if (ua0 * ua0 + ua1 * ua1 >= ub0 * ub0 + ub1 * ub1) { v0 = ua0; v1 = ua1; }
        else { v0 = ub0; v1 = ub1; }
    }
    *theta = (v1 == 0.0) ? 0.0 : atan(v0 / v1);
    return 0;
}

typedef struct {
    long iterate_calls, f_evals, df_evals, lambda_trials;
} counters;

/* One candidate: FitPositions_*::fit_positions loop bodies,
 * Localization.cpp:107-212 (symmetric), :286-380 (fixed width),
 * :453-596 (ellipsoidal), :606-631 (symmetric-PSF filter). */
static void fit_one(lmc_state *st, int *st_n, const uint16_t *frames, int n_frames, int n_rows,
                    int n_cols, const oracle_candidate *cand, int method, double w0,
                    double sigma, const oracle_options *opt, const double *init, double *row,
                    uint8_t *flag, double *pout, double *fnout, double *roi_buf, counters *cnt)
{
    const int ncol = oracle_ref_columns(method);
    const int p = n_params(method);
    for (int k = 0; k < ncol + 2; k++) row[k] = NAN;
    row[0] = (double)cand->frame;
    row[ncol] = 0.0;
    row[ncol + 1] = 0.0;
    if (pout)
        for (int k = 0; k < p; k++) pout[k] = NAN;
    if (fnout) *fnout = NAN;

    if (cand->frame < 0 || cand->frame >= n_frames || !isfinite(cand->x) || !isfinite(cand->y) ||
        !isfinite(cand->intensity) || !isfinite(cand->background) || cand->half_width < 0) {
        *flag = FLAG_BAD_INPUT;
        return;
    }
    int r = cand->half_width > 0 ? cand->half_width : (int)ceil(w0 * 4.0);
    int size = 2 * r + 1;
    int n = size * size;

    double x0i = cand->x, y0i = cand->y;
    int x_off = (int)floor(x0i - (double)r);
    int y_off = (int)floor(y0i - (double)r);
    int x_max = x_off + size - 1, y_max = y_off + size - 1;
    if (x_off < 0 || x_max > n_rows - 1 || y_off < 0 || y_max > n_cols - 1) {
        *flag = FLAG_EDGE;
        return;
    }
    const uint16_t *img = frames + (size_t)cand->frame * (size_t)n_rows * (size_t)n_cols;
    for (int k = y_off; k <= y_max; k++)
        for (int j = x_off; j <= x_max; j++)
            roi_buf[(j - x_off) + (k - y_off) * size] = (double)img[j + (size_t)k * n_rows];

    if (*st_n != n) {
        if (*st_n) lmc_free(st);
        lmc_alloc(st, (size_t)n, (size_t)p);
        *st_n = n;
    }
    fit_data d = {roi_buf, size, (double)x_off, (double)y_off, sigma, w0};
    double x0[7];
    if (init) {
        for (int k = 0; k < p; k++) x0[k] = init[k];
    } else if (method == 0) {
        x0[0] = cand->intensity; x0[1] = w0; x0[2] = x0i; x0[3] = y0i; x0[4] = cand->background;
    } else if (method == 1) {
        x0[0] = cand->intensity; x0[1] = x0i; x0[2] = y0i; x0[3] = cand->background;
    } else {
        x0[0] = cand->intensity; x0[1] = w0; x0[2] = w0; x0[3] = x0i; x0[4] = y0i;
        x0[5] = 0.0; x0[6] = cand->background;
    }
    lmc_f_fn ff = method == 0 ? sym_f : method == 1 ? fixed_f : ell_f;
    lmc_df_fn dff = method == 0 ? sym_df : method == 1 ? fixed_df : ell_df;

    st->n_f_evals = st->n_df_evals = st->n_lambda_trials = 0;
    lmc_set(st, ff, dff, &d, x0);
    long iterations = 0;
    int status;
    do {
        iterations++;
        status = lmc_iterate(st);
        if (status != 0) break;
        status = lmc_test_delta(st->dx, st->x, (size_t)p, opt->epsabs, opt->epsrel);
    } while (status == LMC_CONTINUE && iterations < opt->max_iter);
    cnt->iterate_calls += iterations;
    cnt->f_evals += st->n_f_evals;
    cnt->df_evals += st->n_df_evals;
    cnt->lambda_trials += st->n_lambda_trials;

    row[ncol] = (double)iterations;
    row[ncol + 1] = status == 0 ? 0.0 : (status == LMC_CONTINUE ? 1.0 : (double)status);

    double *x = st->x;
    if (method == 0) {
        x[1] = fabs(x[1]);
    } else if (method != 1) {
        x[1] = fabs(x[1]);
        x[2] = fabs(x[2]);
    }
    if (pout)
        for (int k = 0; k < p; k++) pout[k] = x[k];
    if (fnout) *fnout = lmc_enorm(st->fvec, (size_t)n, 1);

    if (x[0] <= 0) {
        *flag = FLAG_AMPLITUDE;
        return;
    }
    int ix = method == 0 ? 2 : method == 1 ? 1 : 3;
    if (x[ix] < x_off || x[ix] > x_max || x[ix + 1] < y_off || x[ix + 1] > y_max) {
        *flag = FLAG_OUT_OF_WINDOW;
        return;
    }

    double cov[49];
    double chi, dof, c;
    if (method == 0) {
        if (x[1] < 0.4 * w0 || x[1] > w0 * 1.5) {
            *flag = FLAG_WIDTH_RANGE;
            return;
        }
        lmc_covar(st->J, (size_t)n, 5, 5, 0.0, cov);
        chi = lmc_enorm(st->fvec, (size_t)n, 1);
        dof = (2 * r - 1) * (2 * r - 1) - 5; /* Localization.cpp:187, as written */
        c = 1.0 > chi / sqrt(dof) ? 1.0 : chi / sqrt(dof);
        double width = x[1];
        double widthDev = c * sqrt(cov[1 * 5 + 1]);
        double integral = 2 * REF_PI * width * width * x[0];
        double relA = c * sqrt(cov[0]) / x[0];
        double relW = widthDev / width;
        row[1] = integral;
        row[2] = width;
        row[3] = x[2];
        row[4] = x[3];
        row[5] = x[4];
        row[6] = 2 * REF_PI * integral * sqrt(relA * relA + 2 * relW * relW);
        row[7] = widthDev;
        row[8] = c * sqrt(cov[2 * 5 + 2]);
        row[9] = c * sqrt(cov[3 * 5 + 3]);
        row[10] = c * sqrt(cov[4 * 5 + 4]);
        row[11] = 1.0;
    } else if (method == 1) {
        if (fabs(x[1] - x0i) > 2.0 * w0 || fabs(x[2] - y0i) > 2.0 * w0) {
            *flag = FLAG_DRIFT;
            return;
        }
        lmc_covar(st->J, (size_t)n, 4, 4, 0.0, cov);
        chi = lmc_enorm(st->fvec, (size_t)n, 1);
        dof = (2 * r - 1) * (2 * r - 1) - 4; /* Localization.cpp:357 */
        c = 1.0 > chi / sqrt(dof) ? 1.0 : chi / sqrt(dof);
        double integral = 2 * REF_PI * w0 * w0 * x[0];
        double relA = c * sqrt(cov[0]) / x[0];
        row[1] = integral;
        row[2] = x[1];
        row[3] = x[2];
        row[4] = x[3];
        row[5] = 2 * REF_PI * integral * w0 * w0 * sqrt(relA * relA);
        row[6] = c * sqrt(cov[1 * 4 + 1]);
        row[7] = c * sqrt(cov[2 * 4 + 2]);
        row[8] = c * sqrt(cov[3 * 4 + 3]);
        row[9] = 1.0;
    } else {
        double sx = x[1], sy = x[2], rho = x[5];
        double l0, l1, theta;
        if (eig2_theta(sx * sx, rho * sx * sy, sy * sy, &l0, &l1, &theta) != 0) {
            *flag = FLAG_EIGEN;
            return;
        }
        double s1 = sqrt(l0), s2 = sqrt(l1);
        if (!(((s1 >= 0.4 * w0) && (s1 <= 1.5 * w0)) || ((s2 >= 0.4 * w0) && (s2 <= 1.5 * w0)))) {
            *flag = FLAG_NO_AXIS;
            return;
        }
        lmc_covar(st->J, (size_t)n, 7, 7, 0.0, cov);
        chi = lmc_enorm(st->fvec, (size_t)n, 1);
        dof = (2 * r - 1) * (2 * r - 1) - 7; /* Localization.cpp:558 */
        c = 1.0 > chi / sqrt(dof) ? 1.0 : chi / sqrt(dof);
        double corrDev = c * sqrt(cov[5 * 7 + 5]);
        double sxDev = c * sqrt(cov[1 * 7 + 1]);
        double syDev = c * sqrt(cov[2 * 7 + 2]);
        double s1Dev = sxDev * cos(theta) + syDev * sin(theta);
        double s2Dev = sxDev * sin(theta) + syDev * cos(theta);
        double ampDev = c * sqrt(cov[0]);
        double omr = 1 - rho * rho;
        double integral = 2.0 * REF_PI * x[0] * sqrt(omr) * s1 * s2;
        double integralDev = 2.0 * REF_PI * x[0] * sqrt(omr) * s1 * s2 *
                             sqrt(ampDev * ampDev / x[0] / x[0] +
                                  rho * rho * corrDev * corrDev / omr / omr +
                                  s1Dev * s1Dev / s1 / s1 + s2Dev * s2Dev / s2 / s2);
        row[1] = integral;
        row[2] = s1;
        row[3] = s2;
        row[4] = x[3];
        row[5] = x[4];
        row[6] = theta;
        row[7] = x[6];
        row[8] = integralDev;
        row[9] = s1Dev;
        row[10] = s2Dev;
        row[11] = c * sqrt(cov[3 * 7 + 3]);
        row[12] = c * sqrt(cov[4 * 7 + 4]);
        row[13] = 0.0;
        row[14] = c * sqrt(cov[6 * 7 + 6]);
        row[15] = 1.0;
        if (method == 5) {
            if ((0.75 * s1 > s2) || (1.25 * s1 < s2)) {
                *flag = FLAG_SYMPSF_RATIO;
                return;
            }
            if (((s1 < w0 * 0.7) || (s1 > w0 * 1.3)) && ((s2 < w0 * 0.7) || (s2 > w0 * 1.3))) {
                *flag = FLAG_SYMPSF_WIDTH;
                return;
            }
        }
    }
    *flag = FLAG_KEPT;
}

typedef struct {
    const uint16_t *frames;
    int n_frames, n_rows, n_cols;
    const oracle_candidate *cands;
    int method;
    double w0, sigma;
    const oracle_options *opt;
    double *out;
    uint8_t *flags;
    double *params_out, *fnorm_out;
    int begin, end;
    counters cnt;
} work_range;

static void *run_range(void *arg)
{
    work_range *w = (work_range *)arg;
    const int ncol = oracle_ref_columns(w->method);
    const int p = n_params(w->method);
    lmc_state st;
    int st_n = 0;
    memset(&st, 0, sizeof(st));
    double *roi = (double *)malloc(sizeof(double) * 129 * 129);
    for (int i = w->begin; i < w->end; i++) {
        const double *init = w->opt->init_params ? w->opt->init_params + (size_t)i * p : NULL;
        fit_one(&st, &st_n, w->frames, w->n_frames, w->n_rows, w->n_cols, &w->cands[i], w->method,
                w->w0, w->sigma, w->opt, init, w->out + (size_t)i * (ncol + 2), &w->flags[i],
                w->params_out ? w->params_out + (size_t)i * p : NULL,
                w->fnorm_out ? w->fnorm_out + i : NULL, roi, &w->cnt);
    }
    if (st_n) lmc_free(&st);
    free(roi);
    return NULL;
}

static counters g_last;

int oracle_fit(const uint16_t *frames, int n_frames, int n_rows, int n_cols,
               const oracle_candidate *cands, int nc, int method, double w0,
               double sigma, const oracle_options *opt, double *out,
               uint8_t *flags, double *params_out, double *fnorm_out)
{
    if (oracle_ref_columns(method) == 0) return -2;
    if (!(w0 > 0) || !(sigma != 0) || nc < 0) return -3;
    for (int i = 0; i < nc; i++)
        if (cands[i].half_width > 64 || (cands[i].half_width == 0 && ceil(4 * w0) > 64)) return -4;
    oracle_options def = {200, 1e-4, 1e-4, 1, NULL};
    if (!opt) opt = &def;
    int nt = opt->nthreads > 0 ? opt->nthreads : 1;
    if (nt > 256) nt = 256;
    if (nt > nc) nt = nc > 0 ? nc : 1;
    work_range *ranges = (work_range *)calloc((size_t)nt, sizeof(work_range));
    pthread_t *th = (pthread_t *)calloc((size_t)nt, sizeof(pthread_t));
    for (int t = 0; t < nt; t++) {
        work_range *w = &ranges[t];
        w->frames = frames; w->n_frames = n_frames; w->n_rows = n_rows; w->n_cols = n_cols;
        w->cands = cands; w->method = method; w->w0 = w0; w->sigma = sigma; w->opt = opt;
        w->out = out; w->flags = flags; w->params_out = params_out; w->fnorm_out = fnorm_out;
        w->begin = (int)((long long)nc * t / nt);
        w->end = (int)((long long)nc * (t + 1) / nt);
    }
    if (nt == 1) {
        run_range(&ranges[0]);
    } else {
        for (int t = 0; t < nt; t++) pthread_create(&th[t], NULL, run_range, &ranges[t]);
        for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
    }
    memset(&g_last, 0, sizeof(g_last));
    for (int t = 0; t < nt; t++) {
        g_last.iterate_calls += ranges[t].cnt.iterate_calls;
        g_last.f_evals += ranges[t].cnt.f_evals;
        g_last.df_evals += ranges[t].cnt.df_evals;
        g_last.lambda_trials += ranges[t].cnt.lambda_trials;
    }
    free(ranges);
    free(th);
    return 0;
}

void oracle_last_counters(long *n_iterate_calls, long *n_f_evals, long *n_df_evals,
                          long *n_lambda_trials)
{
    if (n_iterate_calls) *n_iterate_calls = g_last.iterate_calls;
    if (n_f_evals) *n_f_evals = g_last.f_evals;
    if (n_df_evals) *n_df_evals = g_last.df_evals;
    if (n_lambda_trials) *n_lambda_trials = g_last.lambda_trials;
}

/* ThresholdImage_GLRT_FFT: constructor Segmentation.cpp:241-252, kernels
 * :254-314, test :316-430. The Gaussian correlation is evaluated directly
 * (the reference's FFT product equals the direct sum on the interior pixels
 * the test visits); the box sums are exact integer sums in double. */
int oracle_glrt_mask(const uint16_t *frame, int n_rows, int n_cols, double pfa,
                     double psf_width, int32_t *mask)
{
    int ws = (int)ceil(4 * psf_width);
    if (ws % 2 == 0) ws += 1;
    int half = ws / 2;
    double npix = (double)ws * (double)ws;
    int xs = n_rows - (n_rows % 2), ys = n_cols - (n_cols % 2);
    for (long i = 0; i < (long)n_rows * n_cols; i++) mask[i] = 0;
    if (xs < ws + 2 || ys < ws + 2) return 0;

    double *g = (double *)malloc(sizeof(double) * ws * ws);
    double sum = 0.0;
    for (int j = -half; j <= half; ++j) {
        for (int i = -half; i <= half; ++i) {
            double v = 1.0 / (1.77245385 * psf_width) *
                       exp(-1.0 / (2.0 * psf_width * psf_width) * ((double)i * i + (double)j * j));
            g[(i + half) + (j + half) * ws] = v;
            sum += v;
        }
    }
    sum /= npix;
    double sumsq = 0.0;
    for (int k = 0; k < ws * ws; k++) {
        g[k] -= sum;
        sumsq += g[k] * g[k];
    }
    double thr = 1.0 - exp(-pfa / npix);
    for (int l = half + 1; l < ys - half; l++) {
        for (int k = half + 1; k < xs - half; k++) {
            double s1 = 0.0, s2 = 0.0, conv = 0.0;
            for (int b = -half; b <= half; b++) {
                for (int a = -half; a <= half; a++) {
                    double v = (double)frame[(k + a) + (size_t)(l + b) * n_rows];
                    s1 += v;
                    s2 += v * v;
                    conv += v * g[(a + half) + (b + half) * ws];
                }
            }
            double avg = s1 / npix;
            double null_h = s2 - avg * avg * npix;
            double alpha = conv / sumsq;
            double test = alpha * alpha / null_h * sumsq;
            if (test < 1.0 && test > thr) mask[k + (size_t)l * n_rows] = 255;
        }
    }
    free(g);
    return 0;
}

/* ParticleFinder_adjacent8::findPositions / growParticle,
 * ParticleFinding.cpp:283-427: raster scan, breadth-first growth over the 8
 * neighbours, unweighted mean of the member coordinates, max member value
 * minus the frame background (mean of the unmasked pixels). */
int oracle_find_adjacent8(const uint16_t *frame, int n_rows, int n_cols,
                          const int32_t *mask, double *out, int max_out)
{
    size_t npx = (size_t)n_rows * n_cols;
    long *mapped = (long *)malloc(sizeof(long) * npx);
    int *queue = (int *)malloc(sizeof(int) * npx);
    for (size_t i = 0; i < npx; i++) mapped[i] = -1;
    double bg = 0.0;
    size_t nbg = 0;
    long pidx = 0;
    int nfound = 0;
    for (int j = 0; j < n_cols; j++) {
        for (int i = 0; i < n_rows; i++) {
            size_t at = (size_t)i + (size_t)j * n_rows;
            if (mask[at] < 128) {
                bg += (double)frame[at];
                ++nbg;
                continue;
            }
            if (mapped[at] != -1) continue;
            mapped[at] = pidx;
            int qh = 0, qt = 0;
            queue[qt++] = (int)at;
            double sx = 0.0, sy = 0.0, mx = 0.0;
            long cnt = 0;
            while (qh < qt) {
                int cur = queue[qh++];
                int cx = cur % n_rows, cy = cur / n_rows;
                int lx = cx - 1 < 0 ? 0 : cx - 1, ux = cx + 1 >= n_rows ? n_rows - 1 : cx + 1;
                int ly = cy - 1 < 0 ? 0 : cy - 1, uy = cy + 1 >= n_cols ? n_cols - 1 : cy + 1;
                for (int b = ly; b <= uy; b++) {
                    for (int a = lx; a <= ux; a++) {
                        if (a == cx && b == cy) continue;
                        size_t nat = (size_t)a + (size_t)b * n_rows;
                        if (mask[nat] < 128) continue;
                        if (mapped[nat] != -1) continue;
                        mapped[nat] = pidx;
                        queue[qt++] = (int)nat;
                    }
                }
                sx += (double)cx;
                sy += (double)cy;
                double v = (double)frame[cur];
                if (v > mx) mx = v;
                cnt++;
            }
            ++pidx;
            if (nfound < max_out) {
                out[4 * nfound + 0] = sx / (double)cnt;
                out[4 * nfound + 1] = sy / (double)cnt;
                out[4 * nfound + 2] = mx;
                out[4 * nfound + 3] = 0.0;
            }
            nfound++;
        }
    }
    bg /= (double)nbg;
    int nw = nfound < max_out ? nfound : max_out;
    for (int k = 0; k < nw; k++) {
        out[4 * k + 2] = out[4 * k + 2] - bg;
        out[4 * k + 3] = bg;
    }
    free(mapped);
    free(queue);
    return nfound;
}

/* Trajectory of one fit for cross-checking the solver restatement against an
 * independent MINPACK: after every iterate() call records the cumulative
 * number of trial evaluations and the current point. Returns the number of
 * records written (at most max_rec). */
int oracle_trajectory(int method, const double *roi, int r, double x_offset, double y_offset, double w0,
                      double sigma, const double *x0, int max_rec, int *trials, double *xs)
{
    const int p = n_params(method);
    const int size = 2 * r + 1, n = size * size;
    fit_data d = {roi, size, x_offset, y_offset, sigma, w0};
    lmc_state st;
    if (lmc_alloc(&st, (size_t)n, (size_t)p) != 0) return -1;
    lmc_f_fn ff = method == 0 ? sym_f : method == 1 ? fixed_f : ell_f;
    lmc_df_fn dff = method == 0 ? sym_df : method == 1 ? fixed_df : ell_df;
    lmc_set(&st, ff, dff, &d, x0);
    int k = 0;
    while (k < max_rec) {
        int status = lmc_iterate(&st);
        trials[k] = (int)st.n_f_evals;
        for (int i = 0; i < p; i++) xs[k * p + i] = st.x[i];
        k++;
        if (status != 0) break;
    }
    lmc_free(&st);
    return k;
}
