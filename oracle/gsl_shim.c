/*
 * TEST INFRASTRUCTURE ONLY — links the reference's own Localization.cpp,
 * Storage.cpp and ParticleFinding.cpp (compiled unmodified into oracle/_ref)
 * against the lmsder restatement in lmsder_core.c. Compiled against the GSL
 * 1.16 headers vendored in the reference (include/gsl) for the struct
 * layouts only; it implements just the GSL entry points those three files
 * import (gsl_vector/gsl_matrix allocation, gsl_blas_dnrm2, the lmsder
 * fdfsolver, gsl_multifit_test_delta, gsl_multifit_covar) and, for the MLEwG
 * fitter (Localization.cpp:633-789), the nmsimplex2 minimiser over the
 * restatement in nmsimplex_core.c, gsl_multimin_test_size and
 * gsl_sf_lngamma (log |Gamma|, from libm).
 *
 * It also records, per solver set() call, how many iterate() calls followed
 * and the last status, so the harness can read the reference's iteration
 * count (a local variable in fit_positions, Localization.cpp:62,149).
 */
#include <gsl/gsl_blas.h>
#include <gsl/gsl_errno.h>
#include <gsl/gsl_matrix.h>
#include <gsl/gsl_multifit_nlin.h>
#include <gsl/gsl_multimin.h>
#include <gsl/gsl_sf_gamma.h>
#include <gsl/gsl_vector.h>

#include <stdlib.h>
#include <string.h>

#include "lmsder_core.h"
#include "nmsimplex_core.h"
#include <math.h>

gsl_vector *gsl_vector_alloc(const size_t n)
{
    gsl_vector *v = (gsl_vector *)calloc(1, sizeof(gsl_vector));
    if (!v) return NULL;
    v->data = (double *)calloc(n ? n : 1, sizeof(double));
    if (!v->data) {
        free(v);
        return NULL;
    }
    v->size = n;
    v->stride = 1;
    v->owner = 1;
    return v;
}

void gsl_vector_free(gsl_vector *v)
{
    if (!v) return;
    if (v->owner) free(v->data);
    free(v);
}

void gsl_vector_set_all(gsl_vector *v, double x)
{
    for (size_t i = 0; i < v->size; i++) v->data[i * v->stride] = x;
}

gsl_matrix *gsl_matrix_alloc(const size_t n1, const size_t n2)
{
    gsl_matrix *m = (gsl_matrix *)calloc(1, sizeof(gsl_matrix));
    if (!m) return NULL;
    m->data = (double *)calloc((n1 * n2) ? n1 * n2 : 1, sizeof(double));
    if (!m->data) {
        free(m);
        return NULL;
    }
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->owner = 1;
    return m;
}

void gsl_matrix_free(gsl_matrix *m)
{
    if (!m) return;
    if (m->owner) free(m->data);
    free(m);
}

double gsl_blas_dnrm2(const gsl_vector *x)
{
    return lmc_enorm(x->data, x->size, x->stride);
}

/* ---- lmsder fdfsolver ---- */

typedef struct {
    lmc_state core;
    gsl_multifit_function_fdf *fdf;
    gsl_vector vx, vf, vdx;
    gsl_matrix mJ;
} shim_state;

static int tramp_f(const double *x, void *params, double *f)
{
    shim_state *s = (shim_state *)params;
    gsl_vector xv = {s->core.p, 1, (double *)x, NULL, 0};
    gsl_vector fv = {s->core.n, 1, f, NULL, 0};
    return GSL_MULTIFIT_FN_EVAL_F(s->fdf, &xv, &fv);
}

static int tramp_df(const double *x, void *params, double *J)
{
    shim_state *s = (shim_state *)params;
    gsl_vector xv = {s->core.p, 1, (double *)x, NULL, 0};
    gsl_matrix jm = {s->core.n, s->core.p, s->core.p, J, NULL, 0};
    return GSL_MULTIFIT_FN_EVAL_DF(s->fdf, &xv, &jm);
}

static int shim_alloc(void *vstate, size_t n, size_t p)
{
    shim_state *s = (shim_state *)vstate;
    return lmc_alloc(&s->core, n, p) == 0 ? GSL_SUCCESS : GSL_ENOMEM;
}

/* iteration log: one entry per set(), counting the iterate() calls after it */
#define LOG_CAP (1 << 20)
/* per host thread, so several threads can drive the reference fitters */
static _Thread_local long g_log_n = 0;
static _Thread_local int *g_log_iters = NULL;
static _Thread_local int *g_log_status = NULL;

void lmshim_log_reset(void)
{
    if (!g_log_iters) {
        g_log_iters = (int *)malloc(sizeof(int) * LOG_CAP);
        g_log_status = (int *)malloc(sizeof(int) * LOG_CAP);
    }
    g_log_n = 0;
}

long lmshim_log_count(void) { return g_log_n; }

void lmshim_log_get(long i, int *iters, int *status)
{
    *iters = g_log_iters[i];
    *status = g_log_status[i];
}

static int shim_set(void *vstate, gsl_multifit_function_fdf *fdf, gsl_vector *x,
                    gsl_vector *f, gsl_matrix *J, gsl_vector *dx)
{
    shim_state *s = (shim_state *)vstate;
    (void)f; (void)J; (void)dx;
    s->fdf = fdf;
    if (g_log_iters && g_log_n < LOG_CAP) {
        g_log_iters[g_log_n] = 0;
        g_log_status[g_log_n] = 0;
        g_log_n++;
    }
    return lmc_set(&s->core, tramp_f, tramp_df, s, x->data);
}

static int shim_iterate(void *vstate, gsl_multifit_function_fdf *fdf, gsl_vector *x,
                        gsl_vector *f, gsl_matrix *J, gsl_vector *dx)
{
    shim_state *s = (shim_state *)vstate;
    (void)fdf; (void)x; (void)f; (void)J; (void)dx;
    int st = lmc_iterate(&s->core);
    if (g_log_iters && g_log_n > 0) {
        g_log_iters[g_log_n - 1]++;
        g_log_status[g_log_n - 1] = st;
    }
    return st;
}

static void shim_free(void *vstate)
{
    shim_state *s = (shim_state *)vstate;
    lmc_free(&s->core);
}

static const gsl_multifit_fdfsolver_type lmsder_type = {
    "lmsder", sizeof(shim_state), shim_alloc, shim_set, shim_iterate, shim_free};

const gsl_multifit_fdfsolver_type *gsl_multifit_fdfsolver_lmsder = &lmsder_type;

gsl_multifit_fdfsolver *gsl_multifit_fdfsolver_alloc(const gsl_multifit_fdfsolver_type *T,
                                                     size_t n, size_t p)
{
    gsl_multifit_fdfsolver *s = (gsl_multifit_fdfsolver *)calloc(1, sizeof(*s));
    if (!s) return NULL;
    shim_state *st = (shim_state *)calloc(1, T->size);
    if (!st || T->alloc(st, n, p) != GSL_SUCCESS) {
        free(st);
        free(s);
        return NULL;
    }
    /* the solver's public x, f, J, dx alias the restatement's arrays */
    st->vx = (gsl_vector){p, 1, st->core.x, NULL, 0};
    st->vf = (gsl_vector){n, 1, st->core.fvec, NULL, 0};
    st->vdx = (gsl_vector){p, 1, st->core.dx, NULL, 0};
    st->mJ = (gsl_matrix){n, p, p, st->core.J, NULL, 0};
    s->type = T;
    s->x = &st->vx;
    s->f = &st->vf;
    s->J = &st->mJ;
    s->dx = &st->vdx;
    s->state = st;
    return s;
}

int gsl_multifit_fdfsolver_set(gsl_multifit_fdfsolver *s, gsl_multifit_function_fdf *fdf,
                               const gsl_vector *x)
{
    shim_state *st = (shim_state *)s->state;
    if (fdf->n != st->core.n || fdf->p != st->core.p || x->size != st->core.p) return GSL_EBADLEN;
    double tmp[16];
    for (size_t i = 0; i < x->size; i++) tmp[i] = x->data[i * x->stride];
    gsl_vector xv = {x->size, 1, tmp, NULL, 0};
    s->fdf = fdf;
    return s->type->set(st, fdf, &xv, s->f, s->J, s->dx);
}

int gsl_multifit_fdfsolver_iterate(gsl_multifit_fdfsolver *s)
{
    return s->type->iterate(s->state, s->fdf, s->x, s->f, s->J, s->dx);
}

void gsl_multifit_fdfsolver_free(gsl_multifit_fdfsolver *s)
{
    if (!s) return;
    s->type->free(s->state);
    free(s->state);
    free(s);
}

int gsl_multifit_test_delta(const gsl_vector *dx, const gsl_vector *x, double epsabs, double epsrel)
{
    if (epsrel < 0.0) return GSL_EBADTOL;
    double a[16], b[16];
    for (size_t i = 0; i < x->size; i++) {
        a[i] = dx->data[i * dx->stride];
        b[i] = x->data[i * x->stride];
    }
    return lmc_test_delta(a, b, x->size, epsabs, epsrel) == LMC_SUCCESS ? GSL_SUCCESS : GSL_CONTINUE;
}

int gsl_multifit_covar(const gsl_matrix *J, double epsrel, gsl_matrix *covar)
{
    double tmp[256];
    if (J->size2 > 16) return GSL_EBADLEN;
    if (lmc_covar(J->data, J->size1, J->size2, J->tda, epsrel, tmp) != 0) return GSL_ENOMEM;
    for (size_t i = 0; i < J->size2; i++)
        for (size_t j = 0; j < J->size2; j++) covar->data[i * covar->tda + j] = tmp[i * J->size2 + j];
    return GSL_SUCCESS;
}

/* ---- Nelder-Mead minimiser (MLEwG fitter, Localization.cpp:633-789) ---- */

typedef struct {
    nm_state nm;
    gsl_multimin_function *fn;
    size_t n;
} nm_shim_state;

static double nm_tramp(const double *x, void *par)
{
    nm_shim_state *s = (nm_shim_state *)par;
    gsl_vector xv = {s->n, 1, (double *)x, NULL, 0};
    return GSL_MULTIMIN_FN_EVAL(s->fn, &xv);
}

static int nms_alloc(void *vstate, size_t n)
{
    nm_shim_state *s = (nm_shim_state *)vstate;
    if (n < 1 || n > NM_NMAX) return GSL_EINVAL;
    s->n = n;
    return GSL_SUCCESS;
}

static int nms_set(void *vstate, gsl_multimin_function *f, const gsl_vector *x, double *size,
                   const gsl_vector *step_size)
{
    nm_shim_state *s = (nm_shim_state *)vstate;
    double xa[NM_NMAX], st[NM_NMAX];
    for (size_t i = 0; i < s->n; i++) {
        xa[i] = x->data[i * x->stride];
        st[i] = step_size->data[i * step_size->stride];
    }
    s->fn = f;
    if (g_log_iters && g_log_n < LOG_CAP) {
        g_log_iters[g_log_n] = 0;
        g_log_status[g_log_n] = 0;
        g_log_n++;
    }
    return nm_set(&s->nm, (int)s->n, nm_tramp, s, xa, st, size);
}

static int nms_iterate(void *vstate, gsl_multimin_function *f, gsl_vector *x, double *size, double *fval)
{
    nm_shim_state *s = (nm_shim_state *)vstate;
    double xa[NM_NMAX];
    s->fn = f;
    const int rc = nm_iterate(&s->nm, nm_tramp, s, xa, size, fval);
    if (rc == 0)
        for (size_t i = 0; i < s->n; i++) x->data[i * x->stride] = xa[i];
    if (g_log_iters && g_log_n > 0) {
        g_log_iters[g_log_n - 1]++;
        g_log_status[g_log_n - 1] = rc;
    }
    return rc;
}

static void nms_free(void *vstate) { (void)vstate; }

static const gsl_multimin_fminimizer_type nmsimplex2_type = {
    "nmsimplex2", sizeof(nm_shim_state), nms_alloc, nms_set, nms_iterate, nms_free};

const gsl_multimin_fminimizer_type *gsl_multimin_fminimizer_nmsimplex2 = &nmsimplex2_type;

gsl_multimin_fminimizer *gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type *T, size_t n)
{
    if (!T) return NULL;
    gsl_multimin_fminimizer *s = (gsl_multimin_fminimizer *)calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->state = calloc(1, T->size);
    s->x = gsl_vector_alloc(n);
    if (!s->state || !s->x || T->alloc(s->state, n) != GSL_SUCCESS) {
        gsl_vector_free(s->x);
        free(s->state);
        free(s);
        return NULL;
    }
    s->type = T;
    return s;
}

void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer *s)
{
    if (!s) return;
    s->type->free(s->state);
    free(s->state);
    gsl_vector_free(s->x);
    free(s);
}

int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer *s, gsl_multimin_function *f, const gsl_vector *x,
                                const gsl_vector *step_size)
{
    if (s->x->size != f->n || x->size != f->n || step_size->size != f->n) return GSL_EBADLEN;
    s->f = f;
    for (size_t i = 0; i < x->size; i++) s->x->data[i] = x->data[i * x->stride];
    return s->type->set(s->state, f, x, &s->size, step_size);
}

int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer *s)
{
    return s->type->iterate(s->state, s->f, s->x, &s->size, &s->fval);
}

double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer *s) { return s->size; }

int gsl_multimin_test_size(const double size, double epsabs)
{
    if (epsabs < 0.0) return GSL_EBADTOL;
    return size < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}

/* log |Gamma(x)| (the reference only calls it at integer + 1) */
double gsl_sf_lngamma(const double x) { return lgamma(x); }
