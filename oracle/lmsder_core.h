/*
 * TEST INFRASTRUCTURE ONLY — part of the CPU oracle. Nothing in the product
 * (the localizer_b200 package, include/, the CUDA kernels) may include, link
 * or call this file; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it, and only as the checker.
 *
 * FP64 restatement of the scaled Levenberg-Marquardt trust-region solver that
 * the reference calls as gsl_multifit_fdfsolver_lmsder (GNU Scientific Library
 * 1.16, pinned by include/gsl/gsl_version.h:28 of the reference). The GSL
 * sources are not part of the reference tree, so this is written from the
 * published algorithm: J. J. More, "The Levenberg-Marquardt algorithm:
 * implementation and theory", Lecture Notes in Mathematics 630 (1978), as
 * realised in MINPACK lmder/lmpar/qrsolv, together with the GSL-specific
 * behaviour documented for lmsder:
 *   - column pivoted Householder QR of J for every new Jacobian;
 *   - diag = running maximum of the Jacobian column norms (zero norms -> 1);
 *   - initial step bound 100*|D x| (100 when |D x| == 0);
 *   - at most 10 rejected trial steps per iterate() call, after which the
 *     call reports "no progress" (GSL_ENOPROG);
 *   - on the first iterate() the step bound is clipped to the first trial step.
 * The reference call sites are source/Localization.cpp:145-155 (symmetric),
 * :324-334 (fixed width) and :494-504 (ellipsoidal); the covariance call is
 * :185, :355, :556 (gsl_multifit_covar(J, 0.0, covar)).
 */
#ifndef LOC_ORACLE_LMSDER_CORE_H
#define LOC_ORACLE_LMSDER_CORE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, numerically equal to the GSL errno values the reference sees. */
enum {
    LMC_SUCCESS = 0,
    LMC_FAILURE = -1,
    LMC_CONTINUE = -2,
    LMC_EBADFUNC = 9,
    LMC_ETOLF = 29,
    LMC_ETOLX = 30,
    LMC_ETOLG = 31,
    LMC_ENOPROG = 27
};

/* f(x) -> fvec (length n); df(x) -> J (n x p, row-major, row stride p). */
typedef int (*lmc_f_fn)(const double *x, void *params, double *f);
typedef int (*lmc_df_fn)(const double *x, void *params, double *J);

typedef struct {
    size_t n, p;
    lmc_f_fn f;
    lmc_df_fn df;
    void *params;

    double *x, *fvec, *J, *dx;          /* current point, residuals, Jacobian, last step */

    double *r, *tau, *diag, *qtf, *newton, *gradient;
    double *x_trial, *f_trial, *sdiag, *rptdx, *w, *work1;
    size_t *perm;

    double fnorm, xnorm, delta, par;
    size_t iter;                        /* 1 + number of accepted steps */

    /* instrumentation (not part of the solver's behaviour) */
    long n_f_evals;                     /* trial-point residual evaluations */
    long n_df_evals;                    /* Jacobian evaluations */
    long n_lambda_trials;               /* qrsolv calls inside lmpar */
    long n_inner_trials;                /* trial steps (lmpar calls) */
} lmc_state;

/* Allocate workspaces for an n x p problem. Returns 0 on success. */
int lmc_alloc(lmc_state *s, size_t n, size_t p);
void lmc_free(lmc_state *s);

/* Equivalent of gsl_multifit_fdfsolver_set for lmsder. */
int lmc_set(lmc_state *s, lmc_f_fn f, lmc_df_fn df, void *params, const double *x0);

/* Equivalent of gsl_multifit_fdfsolver_iterate for lmsder. */
int lmc_iterate(lmc_state *s);

/* Equivalent of gsl_multifit_test_delta: |dx_i| < epsabs + epsrel |x_i| for all i. */
int lmc_test_delta(const double *dx, const double *x, size_t p, double epsabs, double epsrel);

/* Equivalent of gsl_multifit_covar: (J^T J)^-1 by pivoted QR, dropping columns
 * whose |R_kk| <= epsrel |R_00|. J is n x p row-major with row stride ldj;
 * covar is p x p row-major. */
int lmc_covar(const double *J, size_t n, size_t p, size_t ldj, double epsrel, double *covar);

/* Euclidean norm with the scaling of the reference BLAS dnrm2. */
double lmc_enorm(const double *v, size_t n, size_t stride);

#ifdef __cplusplus
}
#endif

#endif
