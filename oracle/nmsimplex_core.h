/*
 * TEST INFRASTRUCTURE ONLY — Nelder-Mead simplex restatement used by the GSL
 * shim (gsl_multimin_fminimizer_nmsimplex2) that links the reference's MLEwG
 * fitter. See nmsimplex_core.c.
 */
#ifndef NMSIMPLEX_CORE_H
#define NMSIMPLEX_CORE_H

#define NM_NMAX 8
#define NM_EINVAL 4     /* GSL_EINVAL */
#define NM_EFAILED 5    /* GSL_EFAILED */
#define NM_EBADFUNC 9   /* GSL_EBADFUNC */

typedef double (*nm_fn)(const double *x, void *par);

typedef struct {
    int n;
    double x1[(NM_NMAX + 1) * NM_NMAX]; /* corners, row-major */
    double y1[NM_NMAX + 1];             /* function values */
    double center[NM_NMAX];
    double ws1[NM_NMAX], ws2[NM_NMAX], delta[NM_NMAX], xmc[NM_NMAX];
    double S2;                          /* squared RMS size */
} nm_state;

double nm_dnrm2(const double *x, int n);
int nm_set(nm_state *s, int n, nm_fn f, void *par, const double *x, const double *step, double *size);
int nm_iterate(nm_state *s, nm_fn f, void *par, double *x, double *size, double *fval);

#endif
