/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle of the Gaussian fitting path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this code, and only as the checker; the product never calls it.
 *
 * FP64 restatement of FitPositions_SymmetricGaussian / _FixedWidthGaussian /
 * _EllipsoidalGaussian / _EllipsoidalGaussian_SymmetricPSF::fit_positions
 * (reference source/Localization.cpp:43-631) and of the model and Jacobian
 * callbacks they use (:1007-1331), driven by the lmsder restatement in
 * lmsder_core.c. One output row per submitted candidate, in submission order.
 */
#ifndef LOC_ORACLE_H
#define LOC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as loc_candidate in the product's public header. */
typedef struct {
    double x, y, intensity, background; /* reference Particle, Storage.h:90-101 */
    int32_t frame;                      /* frame index into the stack */
    int32_t half_width;                 /* ROI half-width r; 0 -> ceil(4*w0) */
} oracle_candidate;

typedef struct {
    int max_iter;        /* 200 in the reference (Localization.cpp:155) */
    double epsabs;       /* 1e-4 (Localization.cpp:154) */
    double epsrel;       /* 1e-4 */
    int nthreads;        /* host threads used to spread candidates (>=1) */
    /* initial parameters per candidate (warm start), NULL for the reference's
     * cold start; layout as the method's parameter vector, absolute coords. */
    const double *init_params;
} oracle_options;

/* Number of reference output columns for a method code (12/10/16), 0 if the
 * method is not a Gaussian LM method. */
int oracle_ref_columns(int method);

/* Fit every candidate. out has nc rows of (oracle_ref_columns(method) + 2)
 * doubles: the reference columns, then the iteration count and the
 * termination status. flags gets one reject code per candidate (0 = kept).
 * params_out (optional) receives the raw fitted parameter vector (p doubles
 * per candidate, absolute coordinates) and fnorm_out the final |f|.
 * Returns 0, or a negative code for invalid arguments. */
int oracle_fit(const uint16_t *frames, int n_frames, int n_rows, int n_cols,
               const oracle_candidate *cands, int nc, int method, double w0,
               double sigma, const oracle_options *opt, double *out,
               uint8_t *flags, double *params_out, double *fnorm_out);

/* Model / Jacobian callbacks evaluated directly (unit tests of the kernels).
 * roi: (2r+1)^2 doubles, x fastest. J row-major n x p. */
int oracle_model_jacobian(int method, const double *params, double w0, double sigma,
                          double x_offset, double y_offset, int r, const double *roi,
                          double *f, double *J);

/* GLRT detection mask of one frame (ThresholdImage_GLRT_FFT,
 * Segmentation.cpp:241-430) by direct correlation; mask 255/0, x fastest. */
int oracle_glrt_mask(const uint16_t *frame, int n_rows, int n_cols, double pfa,
                     double psf_width, int32_t *mask);

/* adjacent-8 particle finder (ParticleFinding.cpp:283-427) on a mask.
 * Writes up to max_out particles as (x, y, intensity, background) and
 * returns the number found (which may exceed max_out). */
int oracle_find_adjacent8(const uint16_t *frame, int n_rows, int n_cols,
                          const int32_t *mask, double *out, int max_out);

/* Solver trajectory of one fit (tests of the lmsder restatement): after each
 * iterate() call, the cumulative trial evaluations and the current point. */
int oracle_trajectory(int method, const double *roi, int r, double x_offset, double y_offset, double w0,
                      double sigma, const double *x0, int max_rec, int *trials, double *xs);

/* Instrumentation of the last oracle_fit call: sums over all candidates. */
void oracle_last_counters(long *n_iterate_calls, long *n_f_evals, long *n_df_evals,
                          long *n_lambda_trials);

#ifdef __cplusplus
}
#endif

#endif
