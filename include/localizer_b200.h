/*
 * localizer_b200 — C ABI of the B200 Gaussian localization engine.
 *
 * Drop-in for the per-emitter Levenberg-Marquardt fitting path of Localizer:
 * the FitPositions_* family (reference source/Localization.h:55-121,
 * source/Localization.cpp:43-631), with the same method codes, PSF-width and
 * noise-weight inputs, ROI half-width rule and output position columns
 * (source/Storage.cpp:268-290, 405-425, 614-640). Plain pointers and sizes
 * only; device pointers are CUDA global-memory addresses on the context's
 * device, streams are cudaStream_t passed as void*.
 *
 * Error convention (mirrors LocalizerDLL, source/LocalizerDLL.cpp:124-128,
 * where every failure returns -1): every int-returning call returns 0 on
 * success and a negative LOC_E* code on failure; loc_last_error() gives a
 * thread-local message for the last failure on the calling thread.
 */
#ifndef LOCALIZER_B200_H
#define LOCALIZER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define LOC_API __declspec(dllexport)
#else
#define LOC_API __attribute__((visibility("default")))
#endif

/* Method codes: LOCALIZATION_METHOD_* of source/Defines.h:157-163. */
#define LOC_METHOD_2DGAUSS 0                          /* FitPositions_SymmetricGaussian */
#define LOC_METHOD_2DGAUSS_FIXEDWIDTH 1               /* FitPositions_FixedWidthGaussian */
#define LOC_METHOD_2DGAUSS_ELLIPSOIDAL 5              /* FitPositions_EllipsoidalGaussian_SymmetricPSF */
#define LOC_METHOD_MLEWG 6                            /* FitPositions_MLEwG: FP64 Nelder-Mead maximum
                                                         likelihood (Localization.cpp:633-789); output
                                                         columns frame, integral, width, x, y,
                                                         background, position deviation, frames
                                                         present; sigma is unused; not available in
                                                         loc_fit_batch_static or with a proposal */
#define LOC_METHOD_2DGAUSS_ELLIPSOIDAL_ASTIGMATISM 7  /* FitPositions_EllipsoidalGaussian */

/* Per-candidate reject codes (0 = kept: the candidate produced an output row
 * in the reference). Each names the reference check that erases it. */
#define LOC_FLAG_KEPT 0
#define LOC_FLAG_EDGE 1            /* ROI leaves the frame, Localization.cpp:120 */
#define LOC_FLAG_AMPLITUDE 2       /* fitted amplitude <= 0, :160 */
#define LOC_FLAG_OUT_OF_WINDOW 3   /* fitted centre outside the ROI, :166 */
#define LOC_FLAG_WIDTH_RANGE 4     /* symmetric width outside [0.4, 1.5] w0, :179 */
#define LOC_FLAG_DRIFT 5           /* fixed width: centre moved > 2 w0, :349 */
#define LOC_FLAG_EIGEN 6           /* ellipsoid eigen-decomposition failed, :534 */
#define LOC_FLAG_NO_AXIS 7         /* no ellipsoid axis in [0.4, 1.5] w0, :550 */
#define LOC_FLAG_SYMPSF_RATIO 8    /* method 5: axis ratio outside [0.75, 1.25], :616 */
#define LOC_FLAG_SYMPSF_WIDTH 9    /* method 5: no axis in [0.7, 1.3] w0, :621 */
#define LOC_FLAG_BAD_INPUT 10      /* frame index out of range or non-finite candidate */
#define LOC_FLAG_INTEGRAL 11       /* MLEwG: integral outside [1/2, 3/2] of the start, :753 */

/* Termination status column (the value of the reference's solver loop at
 * exit, Localization.cpp:148-155): 0 converged (test_delta), 1 iteration
 * cap reached, otherwise the solver's stop code (GSL errno numbering:
 * 9 bad function value, 27 no progress, 29/30/31 tolerance too small). */
#define LOC_TERM_CONVERGED 0
#define LOC_TERM_MAX_ITER 1

/* Error codes. */
#define LOC_OK 0
#define LOC_E_INVALID -1      /* bad argument */
#define LOC_E_CUDA -2         /* CUDA runtime error */
#define LOC_E_NOMEM -3        /* device or host allocation failed */
#define LOC_E_UNSUPPORTED -4  /* method / size outside what this build handles */
#define LOC_E_DEVICE -5       /* a kernel reported an error word */

#define LOC_MAX_HALF_WIDTH 16 /* largest ROI half-width r (ROI (2r+1)^2) */

/* Candidate emitter: the reference's Particle (source/Storage.h:90-101,
 * produced by the particle finders, source/ParticleFinding.cpp:351-377)
 * plus the frame it belongs to and an optional ROI half-width override.
 * half_width == 0 selects the reference rule r = ceil(4 * w0)
 * (source/Localization.h:68). 40 bytes, 8-byte aligned. */
typedef struct loc_candidate {
    double x;            /* pixel coordinate along rows (fastest image axis) */
    double y;            /* pixel coordinate along columns */
    double intensity;    /* initial amplitude */
    double background;   /* initial offset */
    int32_t frame;       /* index into the frame stack */
    int32_t half_width;  /* ROI half-width r, or 0 for ceil(4*w0) */
} loc_candidate;

/* Precision of the iterative solve. FP32 is the production path (FP32
 * model, Jacobian and normal equations; fits whose FP32 outcome could depend
 * on FP32 rounding are re-run in FP64, see fp64_rerun and the rerun_*
 * fields; the final covariance and columns are FP64). FP64 runs the same
 * algorithm entirely in double precision for every fit. */
#define LOC_PRECISION_FP32 0
#define LOC_PRECISION_FP64 1

typedef struct loc_options {
    int32_t max_iter;          /* solver iteration cap; 200 in the reference */
    double epsabs;             /* test_delta absolute tolerance; 1e-4 */
    double epsrel;             /* test_delta relative tolerance; 1e-4 */
    int32_t precision;         /* LOC_PRECISION_* */
    float pivot_threshold;     /* FP32 Cholesky pivots below this fraction of
                                  their diagonal are redone in FP64 inside the
                                  FP32 solver; 0 (default): off, ill-conditioned
                                  fits are re-run in FP64 instead (fp64_rerun) */
    int32_t threads_per_block; /* 0: tuned default */
    int32_t blocks_per_sm;     /* 0: occupancy maximum */
    int32_t stage_u16;         /* reserved, ignored: ROIs are staged in shared
                                  memory as FP32 (kept for the struct layout) */
    int32_t max_half_width;    /* 0: the solver reads the largest ROI half-width
                                  present back from the device (one small
                                  synchronous copy); > 0: caller guarantees
                                  every candidate's r is at most this (no host
                                  synchronisation, capturable in a CUDA graph);
                                  larger candidates are flagged LOC_FLAG_BAD_INPUT */
    const float *d_init_params;/* optional device array, n_cands x p floats of
                                  absolute-coordinate start parameters (warm
                                  start); NULL = reference start values; a NaN
                                  first value selects the reference start for
                                  that candidate */
    float *d_params_out;       /* optional device array, n_cands x p floats:
                                  raw fitted parameters (absolute coordinates) */
    float *d_diag;             /* optional device array, n_cands x 8 floats of
                                  solver diagnostics: smallest undamped pivot
                                  ratio, last step / stopping tolerance, FP64
                                  pivot escalations, smallest relative margin
                                  of a solver branch decision, 1 if the fit was
                                  re-run in FP64, iterations and status of the
                                  FP32 run, reserved */
    int32_t threads_per_fit;   /* threads cooperating on one fit in the first
                                  scheduling level: 1 (default), 4, 8 or 16 */
    int32_t tail_threads_per_fit; /* threads per fit for fits that outlive the
                                  first level's budget: 8 (default), 4 or 1 */
    int32_t level0_budget;     /* solver iterations a fit may use in the first
                                  level before it is suspended and finished by
                                  the second; 0 = default (32), < 0 = one
                                  level only */
    int32_t fp64_rerun;        /* 0 (default): FP32 fits whose result could
                                  depend on FP32 rounding are re-run entirely in
                                  FP64 on the GPU (a solver branch decision within
                                  rerun_margin of its threshold, an undamped pivot
                                  ratio below rerun_pivot, a stop for lack of
                                  progress, or at least rerun_iters iterations;
                                  fits that reach max_iter only with rerun_capped);
                                  -1: never */
    float rerun_margin;        /* 0: default 1e-4 */
    float rerun_pivot;         /* 0: default 1e-4 */
    int32_t rerun_threads_per_fit; /* threads per fit of the FP64 re-run: 2
                                  (default), 1, 4 or 8 */
    int32_t serial_classes;    /* 0 (default): the ROI classes are solved as
                                  concurrent chains on the context's auxiliary
                                  streams, joined back to the call's stream;
                                  1: all on the call's stream */
    const struct loc_proposal *proposal; /* optional trained start proposal
                                  (loc_proposal_*) for this method: every
                                  candidate's start is proposed by the network
                                  and kept when its residual over the ROI is not
                                  worse than the reference start's; NULL (default):
                                  reference start values. Takes precedence over
                                  d_init_params. */
    int32_t warm_iter_limit;   /* with a proposal: warm-started fits that needed
                                  more solver iterations than this are re-run
                                  from the reference start (in FP64, the
                                  reference's algorithm); 0: default 8, < 0: never */
    int32_t long_rerun_iters;  /* FP64 re-runs of fits whose FP32 solve took more
                                  iterations than this form their own queue,
                                  solved with long_rerun_threads_per_fit threads
                                  per fit on a second stream of their chain (they
                                  set the length of the re-run); 0: default, the
                                  level-0 budget; < 0: one queue */
    int32_t long_rerun_threads_per_fit; /* 1, 2, 4 or 8; 0: default 8 */
    int32_t compensated;       /* 1: two-level summation of the FP32 normal
                                  equations: each of a fit's threads sums its
                                  share of the ROI pixels in FP32 and the
                                  partial sums are combined in FP64 and rounded
                                  once (the first scheduling level then runs at
                                  least 4 threads per fit); 0 (default): FP32
                                  throughout */
    int32_t rerun_capped;      /* 1: fits the FP32 solver stopped at max_iter are
                                  re-run in FP64 as well; 0: they are kept as
                                  they are */
    float rerun_cond;          /* > 0: a fit is also re-run in FP64 when its
                                  closest branch margin is below rerun_cond x
                                  FP32 epsilon / its smallest undamped pivot
                                  ratio (the FP32 error its conditioning
                                  allows); 0 (default): off */
    int32_t rerun_iters;       /* fits whose FP32 solve took at least this many
                                  iterations are re-run in FP64 as well (long,
                                  slowly converging fits stop where their path
                                  takes them under the reference's test_delta, so
                                  FP32 rounding moves their end point); 0: default,
                                  16 for the ellipsoidal methods 5 and 7, off for
                                  methods 0 and 1; < 0: off */
    float rerun_skip_rejected; /* > 0: a flagged fit whose FP32 end point is
                                  rejected by a clear margin (centre more than
                                  this many px outside its ROI, amplitude below
                                  zero by more than this fraction of its
                                  offset, or every width more than this fraction
                                  outside [0.4, 1.5] w0) is not re-run in FP64;
                                  only its reject code could change; 0
                                  (default): 0.5 for the ellipsoidal methods 5
                                  and 7, off for methods 0 and 1; < 0: off;
                                  never applied with a proposal (a warm fit's
                                  end point says nothing about the reference
                                  start's) */
    int32_t host_roi_mode;     /* loc_fit_host / loc_fit_host_async: 0
                                  (default): when the candidates' ROIs hold
                                  fewer than half the stack's pixels and there
                                  are at least 10^5 candidates, only the ROIs
                                  cross PCIe (gathered by host threads into one
                                  packed stack, each ROI at its own size; rows
                                  identical to the whole-frame upload); > 0:
                                  whenever the stack is smaller than the
                                  frames; < 0: always whole frames. Not with a
                                  proposal or method 6 */
} loc_options;

/* Fills *opt with the reference's defaults. */
LOC_API void loc_default_options(loc_options *opt);

typedef struct loc_ctx loc_ctx;

/* Create a context on CUDA device `device` (device memory pools, tuned
 * launch shapes, counters). The context is not thread-safe; use one per
 * host thread. */
LOC_API int loc_ctx_create(loc_ctx **ctx, int device);
LOC_API int loc_ctx_destroy(loc_ctx *ctx);

/* Thread-local description of the last failure on this thread. */
LOC_API const char *loc_last_error(void);

/* Number of reference output columns for a method (12 / 10 / 16), or a
 * negative error. Rows written by the fit calls carry two more columns:
 * the solver's iteration count and the termination status. */
LOC_API int loc_reference_columns(int method);
LOC_API int loc_output_columns(int method);

/* Number of fitted parameters for a method (5 / 4 / 7). */
LOC_API int loc_parameter_count(int method);

/*
 * Fit every candidate of a frame stack on the GPU (the batched
 * FitPositions::fit_positions, reference source/Localization.h:60, called
 * per frame at source/PALMAnalysis.cpp:234).
 *
 * d_frames: n_frames x n_cols x n_rows uint16, x fastest (frame f, pixel
 *           (x, y) at f*n_rows*n_cols + x + y*n_rows), as the reference
 *           lays out images (source/Defines.h:44, source/FileIO.cpp:195).
 * d_cands:  n_cands candidates (any order; any frames).
 * d_out:    n_cands rows of loc_output_columns(method) doubles, one row per
 *           candidate in submission order. Rows of kept candidates hold the
 *           reference's columns; the reference columns of rejected rows are
 *           NaN except column 0 (frame).
 * d_flags:  n_cands reject codes (LOC_FLAG_*).
 * w0:       initialPSFWidth (> 0); sigma: the noise weight (non-zero).
 * Asynchronous on `stream`; device errors are reported by the next call or
 * by loc_sync.
 */
LOC_API int loc_fit_batch(loc_ctx *ctx, const uint16_t *d_frames, int n_frames, int n_rows,
                          int n_cols, const loc_candidate *d_cands, int n_cands, int method,
                          double w0, double sigma, const loc_options *opt, double *d_out,
                          uint8_t *d_flags, void *stream);

/* Same fit with host buffers: copies frames and candidates to the device,
 * fits and copies rows and flags back (the whole path a host caller sees).
 * Where the candidates' ROIs are a small part of the frames (host_roi_mode),
 * the host threads gather the candidates' ROIs into one packed stack and
 * only the stack (plus one pixel offset per candidate) is copied; the solver
 * reads the same pixels from it. */
LOC_API int loc_fit_host(loc_ctx *ctx, const uint16_t *frames, int n_frames, int n_rows,
                         int n_cols, const loc_candidate *cands, int n_cands, int method,
                         double w0, double sigma, const loc_options *opt, double *out,
                         uint8_t *flags);

/*
 * The same fit for a stream of stacks (the reference's analysis keeps its
 * worker threads busy on frame after frame, source/PALMAnalysis.cpp:126-130,
 * 196-250): enqueues the upload, the fit and the download of one stack and
 * returns without waiting. Calls run in order; the upload of a call overlaps
 * the fit of the one before it and its download the fit of the one after
 * it (two device slots used in turn). `frames`, `cands`, `out` and `flags`
 * must stay valid, and `out`/`flags` unread, until loc_fit_host_wait
 * returns; pinned host memory (cudaHostAlloc / cudaHostRegister) is needed
 * for the copies to overlap (in ROI mode the frames are read by the host
 * threads during the call and the ROI stack is copied from the library's
 * own pinned staging). Make no other fit call on the context while calls are in
 * flight. Results are identical to loc_fit_host's.
 */
LOC_API int loc_fit_host_async(loc_ctx *ctx, const uint16_t *frames, int n_frames, int n_rows,
                               int n_cols, const loc_candidate *cands, int n_cands, int method,
                               double w0, double sigma, const loc_options *opt, double *out,
                               uint8_t *flags);
/* Waits for every loc_fit_host_async call of the context; reports the first
 * device error of those calls. */
LOC_API int loc_fit_host_wait(loc_ctx *ctx);

/* Bytes the context's host-buffer calls (loc_fit_host, loc_fit_host_async)
 * have copied host -> device and device -> host since it was created. */
LOC_API int loc_host_bytes(const loc_ctx *ctx, uint64_t *h2d, uint64_t *d2h);

/*
 * Allocation-free form of loc_fit_batch (same arguments, no context, same
 * results for methods 0, 1, 5 and 7; method 6 and start proposals are
 * refused with LOC_E_UNSUPPORTED). It has no counterpart in the reference,
 * which fits on the CPU and allocates freely; it exists for callers that may
 * not allocate device memory: code running under a framework whose caching
 * allocator owns the device heap, plugins handed only their input and output
 * buffers, and acquisition loops that must not call cudaMalloc/cudaFree
 * between frames. All device scratch comes from one file-scope device array
 * of 16 MiB, reserved until the process exits on each GPU where the
 * library's device code is loaded (with CUDA's default lazy module loading:
 * where this entry point is used). At most 16384 candidates per call (larger
 * calls fail with LOC_E_UNSUPPORTED before any device work). Calls share the
 * array: the call resets what must start at zero, but calls that overlap on
 * the GPU race and must be serialised. The first call on a device resolves
 * the array's address; make it before any stream capture, and make no call
 * on a device after a cudaDeviceReset of it. Errors: negative LOC_E_* code,
 * message through loc_last_error().
 */
LOC_API int loc_fit_batch_static(const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                                 const loc_candidate *d_cands, int n_cands, int method, double w0,
                                 double sigma, const loc_options *opt, double *d_out, uint8_t *d_flags,
                                 void *stream);

/*
 * Launch-shape tuner (no reference counterpart: the reference's fit is a
 * serial CPU loop). Times the FP32 solver on a caller-supplied sample of
 * candidates (device buffers, as for loc_fit_batch; a few 10^4 to 10^5
 * candidates of the workload to be fitted) over its launch shapes -- threads
 * per block, threads per fit in the first and second scheduling levels, the
 * first level's iteration budget, threads per fit of the FP64 re-runs --
 * by coordinate descent with CUDA events (median of three calls per shape),
 * and keeps a shape only if it is at least 1 % faster and its rows match the
 * default shape's (at most one candidate in 10^4 with another reject code or
 * a position moved by 1e-3 px or more: the launch shape changes the FP32
 * summation order, nothing else). The winner is stored in the context for
 * `method` and used by later fit calls of that method wherever their
 * options leave these fields at 0. `base` supplies every other option
 * (NULL: defaults). Blocks until done; allocates its own output buffers.
 */
typedef struct loc_tuning {
    int32_t threads_per_fit;
    int32_t tail_threads_per_fit;
    int32_t level0_budget;
    int32_t rerun_threads_per_fit;
    int32_t long_rerun_threads_per_fit;
    int32_t threads_per_block;
    float ms_default;          /* device time of one call on the sample, default shape */
    float ms_tuned;            /* ... tuned shape */
    int32_t trials;            /* shapes timed */
    int32_t flag_changes;      /* reject codes that differ from the default shape's */
    int32_t position_changes;  /* kept positions that moved by >= 1e-3 px */
} loc_tuning;
LOC_API int loc_autotune(loc_ctx *ctx, const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                         const loc_candidate *d_cands, int n_cands, int method, double w0, double sigma,
                         const loc_options *base, loc_tuning *result, void *stream);

/* Wait for all work of the context on `stream` and report device errors. */
LOC_API int loc_sync(loc_ctx *ctx, void *stream);

/* Counters of the last fit call (after loc_sync): trial-point evaluations,
 * Jacobian evaluations, damped Cholesky solves, FP64 pivot escalations,
 * candidates enqueued, total solver iterations, and the device time of each
 * stage (CUDA events on the call's stream; not recorded while the stream is
 * being captured into a graph). */
typedef struct loc_stats {
    uint64_t f_evals;
    uint64_t jacobian_evals;
    uint64_t lambda_solves;
    uint64_t fp64_escalations;
    uint64_t fits;
    uint64_t iterations;
    uint64_t pixels_f;     /* sum over trial evaluations of ROI pixels */
    uint64_t pixels_j;     /* sum over Jacobian evaluations of ROI pixels */
    uint64_t kcycles_refill;  /* thousands of SM cycles, summed over warps, spent */
    uint64_t kcycles_step;    /* refilling fits, solving the damped step, in the */
    uint64_t kcycles_pass;    /* pixel pass and in the accept/reject decision */
    uint64_t kcycles_decide;
    uint64_t fits_fp64_rerun;       /* fits re-run in FP64 after the FP32 solve */
    uint64_t iterations_fp64_rerun; /* their solver iterations */
    uint64_t kcycles_fp64_rerun;    /* thousands of SM cycles (summed over warps) of the re-run */
    uint64_t kcycles_fp64_rerun_pass; /* ... of which in the pixel pass */
    float queue_ms;        /* device time of the work-queue build (-1 if not timed) */
    float solver_ms;       /* device time of the persistent solver kernel */
    float finalize_ms;     /* device time of the FP64 finaliser */
    float proposal_ms;     /* device time of the start proposal (-1 if none ran) */
    int32_t kernel_launches; /* kernels the last fit call launched */
    uint64_t fits_warm;    /* fits started from the proposal's parameters */
} loc_stats;
LOC_API int loc_last_stats(loc_ctx *ctx, loc_stats *stats);

/*
 * Reference output matrix of the kept rows: the N x C double matrix that
 * getLocalizedPositionsAsMatrix() returns (Storage.cpp:268-290, 405-425,
 * 614-640), rows in submission order (the reference sorts by frame,
 * PALMAnalysis.cpp:188, so submit candidates in frame order), stored
 * column-major like the reference's Eigen matrix. Host buffers.
 * Returns the number of kept rows, or a negative error; writes at most
 * max_rows rows.
 */
LOC_API int loc_compact_host(const double *out, const uint8_t *flags, int n_cands, int method,
                             double *matrix, int max_rows);

/*
 * Candidate finder on one frame stack (host): the GLRT detector
 * (ThresholdImage_GLRT_FFT, source/Segmentation.cpp:241-430) followed by the
 * adjacent-8 particle finder (source/ParticleFinding.cpp:283-427), one
 * loc_candidate per particle in frame order, half_width 0.
 * Returns the number of candidates found (may exceed max_cands; only
 * max_cands are written) or a negative error.
 */
LOC_API long loc_find_candidates_host(const uint16_t *frames, int n_frames, int n_rows,
                                      int n_cols, double pfa, double psf_width, int n_threads,
                                      loc_candidate *cands, long max_cands);

/*
 * Synthetic frames on the device (workload generation for tests and
 * benchmarks; not part of the fit path): background + point-sampled 2D
 * Gaussians, Poisson shot noise plus Gaussian read noise, uint16 output.
 * d_emitters: 5 floats per emitter (x, y, amplitude, sigma_x, sigma_y),
 * grouped by frame; d_frame_start: n_frames + 1 offsets into it;
 * d_background: one value per frame. No reference counterpart (the
 * reference reads camera files, source/FileIO.cpp).
 */
LOC_API int loc_synth_frames(uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                             const float *d_emitters, const int *d_frame_start,
                             const float *d_background, float read_noise, unsigned long long seed,
                             void *stream);

/*
 * Frame ingest (reference BufferWithFormatToImage / CopyBufferToImage,
 * source/FileIO.cpp:195-234, FileIO.h:96-116): n_frames camera buffers of
 * storage type `format` (the reference's LocalizerStorageType codes,
 * source/Defines.h:82-95: 2 int8, 3 uint8, 4 int16, 5 uint16, 6 int32,
 * 7 uint32, 8 int64, 9 uint64, 10 float, 11 double; the 4-bit types are not
 * supported), each n_rows x n_cols and column-major (row_major = 0, element
 * (i, j) at i + j * n_rows) or row-major (1, at i * n_cols + j), to the fit
 * path's uint16 stack. Values are rounded to the nearest integer and clamped
 * to [0, 65535]; returns the number of pixels whose value that changed (0:
 * lossless, as for 8/16-bit unsigned cameras), or a negative error. Device
 * buffers; blocks until done.
 */
LOC_API long long loc_ingest_frames(const void *d_src, int format, int n_frames, int n_rows, int n_cols,
                                    int row_major, uint16_t *d_dst, void *stream);

/*
 * Text file of the kept positions in the reference's format
 * (LocalizedPositionsContainer_*::writePositionsToFile, reference
 * source/Storage.cpp:292-345, 427-470, 642-700): title line, `header`, "DATA
 * FOLLOWS", column titles, one tab-separated line per row whose flag is 0 (all
 * rows if flags is NULL), in row order. rows: n host rows as the fit calls
 * write them (loc_output_columns(method) doubles). Byte-identical to the
 * reference's file for the same positions. Returns the number of positions
 * written; LOC_E_INVALID if none is kept (the reference throws "No
 * positions localized!") or the file cannot be written.
 */
LOC_API long loc_write_positions_text(const double *rows, const uint8_t *flags, long n, int method,
                                      const char *path, const char *header);

/*
 * GLRT + adjacent-8 candidate finder on the GPU (reference
 * ThresholdImage_GLRT_FFT, source/Segmentation.cpp:241-430, and
 * ParticleFinder_adjacent8, source/ParticleFinding.cpp:283-427), with the
 * same results, bit for bit and in the same order, as
 * loc_find_candidates_host. d_frames: device frame stack (x fastest);
 * d_cands: device array receiving up to max_cands candidates in frame order
 * (half_width 0). Returns the total number found (which may exceed
 * max_cands: call again with a larger buffer), or a negative error. Blocks
 * until the candidates are written. PSF widths up to 8 px (window <= 33).
 */
LOC_API long loc_find_candidates(const uint16_t *d_frames, int n_frames, int n_rows, int n_cols, double pfa,
                                 double psf_width, loc_candidate *d_cands, long max_cands, void *stream);

/*
 * Learned start proposal (no reference counterpart: the reference starts
 * every fit from the finder's centroid and the PSF width, Localization.cpp
 * :122-142, 301-321, 466-491). A small convolutional network (1x11x11 window
 * -> 3x3 convolutions with 16, 32, 32 channels -> linear head with one output
 * per fit parameter) trained on synthetic windows labelled by the LM fit
 * itself. Weights are FP32 masters; the two wide convolutions run on the
 * tensor cores in BF16 with FP32 accumulation. Handles belong to one device.
 */
typedef struct loc_proposal loc_proposal;

/* Weight count of the network for a method (its head has one output per
 * parameter: 5, 4 or 7), or a negative error. */
LOC_API int loc_proposal_weight_count(int method);
/* New network with deterministic He-normal weights from `seed`. */
LOC_API int loc_proposal_create(loc_proposal **net, int device, int method, unsigned long long seed);
LOC_API int loc_proposal_destroy(loc_proposal *net);
/* FP32 master weights, host buffers of loc_proposal_weight_count floats.
 * Setting weights also resets the optimiser state. */
LOC_API int loc_proposal_get_weights(loc_proposal *net, float *weights, int n);
LOC_API int loc_proposal_set_weights(loc_proposal *net, const float *weights, int n);
/*
 * Raw head outputs for a stack of 11 x 11 uint16 windows (x fastest, window
 * centre at (5, 5)): d_out receives n x P floats; d_index (optional) gathers
 * window d_index[i] for row i; d_stat (optional) receives n x 2 floats of the
 * window normalisation (border mean b0, scale s0). Device buffers.
 */
LOC_API int loc_proposal_forward(loc_proposal *net, const uint16_t *d_rois, const int *d_index, int n,
                                 float *d_out, float *d_stat, void *stream);
/*
 * Training objective over a batch: mean over windows of sum_j lam[j] (o_j -
 * t_j)^2, t the label mapped to the network's output scale (log amplitude /
 * s0, log width / 1.5, position relative to the window centre, correlation,
 * (offset - b0) / s0). d_labels: N x P floats in the method's parameter order
 * with positions relative to the window centre, row d_index[i] used for
 * window i; lam: P host floats. loc_proposal_gradient writes the gradient
 * (weight layout) to d_grad and the loss to *loss; loc_proposal_train_step
 * also applies one Adam step of learning rate lr.
 */
LOC_API int loc_proposal_gradient(loc_proposal *net, const uint16_t *d_rois, const int *d_index, int n,
                                  const float *d_labels, const float *lam, float *d_grad, float *loss,
                                  void *stream);
LOC_API int loc_proposal_train_step(loc_proposal *net, const uint16_t *d_rois, const int *d_index, int n,
                                    const float *d_labels, const float *lam, float lr, float *loss, void *stream);
/* LOC_OK, or LOC_E_CUDA if a tensor-core wait in a proposal kernel ran out
 * (the kernel then skipped its remaining work). */
LOC_API int loc_proposal_status(loc_proposal *net);
/*
 * Synthetic training windows (11 x 11 uint16, x fastest) from the fit's
 * forward model: one emitter within 1 px of the centre, widths U[1, 2] px
 * (independent per axis if elliptic), amplitude lognormal (median 500,
 * log-sd 0.6), background U[50, 200], Poisson(0.5) neighbours, Poisson +
 * Gaussian read noise (sd 2). d_truth (optional): n x 6 floats (x, y,
 * amplitude, sigma_x, sigma_y, background). No reference counterpart.
 */
LOC_API int loc_synth_rois(uint16_t *d_rois, int n, int elliptic, unsigned long long seed, float *d_truth,
                           void *stream);

/*
 * Compatibility entry points with the signatures of the reference DLL
 * (source/LocalizerDLL.h:53-56): GLRT + adjacent-8 candidates, then the
 * ellipsoidal fit (FitPositions_EllipsoidalGaussian(psfWidth, 1.0),
 * LocalizerDLL.cpp:107) on the GPU; *emitterCoordinates receives the
 * N x 16 column-major matrix, allocated by the callee; release it with
 * LocalizerFree. Returns 0 or -1, as the reference does.
 */
LOC_API int LocalizerFitEmitters(unsigned short *imageData, int nRows, int nCols, int nImages,
                                 double psfWidth, double glrtInsensitivity, int *nEmitters,
                                 double **emitterCoordinates);
LOC_API void LocalizerFree(double *ptrToFree);

#ifdef __cplusplus
}
#endif

#endif
