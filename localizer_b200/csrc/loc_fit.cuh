// Host-side interface of the fit kernels (used by the C ABI layer).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "loc_proposal.cuh"

namespace locb {

constexpr int kMaxHalfWidth = 16;  // LOC_MAX_HALF_WIDTH
constexpr int kMaxAux = 4;         // auxiliary streams the per-class chains are spread over

// Device scratch of one fit call. The caller provides the memory; sizes in
// bytes come from scratch_bytes().
struct Scratch {
    int *cls;            // n: ROI half-width class of each candidate, -1 if not enqueued
    int *order;          // n: enqueued candidates grouped by class
    int *meta;           // kMetaInts: class table (see loc_fit.cu)
    void *state;         // n * state_stride(method) elements of the solver precision
    unsigned long long *stats;  // 8 counters
    int *cont;           // n: continuation queue (fits suspended after the level-0 budget)
    float *cont_state;   // n * cont stride: their saved solver state
    int *cls2;           // n: half-width class of fits re-run in FP64, -1 otherwise
    int *order2;         // n: their queue (fits whose FP32 solve ended within the level-0 budget)
    int *meta2;          // kMetaInts: its class table
    int *order3;         // n: queue of the long re-runs (FP32 solve outlived the level-0 budget)
    int *meta3;          // kMetaInts: its class table
    double *state64;     // n * state_stride(method): FP64 state of re-run fits
    float *init;         // n * P: proposed starts (warm mode only)
};

constexpr int kMetaInts = 8 + 8 * (kMaxHalfWidth + 1);

struct FitParams {
    const uint16_t *frames;
    int n_frames, n_rows, n_cols;
    const void *cands;  // loc_candidate / Cand
    int n_cands;
    int method;
    double w0, sigma;
    int max_iter;
    double epsabs, epsrel;
    int precision;       // 0 fp32, 1 fp64
    float pivot_thr;
    int threads_per_block;
    int blocks_per_sm;
    int max_half_width;  // largest r present (known to the caller) or 0 = read back
    int threads_per_fit;       // level 0: 1, 4 or 8
    int tail_threads_per_fit;  // level 1: 1, 4 or 8
    int level0_budget;         // iterations before a fit moves to level 1 (0: single level)
    int fp64_rerun;            // re-run flagged FP32 fits in FP64
    int rerun_threads_per_fit; // 1, 2, 4 or 8
    int long_rerun_threads_per_fit; // 1, 2, 4 or 8: re-runs of fits whose FP32 solve took more
                                    // than long_rerun_iters iterations
    int long_rerun_iters;      // 0: no separate long queue
    int compensated;           // FP32 group sums of the normal equations in FP64 (threads per fit > 1)
    int rerun_capped;          // also re-run in FP64 the fits FP32 stopped at the iteration cap
    float rerun_cond;          // > 0: margin threshold raised to rerun_cond * eps32 / smallest pivot ratio
    int rerun_iters;           // > 0: also re-run fits whose FP32 solve took at least this many iterations
    float rerun_skip_rejected; // > 0: flagged fits that end clearly rejected in FP32 are not re-run
    float rerun_margin;        // branch-decision margin below which a fit is flagged
    float rerun_pivot;         // undamped pivot ratio below which a fit is flagged
    const float *init_params;
    bool warm;                 // start proposal active (prop, warm_iter_limit)
    ProposalView prop;
    int warm_iter_limit;       // warm fits with more iterations are re-run from the reference start
    cudaEvent_t ev_prop;       // optional: after the proposal kernel
    int *launches;             // optional: incremented per kernel launch
    float *params_out;
    float *diag;
    cudaEvent_t ev[4];   // optional: before the queue build, around the solver, after the finaliser
    cudaStream_t aux[kMaxAux];  // optional auxiliary streams (NULL-terminated) for the class chains
    cudaEvent_t fork;           // fork / join events for them
    cudaEvent_t join[kMaxAux];
    cudaStream_t aux_long[kMaxAux];  // optional streams for the long FP64 re-runs, one per chain
    cudaEvent_t flagged[kMaxAux];    // chain j's flag pass done
    cudaEvent_t join_long[kMaxAux];
    double *out;
    uint8_t *flags;
    // ROI mode (host-buffer calls): the pixels are not whole frames but the
    // candidates' ROIs packed one after another, candidate i's (2r+1)^2 ROI
    // (row pitch 2r+1, x fastest) starting at pixel roi_slot[i] of roi_stack,
    // which holds roi_px pixels (roi_slot NULL: frame mode). Frames,
    // n_frames, n_rows and n_cols above still describe the original stack
    // (the edge and input rules use them).
    const int *roi_slot;
    const uint16_t *roi_stack;
    long long roi_px;
};

int state_stride(int method);
size_t scratch_bytes(int method, int n_cands, int precision, int rerun, int warm = 0);
void carve_scratch(void *base, int method, int n_cands, int precision, int rerun, Scratch *s, int warm = 0);
constexpr int kStatWords = 2 * 12 + 2;  // solver counters, FP64 re-run counters, proposals taken, spare

// Enqueue the whole fit on `stream`. Returns cudaSuccess or the launch error;
// *used_smem_side receives the ROI side the solver was sized for.
cudaError_t enqueue_fit(const FitParams &p, const Scratch &s, cudaStream_t stream, int *err_detail);

// MLEwG (method 6): one kernel, no scratch but the statistics counters.
cudaError_t enqueue_mlewg(const FitParams &p, unsigned long long *stats, cudaStream_t stream);

}  // namespace locb
