// Allocation-free batched fit: the same fit as loc_fit_batch, with every
// byte of its device scratch (work queues, solver state, FP64 re-run
// buffers, counters) taken from one file-scope device array instead of a
// context's cudaMalloc'd pool.
//
// Who needs this: callers that may not allocate device memory themselves
// or through us -- code that runs under a framework which owns the whole
// device heap through its own caching allocator (a raw cudaMalloc behind its
// back fragments the pool and is invisible to its accounting), plugins that
// are handed only input and output buffers by their host, and real-time
// acquisition loops in which a cudaMalloc/cudaFree (which can synchronise the
// device) is not allowed between frames.
//
// Limits and sharing rules:
//  - at most kStaticMaxCands candidates per call (16384); larger calls are
//    rejected with LOC_E_UNSUPPORTED before any device work;
//  - the array (kStaticScratchBytes, 16 MiB) is reserved, until the process
//    exits, on every GPU where the library's device code is loaded: with
//    lazy module loading (CUDA's default, CUDA_MODULE_LOADING=LAZY) that is
//    the GPUs on which this entry point has been called, with
//    CUDA_MODULE_LOADING=EAGER every GPU whose context loads the library;
//  - method 6 (MLEwG) and start proposals are not available here (they
//    need a context); every other method and option gives loc_fit_batch's
//    results;
//  - every call on a device uses the same array and leaves its contents
//    behind; the call clears what must start at zero (queue tables and
//    counters) itself, so results never depend on a previous call, but two
//    calls whose work overlaps on the GPU (different streams, or host threads
//    without ordering) race on the array and corrupt each other -- serialise
//    them;
//  - the first call on each device resolves the array's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture begins.
#include "../../include/localizer_b200.h"
#include "loc_fit.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

namespace locb {
int record_error_fixed(int code, const char *msg);
}

namespace {

constexpr int kStaticMaxCands = 16384;
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// resolved once per device; the address does not survive cudaDeviceReset
// (the module is loaded again and the array may move), so a process that
// resets a device must not call this entry point on it afterwards
// resolved once per device; the address does not survive cudaDeviceReset
// (the module is loaded again and the array may move), so a process that
// resets a device must not call this entry point on it afterwards
void *g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mu;

int err(int code, const char *msg) { return locb::record_error_fixed(code, msg); }

}  // namespace

extern "C" LOC_API int loc_fit_batch_static(const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                                            const loc_candidate *d_cands, int n_cands, int method, double w0,
                                            double sigma, const loc_options *opt, double *d_out, uint8_t *d_flags,
                                            void *stream)
{
    if (!(method == 0 || method == 1 || method == 5 || method == 7)) return err(LOC_E_UNSUPPORTED, "unsupported method code");
    if (n_cands < 0) return err(LOC_E_INVALID, "n_cands < 0");
    if (n_cands > kStaticMaxCands) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "loc_fit_batch_static: %d candidates exceed the static scratch limit of %d per call; "
                      "split the batch or use loc_fit_batch",
                      n_cands, kStaticMaxCands);
        return err(LOC_E_UNSUPPORTED, msg);
    }
    if (n_cands > 0 && (!d_cands || !d_out || !d_flags)) return err(LOC_E_INVALID, "NULL buffer");
    if (n_frames < 0 || n_rows <= 0 || n_cols <= 0) return err(LOC_E_INVALID, "bad frame stack shape");
    if (n_frames > 0 && !d_frames) return err(LOC_E_INVALID, "frames is NULL");
    if (!(w0 > 0) || !std::isfinite(w0)) return err(LOC_E_INVALID, "w0 must be finite and > 0");
    if (!(sigma != 0) || !std::isfinite(sigma)) return err(LOC_E_INVALID, "sigma must be finite and non-zero");
    loc_options o;
    if (opt) o = *opt;
    else loc_default_options(&o);
    if (o.max_iter < 1) return err(LOC_E_INVALID, "max_iter < 1");
    if (!(o.epsrel >= 0) || !(o.epsabs >= 0)) return err(LOC_E_INVALID, "negative tolerance");
    if (o.proposal) return err(LOC_E_UNSUPPORTED, "start proposals need a context (loc_fit_batch)");
    int tpf0 = o.threads_per_fit > 0 ? o.threads_per_fit : (o.compensated > 0 ? 4 : 1);
    if (o.compensated > 0 && tpf0 < 4) tpf0 = 4;
    const int tpf1 = o.tail_threads_per_fit > 0 ? o.tail_threads_per_fit : 8;
    if (!(tpf0 == 1 || tpf0 == 4 || tpf0 == 8) || !(tpf1 == 1 || tpf1 == 4 || tpf1 == 8))
        return err(LOC_E_INVALID, "threads per fit must be 1, 4 or 8");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return err(LOC_E_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices) return err(LOC_E_UNSUPPORTED, "device index beyond the static table");
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_ptr[dev]) {
            // host code may not use g_static_scratch's name as a device address
            e = cudaGetSymbolAddress(&g_scratch_ptr[dev], g_static_scratch);
            if (e != cudaSuccess) {
                g_scratch_ptr[dev] = nullptr;
                return err(LOC_E_CUDA, "cudaGetSymbolAddress of the static scratch failed");
            }
        }
        base = g_scratch_ptr[dev];
    }

    const int rerun = o.fp64_rerun >= 0 ? 1 : 0;
    if (locb::scratch_bytes(method, n_cands, o.precision, rerun) > kStaticScratchBytes)
        return err(LOC_E_UNSUPPORTED, "loc_fit_batch_static: scratch need exceeds the static array");
    locb::Scratch s;
    locb::carve_scratch(base, method, n_cands, o.precision, rerun, &s);

    locb::FitParams p{};
    p.frames = d_frames;
    p.n_frames = n_frames;
    p.n_rows = n_rows;
    p.n_cols = n_cols;
    p.cands = d_cands;
    p.n_cands = n_cands;
    p.method = method;
    p.w0 = w0;
    p.sigma = sigma;
    p.max_iter = o.max_iter;
    p.epsabs = o.epsabs;
    p.epsrel = o.epsrel;
    p.precision = o.precision;
    p.pivot_thr = o.pivot_threshold > 0 ? o.pivot_threshold : 0.0f;
    p.threads_per_block = o.threads_per_block;
    p.blocks_per_sm = o.blocks_per_sm;
    p.max_half_width = o.max_half_width;
    p.threads_per_fit = tpf0;
    p.tail_threads_per_fit = tpf1;
    p.level0_budget = o.level0_budget == 0 ? 32 : (o.level0_budget < 0 ? 0 : o.level0_budget);
    p.fp64_rerun = rerun;
    p.rerun_threads_per_fit = (o.rerun_threads_per_fit == 1 || o.rerun_threads_per_fit == 4 ||
                               o.rerun_threads_per_fit == 8) ? o.rerun_threads_per_fit : 2;
    p.long_rerun_threads_per_fit = (o.long_rerun_threads_per_fit == 1 || o.long_rerun_threads_per_fit == 2 ||
                                    o.long_rerun_threads_per_fit == 4) ? o.long_rerun_threads_per_fit : 8;
    p.long_rerun_iters = o.long_rerun_iters == 0 ? (p.level0_budget > 0 ? p.level0_budget : 32)
                                                 : (o.long_rerun_iters < 0 ? 0 : o.long_rerun_iters);
    p.compensated = o.compensated > 0 ? 1 : 0;
    p.rerun_capped = o.rerun_capped > 0 ? 1 : 0;
    p.rerun_cond = o.rerun_cond > 0 ? o.rerun_cond : 0.0f;
    // default: the iteration rule for the ellipsoidal fits only (symmetric
    // and fixed-width fits keep their FP32 end points to 1e-3 px without it)
    p.rerun_iters = o.rerun_iters == 0 ? (method == 5 || method == 7 ? 16 : 0)
                                       : (o.rerun_iters < 0 ? 0 : o.rerun_iters);
    p.rerun_skip_rejected = o.rerun_skip_rejected == 0.0f ? (method == 5 || method == 7 ? 0.5f : 0.0f)
                                                          : (o.rerun_skip_rejected < 0.0f ? 0.0f : o.rerun_skip_rejected);
    p.rerun_margin = o.rerun_margin > 0 ? o.rerun_margin : 1e-4f;
    p.rerun_pivot = o.rerun_pivot > 0 ? o.rerun_pivot : 1e-4f;
    p.init_params = o.d_init_params;
    p.params_out = o.d_params_out;
    p.diag = o.d_diag;
    p.out = d_out;
    p.flags = d_flags;
    // no context: no timing events, every ROI class on the caller's stream
    int detail = 0;
    e = locb::enqueue_fit(p, s, (cudaStream_t)stream, &detail);
    if (e != cudaSuccess)
        return detail == 1 ? err(LOC_E_UNSUPPORTED, "ROI too large for shared memory")
                           : err(LOC_E_CUDA, cudaGetErrorString(e));
    return LOC_OK;
}
