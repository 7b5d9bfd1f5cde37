// C ABI of the B200 localization engine (declared in include/localizer_b200.h).
#include "../../include/localizer_b200.h"
#include "loc_fit.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

namespace {

thread_local std::string g_err;
// Messages recorded without heap allocation (by the allocation-free entry
// point); the most recent of the two is what loc_last_error returns.
thread_local char g_err_fixed[256];
thread_local bool g_err_fixed_latest = false;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    g_err_fixed_latest = false;
    return code;
}

int cuda_fail(cudaError_t e, const char *where)
{
    return fail(LOC_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

int method_ok(int m) { return m == 0 || m == 1 || m == 5 || m == 6 || m == 7; }

// Device buffer that grows on demand.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 8 + 4096;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

// Page-locked host buffer, grown on demand (the ROI staging of host calls).
struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 8 + 4096;
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

// ROI mode of the host-buffer calls. Instead of whole frames, the (2r+1)^2
// ROI of each candidate that the fit's input and edge rules keep (the rules
// of k0_classify, the reference's Localization.cpp:115-124) is copied into
// one packed stack, ROI after ROI in candidate order, each with its own row
// pitch 2r+1; only the stack and one pixel offset per candidate cross PCIe.
// The solver reads the same pixels from the stack, so the rows are those of
// the frame upload.
// Automatic ROI mode needs the stack to hold fewer bytes than kRoiFraction of
// the frames and at least kRoiMinCands candidates: otherwise the gather
// (thread start-up, one cache miss per ROI row) costs more than the copy it
// saves (measured: at 0.52 the gather of a single 1.8 M-candidate call took
// longer than the whole-frame copy it replaced; at 0.43 and 0.09 it paid)
constexpr double kRoiFraction = 0.5;
constexpr int kRoiMinCands = 100000;

struct RoiPlan {
    bool use = false;
    long long px = 0;   // pixels in the packed stack
};

int host_threads()
{
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hc ? hc : 1u, 32u));
}

// Copies the sd x sd ROI at src (row pitch src_pitch) to dst (row pitch sd).
// Rows of up to 16 pixels move as fixed 32-byte copies while such a copy
// ends inside the ROI: it spills into the following destination rows, which
// later copies overwrite. The remaining rows are copied exactly (two
// overlapping fixed copies), so nothing past the ROI is written. end bounds
// the source buffer.
inline void copy_roi(uint16_t *dst, const uint16_t *src, int sd, size_t src_pitch, const uint16_t *end)
{
    int j = 0;
    const int nfast = sd <= 16 && sd * sd >= 16 ? std::min(sd - 1, (sd * sd - 16) / sd + 1) : 0;
    if (nfast > 0 && src + (size_t)(nfast - 1) * src_pitch + 16 <= end)
        for (; j < nfast; ++j) std::memcpy(dst + (size_t)j * sd, src + (size_t)j * src_pitch, 32);
    for (; j < sd; ++j) {
        unsigned char *d = reinterpret_cast<unsigned char *>(dst + (size_t)j * sd);
        const unsigned char *s = reinterpret_cast<const unsigned char *>(src + (size_t)j * src_pitch);
        const size_t nb = (size_t)sd * sizeof(uint16_t);
        if (nb >= 16 && nb <= 32) {
            std::memcpy(d, s, 16);
            std::memcpy(d + nb - 16, s + nb - 16, 16);
        } else if (nb >= 8 && nb < 16) {
            std::memcpy(d, s, 8);
            std::memcpy(d + nb - 8, s + nb - 8, 8);
        } else {
            std::memcpy(d, s, nb);
        }
    }
}

// Writes one thread's contiguous byte range [begin, end) of the packed stack
// in order. Whole 64-byte lines inside the range go out as non-temporal
// stores (the stack is read only by the copy engine, so caching it would
// first cost a read of every line it touches); the partial lines at both
// ends, which the neighbouring threads' ranges share, use ordinary stores.
// A ROI is assembled in line[] behind the bytes still pending.
class StackWriter {
  public:
    StackWriter(unsigned char *begin, unsigned char *end) : begin_(begin), end_(end)
    {
        base_ = reinterpret_cast<unsigned char *>(reinterpret_cast<uintptr_t>(begin) & ~(uintptr_t)63);
        fill_ = (size_t)(begin - base_);
    }
    // room for the next ROI's bytes, at most kMaxRoiBytes
    uint16_t *slot() { return reinterpret_cast<uint16_t *>(line_ + fill_); }
    void commit(size_t bytes)
    {
        fill_ += bytes;
        size_t k = 0;
        for (; fill_ - k >= 64; k += 64, base_ += 64) put_line(line_ + k, base_, 64);
        if (k) {
            std::memmove(line_, line_ + k, fill_ - k);
            fill_ -= k;
        }
    }
    void finish()
    {
        if (fill_) put_line(line_, base_, fill_);
#if defined(__x86_64__)
        _mm_sfence();
#endif
    }
    static constexpr size_t kMaxRoiBytes = (size_t)(2 * locb::kMaxHalfWidth + 1) * (2 * locb::kMaxHalfWidth + 1) * 2;

  private:
    // bytes [0, n) of src belong at dst (64-byte aligned); only those inside
    // [begin_, end_) are written
    void put_line(const unsigned char *src, unsigned char *dst, size_t n)
    {
#if defined(__x86_64__)
        if (n == 64 && dst >= begin_ && dst + 64 <= end_) {
            const __m128i *q = reinterpret_cast<const __m128i *>(src);
            __m128i *d = reinterpret_cast<__m128i *>(dst);
            _mm_stream_si128(d, _mm_load_si128(q));
            _mm_stream_si128(d + 1, _mm_load_si128(q + 1));
            _mm_stream_si128(d + 2, _mm_load_si128(q + 2));
            _mm_stream_si128(d + 3, _mm_load_si128(q + 3));
            return;
        }
#endif
        unsigned char *lo = std::max(dst, begin_), *hi = std::min(dst + n, end_);
        if (hi > lo) std::memcpy(lo, src + (lo - dst), (size_t)(hi - lo));
    }
    unsigned char *begin_, *end_, *base_;
    size_t fill_;
    alignas(64) unsigned char line_[64 + kMaxRoiBytes + 64];
};

// off[i]: the first pixel of the candidate's ROI in the packed stack, -1 for
// a candidate the fit rejects before reading pixels. Gathers into roi when
// the stack holds fewer bytes than max_fraction of the frames (and fewer
// than 2^31 pixels, the range of the offsets).
RoiPlan plan_and_gather_rois(const uint16_t *frames, int n_frames, int n_rows, int n_cols, const loc_candidate *c,
                             int n, double w0, int max_half_width, bool force, int *off, HostBuf *roi,
                             cudaError_t *err)
{
    RoiPlan plan;
    *err = cudaSuccess;
    if (n <= 0) return plan;
    const int r_default = (int)std::ceil(w0 * 4.0);
    const int r_cap = max_half_width > 0 ? std::min(max_half_width, locb::kMaxHalfWidth) : locb::kMaxHalfWidth;
    const int nt = std::min(host_threads(), std::max(1, n / 4096));
    std::vector<long long> cnt(nt, 0), npx(nt, 0);
    auto chunk = [&](int t, int &lo, int &hi) {
        lo = (int)((long long)n * t / nt);
        hi = (int)((long long)n * (t + 1) / nt);
    };
    auto run = [&](auto fn) {
        std::vector<std::thread> th;
        for (int t = 1; t < nt; ++t) th.emplace_back(fn, t);
        fn(0);
        for (auto &x : th) x.join();
    };
    auto half_width = [&](const loc_candidate &q) { return q.half_width > 0 ? q.half_width : r_default; };
    // pass 1: which candidates read pixels, and each thread's pixel count
    run([&](int t) {
        int lo, hi;
        long long k = 0, px = 0;
        chunk(t, lo, hi);
        for (int i = lo; i < hi; ++i) {
            const loc_candidate &q = c[i];
            const bool finite = std::isfinite(q.x) && std::isfinite(q.y) && std::isfinite(q.intensity) &&
                                std::isfinite(q.background);
            const int r = half_width(q);
            int o = -1;
            if (finite && q.frame >= 0 && q.frame < n_frames && q.half_width >= 0 && r >= 1 && r <= r_cap) {
                const double xo = std::floor(q.x - (double)r), yo = std::floor(q.y - (double)r);
                if (!(xo < 0 || xo + 2 * r > n_rows - 1 || yo < 0 || yo + 2 * r > n_cols - 1)) {
                    o = 0;
                    ++k;
                    px += (long long)(2 * r + 1) * (2 * r + 1);
                }
            }
            off[i] = o;
        }
        cnt[t] = k;
        npx[t] = px;
    });
    std::vector<long long> base(nt, 0);
    long long total = 0, kept = 0;
    for (int t = 0; t < nt; ++t) {
        base[t] = total;
        total += npx[t];
        kept += cnt[t];
    }
    if (kept == 0 || (!force && kept < kRoiMinCands) || total >= (1ll << 31)) return plan;
    const double roi_bytes = (double)total * sizeof(uint16_t);
    const double frame_bytes = (double)n_frames * n_rows * n_cols * sizeof(uint16_t);
    if (!(roi_bytes < (force ? 1.0 : kRoiFraction) * frame_bytes)) return plan;
    if ((*err = roi->ensure((size_t)roi_bytes)) != cudaSuccess) return plan;
    uint16_t *dst0 = (uint16_t *)roi->p;
    const size_t fpx = (size_t)n_rows * n_cols;
    const uint16_t *end = frames + (size_t)n_frames * fpx;
    // the rows of a ROI 16 candidates ahead are requested before the
    // current ROI is copied: every row is a cache miss in another frame row,
    // and the copy is bound by their latency (16 ahead: +20 % over 8 on 16
    // host threads)
    constexpr int kAhead = 16;
    auto roi_src = [&](const loc_candidate &q, int &sd) {
        const int r = half_width(q);
        sd = 2 * r + 1;
        const size_t xo = (size_t)std::floor(q.x - (double)r), yo = (size_t)std::floor(q.y - (double)r);
        return frames + (size_t)q.frame * fpx + xo + yo * (size_t)n_rows;
    };
    // pass 2: offsets in candidate order, rows copied into the stack
    run([&](int t) {
        int lo, hi;
        chunk(t, lo, hi);
        long long at = base[t];
        const long long stop = t + 1 < nt ? base[t + 1] : total;
        // one writer per thread (its line buffer is a few KB: kept off the stack)
        std::unique_ptr<StackWriter> wr(new StackWriter(reinterpret_cast<unsigned char *>(dst0 + at),
                                                        reinterpret_cast<unsigned char *>(dst0 + stop)));
        for (int i = lo; i < hi; ++i) {
            if (i + kAhead < hi && off[i + kAhead] >= 0) {
                int sa;
                const uint16_t *pa = roi_src(c[i + kAhead], sa);
                for (int j = 0; j < sa; ++j) {
                    __builtin_prefetch(pa + (size_t)j * n_rows);
                    __builtin_prefetch(pa + (size_t)j * n_rows + sa - 1);
                }
            }
            if (off[i] < 0) continue;
            int sd;
            const uint16_t *src = roi_src(c[i], sd);
            off[i] = (int)at;
            copy_roi(wr->slot(), src, sd, (size_t)n_rows, end);
            wr->commit((size_t)sd * sd * sizeof(uint16_t));
            at += (long long)sd * sd;
        }
        wr->finish();
    });
    plan.use = true;
    plan.px = total;
    return plan;
}

// the pixel view a fit call reads in ROI mode
struct RoiView {
    const int *off;
    const uint16_t *stack;
    long long px;
};

}  // namespace

struct loc_ctx {
    int device = 0;
    DevBuf scratch;
    // device copies for the host-buffer path
    DevBuf frames, cands, out, flags, roi_slot;
    HostBuf pin_roi, pin_slot;   // ROI-mode staging of loc_fit_host
    unsigned long long h2d_bytes = 0, d2h_bytes = 0;   // copied by host-buffer calls
    unsigned long long *stats_dev = nullptr;  // points into scratch of the last call
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_prop = nullptr;
    bool events_recorded = false;
    bool warm_recorded = false;
    int launches = 0;
    cudaStream_t aux[locb::kMaxAux] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[locb::kMaxAux] = {};
    cudaStream_t aux_long[locb::kMaxAux] = {};
    cudaEvent_t flagged[locb::kMaxAux] = {};
    cudaEvent_t join_long[locb::kMaxAux] = {};
    // launch shapes picked by loc_autotune, per method code; applied where
    // a call leaves the corresponding option at 0
    struct Shape {
        bool set = false;
        int tpf = 1, tail_tpf = 8, budget = 32, rerun_tpf = 2, long_tpf = 8, tpb = 128;
    } tuned[8];
    // loc_fit_host_async: two device slots used in turn, and one stream each
    // for uploads, fits and downloads, so that a call's upload runs while the
    // previous call fits and its download while the next call fits
    struct HostSlot {
        DevBuf frames, cands, out, flags, roi_slot;
        HostBuf pin_roi, pin_slot;   // ROI-mode staging
        cudaEvent_t in_done = nullptr, fit_done = nullptr, out_done = nullptr;
    } slot[2];
    int next_slot = 0;
    cudaStream_t s_in = nullptr, s_fit = nullptr, s_out = nullptr;
};

extern "C" {

LOC_API const char *loc_last_error(void) { return g_err_fixed_latest ? g_err_fixed : g_err.c_str(); }

LOC_API void loc_default_options(loc_options *opt)
{
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->max_iter = 200;   // Localization.cpp:155
    opt->epsabs = 1e-4;    // Localization.cpp:154
    opt->epsrel = 1e-4;
    opt->precision = LOC_PRECISION_FP32;
    opt->pivot_threshold = 0.0f;
    opt->threads_per_block = 0;
    opt->blocks_per_sm = 0;
    opt->stage_u16 = -1;
    opt->max_half_width = 0;
}

LOC_API int loc_reference_columns(int method)
{
    if (!method_ok(method)) return fail(LOC_E_UNSUPPORTED, "unsupported method code");
    return method == 0 ? 12 : method == 1 ? 10 : method == 6 ? 8 : 16;
}

LOC_API int loc_output_columns(int method)
{
    int c = loc_reference_columns(method);
    return c < 0 ? c : c + 2;
}

LOC_API int loc_parameter_count(int method)
{
    if (!method_ok(method)) return fail(LOC_E_UNSUPPORTED, "unsupported method code");
    return method == 0 || method == 6 ? 5 : method == 1 ? 4 : 7;
}

LOC_API int loc_ctx_create(loc_ctx **ctx, int device)
{
    if (!ctx) return fail(LOC_E_INVALID, "ctx is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(LOC_E_INVALID, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    loc_ctx *c = new (std::nothrow) loc_ctx();
    if (!c) return fail(LOC_E_NOMEM, "context allocation failed");
    c->device = device;
    for (int k = 0; k < 4; ++k) {
        if ((e = cudaEventCreate(&c->ev[k])) != cudaSuccess) {
            delete c;
            return cuda_fail(e, "cudaEventCreate");
        }
    }
    if ((e = cudaEventCreate(&c->ev_prop)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
    if ((e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)) != cudaSuccess)
        return cuda_fail(e, "cudaEventCreate");
    for (int k = 0; k < locb::kMaxAux; ++k) {
        if ((e = cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&c->join[k], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&c->aux_long[k], cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&c->flagged[k], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&c->join_long[k], cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "auxiliary stream");
    }
    *ctx = c;
    return LOC_OK;
}

LOC_API int loc_ctx_destroy(loc_ctx *ctx)
{
    if (!ctx) return LOC_OK;
    cudaSetDevice(ctx->device);
    ctx->scratch.release();
    ctx->frames.release();
    ctx->cands.release();
    ctx->out.release();
    ctx->flags.release();
    ctx->roi_slot.release();
    for (int k = 0; k < 4; ++k)
        if (ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
    if (ctx->ev_prop) cudaEventDestroy(ctx->ev_prop);
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    for (int k = 0; k < locb::kMaxAux; ++k) {
        if (ctx->aux[k]) cudaStreamDestroy(ctx->aux[k]);
        if (ctx->join[k]) cudaEventDestroy(ctx->join[k]);
        if (ctx->aux_long[k]) cudaStreamDestroy(ctx->aux_long[k]);
        if (ctx->flagged[k]) cudaEventDestroy(ctx->flagged[k]);
        if (ctx->join_long[k]) cudaEventDestroy(ctx->join_long[k]);
    }
    for (cudaStream_t s : {ctx->s_in, ctx->s_fit, ctx->s_out})
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    for (auto &sl : ctx->slot) {
        sl.frames.release();
        sl.cands.release();
        sl.out.release();
        sl.flags.release();
        sl.roi_slot.release();
        sl.pin_roi.release();
        sl.pin_slot.release();
        for (cudaEvent_t ev : {sl.in_done, sl.fit_done, sl.out_done})
            if (ev) cudaEventDestroy(ev);
    }
    ctx->pin_roi.release();
    ctx->pin_slot.release();
    delete ctx;
    return LOC_OK;
}

static int validate(const loc_ctx *ctx, const void *frames, int n_frames, int n_rows, int n_cols,
                    const void *cands, int n_cands, int method, double w0, double sigma, const void *out,
                    const void *flags)
{
    if (!ctx) return fail(LOC_E_INVALID, "ctx is NULL");
    if (!method_ok(method)) return fail(LOC_E_UNSUPPORTED, "unsupported method code");
    if (n_cands < 0) return fail(LOC_E_INVALID, "n_cands < 0");
    if (n_cands > 0 && (!cands || !out || !flags)) return fail(LOC_E_INVALID, "NULL buffer");
    if (n_frames < 0 || n_rows <= 0 || n_cols <= 0) return fail(LOC_E_INVALID, "bad frame stack shape");
    if (n_frames > 0 && !frames) return fail(LOC_E_INVALID, "frames is NULL");
    if (!(w0 > 0) || !std::isfinite(w0)) return fail(LOC_E_INVALID, "w0 must be finite and > 0");
    if (!(sigma != 0) || !std::isfinite(sigma)) return fail(LOC_E_INVALID, "sigma must be finite and non-zero");
    return LOC_OK;
}

namespace {

bool roi_mode_allowed(int method, const loc_options &o)
{
    // the proposal cuts its windows from whole frames; MLEwG has its own kernel
    return method != LOC_METHOD_MLEWG && o.proposal == nullptr && o.host_roi_mode >= 0;
}

// loc_fit_batch, or with roi set a host call's ROI-mode fit (d_frames then
// the slot stack; n_frames, n_rows and n_cols the original stack's shape)
int fit_impl(loc_ctx *ctx, const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
             const loc_candidate *d_cands, int n_cands, int method, double w0, double sigma, const loc_options *opt,
             double *d_out, uint8_t *d_flags, void *stream, const RoiView *roi)
{
    int rc = validate(ctx, d_frames, n_frames, n_rows, n_cols, d_cands, n_cands, method, w0, sigma, d_out, d_flags);
    if (rc) return rc;
    loc_options o;
    if (opt) o = *opt;
    else loc_default_options(&o);
    if (o.max_iter < 1) return fail(LOC_E_INVALID, "max_iter < 1");
    if (!(o.epsrel >= 0) || !(o.epsabs >= 0)) return fail(LOC_E_INVALID, "negative tolerance");
    const loc_ctx::Shape &tu = ctx->tuned[method];
    if (tu.set) {
        if (o.threads_per_fit == 0) o.threads_per_fit = tu.tpf;
        if (o.tail_threads_per_fit == 0) o.tail_threads_per_fit = tu.tail_tpf;
        if (o.level0_budget == 0) o.level0_budget = tu.budget;
        if (o.rerun_threads_per_fit == 0) o.rerun_threads_per_fit = tu.rerun_tpf;
        if (o.long_rerun_threads_per_fit == 0) o.long_rerun_threads_per_fit = tu.long_tpf;
        if (o.threads_per_block == 0) o.threads_per_block = tu.tpb;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    const int rerun = o.fp64_rerun >= 0 ? 1 : 0;
    locb::ProposalView prop{};
    const bool warm = o.proposal != nullptr;
    if (warm) {
        locb::proposal_view(o.proposal, &prop);
        if (prop.nout != locb::proposal_nout(method))
            return fail(LOC_E_INVALID, "the proposal network was built for another method");
        if (prop.device != ctx->device) return fail(LOC_E_INVALID, "the proposal network lives on another device");
        if (o.precision == LOC_PRECISION_FP64) return fail(LOC_E_UNSUPPORTED, "start proposals run with FP32 solves");
    }
    const size_t need = locb::scratch_bytes(method, n_cands, o.precision, rerun, warm ? 1 : 0);
    e = ctx->scratch.ensure(need);
    if (e != cudaSuccess) return fail(LOC_E_NOMEM, std::string("scratch allocation: ") + cudaGetErrorString(e));
    locb::Scratch s;
    locb::carve_scratch(ctx->scratch.p, method, n_cands, o.precision, rerun, &s, warm ? 1 : 0);
    if (roi && (warm || method == LOC_METHOD_MLEWG))
        return fail(LOC_E_UNSUPPORTED, "ROI mode: no start proposal and no MLEwG");
    locb::FitParams p{};
    p.frames = d_frames;
    p.n_frames = n_frames;
    p.n_rows = n_rows;
    p.n_cols = n_cols;
    p.cands = d_cands;
    p.n_cands = n_cands;
    if (roi) {
        p.roi_slot = roi->off;
        p.roi_stack = roi->stack;
        p.roi_px = roi->px;
    }
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
    p.threads_per_fit = o.threads_per_fit > 0 ? o.threads_per_fit : (o.compensated > 0 ? 4 : 1);
    if (o.compensated > 0 && p.threads_per_fit < 4) p.threads_per_fit = 4;
    p.tail_threads_per_fit = o.tail_threads_per_fit > 0 ? o.tail_threads_per_fit : 8;
    p.level0_budget = o.level0_budget == 0 ? 32 : (o.level0_budget < 0 ? 0 : o.level0_budget);
    p.fp64_rerun = rerun;
    p.rerun_threads_per_fit = (o.rerun_threads_per_fit == 1 || o.rerun_threads_per_fit == 4 ||
                               o.rerun_threads_per_fit == 8) ? o.rerun_threads_per_fit : 2;
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
    p.long_rerun_threads_per_fit = o.long_rerun_threads_per_fit > 0 ? o.long_rerun_threads_per_fit : 8;
    p.long_rerun_iters = o.long_rerun_iters == 0 ? (p.level0_budget > 0 ? p.level0_budget : 32)
                                                 : (o.long_rerun_iters < 0 ? 0 : o.long_rerun_iters);
    if (!(p.long_rerun_threads_per_fit == 1 || p.long_rerun_threads_per_fit == 2 ||
          p.long_rerun_threads_per_fit == 4 || p.long_rerun_threads_per_fit == 8))
        return fail(LOC_E_INVALID, "long_rerun_threads_per_fit must be 1, 2, 4 or 8");
    if (!(p.threads_per_fit == 1 || p.threads_per_fit == 4 || p.threads_per_fit == 8 || p.threads_per_fit == 16) ||
        !(p.tail_threads_per_fit == 1 || p.tail_threads_per_fit == 4 || p.tail_threads_per_fit == 8))
        return fail(LOC_E_INVALID, "threads per fit must be 1, 4, 8 or 16 (second level: 1, 4 or 8)");
    p.init_params = o.d_init_params;
    p.warm = warm;
    p.prop = prop;
    p.warm_iter_limit = o.warm_iter_limit == 0 ? 8 : (o.warm_iter_limit < 0 ? 0 : o.warm_iter_limit);
    ctx->launches = 0;
    p.launches = &ctx->launches;
    p.params_out = o.d_params_out;
    p.diag = o.d_diag;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing((cudaStream_t)stream, &cap);
    for (int k = 0; k < 4; ++k) p.ev[k] = cap == cudaStreamCaptureStatusNone ? ctx->ev[k] : nullptr;
    ctx->events_recorded = cap == cudaStreamCaptureStatusNone;
    p.ev_prop = warm && cap == cudaStreamCaptureStatusNone ? ctx->ev_prop : nullptr;
    ctx->warm_recorded = p.ev_prop != nullptr;
    for (int k = 0; k < locb::kMaxAux; ++k) {
        p.aux[k] = o.serial_classes ? nullptr : ctx->aux[k];
        p.join[k] = ctx->join[k];
        p.aux_long[k] = o.serial_classes ? nullptr : ctx->aux_long[k];
        p.flagged[k] = ctx->flagged[k];
        p.join_long[k] = ctx->join_long[k];
    }
    p.fork = ctx->fork;
    p.out = d_out;
    p.flags = d_flags;
    int detail = 0;
    e = locb::enqueue_fit(p, s, (cudaStream_t)stream, &detail);
    ctx->stats_dev = s.stats;
    if (e != cudaSuccess) {
        if (detail == 1) return fail(LOC_E_UNSUPPORTED, "ROI too large for shared memory");
        return cuda_fail(e, "fit launch");
    }
    return LOC_OK;
}

}  // namespace

LOC_API int loc_fit_batch(loc_ctx *ctx, const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                          const loc_candidate *d_cands, int n_cands, int method, double w0, double sigma,
                          const loc_options *opt, double *d_out, uint8_t *d_flags, void *stream)
{
    return fit_impl(ctx, d_frames, n_frames, n_rows, n_cols, d_cands, n_cands, method, w0, sigma, opt, d_out, d_flags,
                    stream, nullptr);
}

namespace {

// Device buffer owned by one loc_autotune call.
struct TuneBuf {
    void *p = nullptr;
    ~TuneBuf() { if (p) cudaFree(p); }
};

// Rows of a trial shape against the default shape's: reject codes and
// positions (x, y columns) of the fits both keep. A shape is admissible when
// at most one fit in 10^4 (at least one) changes its reject code and at most
// as many kept positions move by 1e-3 px or more.
bool same_results(const std::vector<double> &a, const std::vector<uint8_t> &fa, const std::vector<double> &b,
                  const std::vector<uint8_t> &fb, int ncol, int xcol, long *n_flag, long *n_pos)
{
    const size_t n = fa.size();
    long df = 0, dp = 0;
    for (size_t i = 0; i < n; ++i) {
        if ((fa[i] == 0) != (fb[i] == 0)) {
            ++df;
            continue;
        }
        if (fa[i] != 0) continue;
        const double dx = std::fabs(a[i * ncol + xcol] - b[i * ncol + xcol]);
        const double dy = std::fabs(a[i * ncol + xcol + 1] - b[i * ncol + xcol + 1]);
        if (!(dx < 1e-3 && dy < 1e-3)) ++dp;
    }
    *n_flag = df;
    *n_pos = dp;
    const long lim = std::max<long>(1, (long)(n / 10000));
    return df <= lim && dp <= lim;
}

}  // namespace

LOC_API int loc_autotune(loc_ctx *ctx, const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                         const loc_candidate *d_cands, int n_cands, int method, double w0, double sigma,
                         const loc_options *base, loc_tuning *result, void *stream)
{
    int dummy = 0;
    int rc = validate(ctx, d_frames, n_frames, n_rows, n_cols, d_cands, n_cands, method, w0, sigma, &dummy, &dummy);
    if (rc) return rc;
    if (method == LOC_METHOD_MLEWG) return fail(LOC_E_UNSUPPORTED, "MLEwG has no launch shape to tune");
    if (n_cands < 1) return fail(LOC_E_INVALID, "the tuning sample is empty");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    const cudaStream_t st = (cudaStream_t)stream;
    loc_options b;
    if (base) b = *base;
    else loc_default_options(&b);
    if (b.precision == LOC_PRECISION_FP64) return fail(LOC_E_UNSUPPORTED, "the tuner times the FP32 solver");
    const int ncol = loc_output_columns(method);
    const int xcol = method == 0 ? 3 : method == 1 ? 2 : 4;
    TuneBuf out, flg;
    if ((e = cudaMalloc(&out.p, sizeof(double) * (size_t)n_cands * ncol)) != cudaSuccess ||
        (e = cudaMalloc(&flg.p, (size_t)n_cands)) != cudaSuccess)
        return fail(LOC_E_NOMEM, std::string("tuning buffers: ") + cudaGetErrorString(e));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if ((e = cudaEventCreate(&t0)) != cudaSuccess || (e = cudaEventCreate(&t1)) != cudaSuccess) {
        if (t0) cudaEventDestroy(t0);
        return cuda_fail(e, "tuning events");
    }
    ctx->tuned[method].set = false;   // zeros mean the built-in defaults while tuning
    std::vector<double> rows_ref((size_t)n_cands * ncol), rows((size_t)n_cands * ncol);
    std::vector<uint8_t> flags_ref(n_cands), flags(n_cands);
    int trials = 0;
    // median device time of three calls after one untimed call; rows, flags
    // and the number of fits the FP32 solver finished in the last call copied
    // to the host (a shape must finish every fit: the rows alone could come
    // from solver state an earlier call left in the scratch)
    auto time_shape = [&](const loc_ctx::Shape &sh, float *ms, std::vector<double> &r,
                          std::vector<uint8_t> &f, unsigned long long *fits) -> int {
        loc_options o = b;
        o.threads_per_fit = sh.tpf;
        o.tail_threads_per_fit = sh.tail_tpf;
        o.level0_budget = sh.budget;
        o.rerun_threads_per_fit = sh.rerun_tpf;
        o.long_rerun_threads_per_fit = sh.long_tpf;
        o.threads_per_block = sh.tpb;
        float t[3];
        for (int k = 0; k < 4; ++k) {
            if (k > 0) cudaEventRecord(t0, st);
            int r2 = loc_fit_batch(ctx, d_frames, n_frames, n_rows, n_cols, d_cands, n_cands, method, w0, sigma, &o,
                                   (double *)out.p, (uint8_t *)flg.p, stream);
            if (r2) return r2;
            if (k > 0) {
                cudaEventRecord(t1, st);
                cudaError_t e2 = cudaEventSynchronize(t1);
                if (e2 != cudaSuccess) return cuda_fail(e2, "tuning run");
                cudaEventElapsedTime(&t[k - 1], t0, t1);
            }
        }
        std::sort(t, t + 3);
        *ms = t[1];
        ++trials;
        cudaError_t e2 = cudaMemcpy(r.data(), out.p, sizeof(double) * r.size(), cudaMemcpyDeviceToHost);
        if (e2 == cudaSuccess) e2 = cudaMemcpy(f.data(), flg.p, f.size(), cudaMemcpyDeviceToHost);
        if (e2 == cudaSuccess) e2 = cudaMemcpy(fits, ctx->stats_dev + 4, sizeof(*fits), cudaMemcpyDeviceToHost);
        if (e2 != cudaSuccess) return cuda_fail(e2, "tuning rows");
        return LOC_OK;
    };
    loc_ctx::Shape best;   // the built-in defaults
    float best_ms = 0.0f;
    long worst_flag = 0, worst_pos = 0;
    unsigned long long fits_ref = 0, fits = 0;
    rc = time_shape(best, &best_ms, rows_ref, flags_ref, &fits_ref);
    const float ms_default = best_ms;
    // coordinate descent: each knob in turn over its values, the others held
    // at the best shape so far; a value must be 1 % faster and give the
    // default shape's results
    const std::vector<std::pair<int loc_ctx::Shape::*, std::vector<int>>> knobs = {
        {&loc_ctx::Shape::tpb, {128, 96, 64}},
        {&loc_ctx::Shape::tpf, {1, 4, 8, 16}},
        {&loc_ctx::Shape::budget, {16, 24, 32, 48, 64}},
        {&loc_ctx::Shape::tail_tpf, {8, 4}},
        {&loc_ctx::Shape::rerun_tpf, {2, 1, 4, 8}},
        {&loc_ctx::Shape::long_tpf, {8, 4, 2}},
    };
    for (size_t kk = 0; rc == LOC_OK && kk < knobs.size(); ++kk) {
        const auto &kn = knobs[kk];
        for (int v : kn.second) {
            if (rc != LOC_OK || best.*(kn.first) == v) continue;
            loc_ctx::Shape trial = best;
            trial.*(kn.first) = v;
            float ms = 0.0f;
            rc = time_shape(trial, &ms, rows, flags, &fits);
            if (rc != LOC_OK) break;
            long nf = 0, np = 0;
            const bool same = fits == fits_ref && same_results(rows, flags, rows_ref, flags_ref, ncol, xcol, &nf, &np);
            if (same && ms < 0.99f * best_ms) {
                best = trial;
                best_ms = ms;
                worst_flag = std::max(worst_flag, nf);
                worst_pos = std::max(worst_pos, np);
            }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != LOC_OK) return rc;
    best.set = true;
    ctx->tuned[method] = best;
    if (result) {
        result->threads_per_fit = best.tpf;
        result->tail_threads_per_fit = best.tail_tpf;
        result->level0_budget = best.budget;
        result->rerun_threads_per_fit = best.rerun_tpf;
        result->long_rerun_threads_per_fit = best.long_tpf;
        result->threads_per_block = best.tpb;
        result->ms_default = ms_default;
        result->ms_tuned = best_ms;
        result->trials = trials;
        result->flag_changes = (int32_t)worst_flag;
        result->position_changes = (int32_t)worst_pos;
    }
    return LOC_OK;
}

LOC_API int loc_sync(loc_ctx *ctx, void *stream)
{
    if (!ctx) return fail(LOC_E_INVALID, "ctx is NULL");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
    return LOC_OK;
}

LOC_API int loc_last_stats(loc_ctx *ctx, loc_stats *st)
{
    if (!ctx || !st) return fail(LOC_E_INVALID, "NULL argument");
    if (!ctx->stats_dev) {
        std::memset(st, 0, sizeof(*st));
        return LOC_OK;
    }
    unsigned long long v[locb::kStatWords];
    cudaError_t e = cudaMemcpy(v, ctx->stats_dev, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "stats copy");
    st->f_evals = v[0];
    st->jacobian_evals = v[1];
    st->lambda_solves = v[2];
    st->fp64_escalations = v[3];
    st->fits = v[4];
    st->iterations = v[5];
    st->pixels_f = v[6];
    st->pixels_j = v[7];
    st->kcycles_refill = v[8];
    st->kcycles_step = v[9];
    st->kcycles_pass = v[10];
    st->kcycles_decide = v[11];
    st->fits_fp64_rerun = v[12 + 4];
    st->iterations_fp64_rerun = v[12 + 5];
    st->kcycles_fp64_rerun = v[12 + 8] + v[12 + 9] + v[12 + 10] + v[12 + 11];
    st->kcycles_fp64_rerun_pass = v[12 + 10];
    st->fits_warm = v[2 * 12];
    st->kernel_launches = ctx->launches;
    st->queue_ms = st->solver_ms = st->finalize_ms = st->proposal_ms = -1.0f;
    if (ctx->events_recorded && cudaEventSynchronize(ctx->ev[3]) == cudaSuccess) {
        cudaEventElapsedTime(&st->queue_ms, ctx->ev[0], ctx->ev[1]);
        if (ctx->warm_recorded) {
            cudaEventElapsedTime(&st->proposal_ms, ctx->ev[1], ctx->ev_prop);
            cudaEventElapsedTime(&st->solver_ms, ctx->ev_prop, ctx->ev[2]);
        } else {
            cudaEventElapsedTime(&st->solver_ms, ctx->ev[1], ctx->ev[2]);
        }
        cudaEventElapsedTime(&st->finalize_ms, ctx->ev[2], ctx->ev[3]);
    }
    return LOC_OK;
}

LOC_API int loc_fit_host(loc_ctx *ctx, const uint16_t *frames, int n_frames, int n_rows, int n_cols,
                         const loc_candidate *cands, int n_cands, int method, double w0, double sigma,
                         const loc_options *opt, double *out, uint8_t *flags)
{
    int rc = validate(ctx, frames, n_frames, n_rows, n_cols, cands, n_cands, method, w0, sigma, out, flags);
    if (rc) return rc;
    // asynchronous calls still in flight share the context's scratch
    if ((rc = loc_fit_host_wait(ctx)) != LOC_OK) return rc;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    loc_options o;
    if (opt) o = *opt;
    else loc_default_options(&o);
    const size_t cbytes = (size_t)n_cands * sizeof(loc_candidate);
    const int ncol = loc_output_columns(method);
    const size_t obytes = (size_t)n_cands * ncol * sizeof(double);
    // ROI mode when the candidates' ROIs are a small part of the frames
    RoiPlan plan;
    if (roi_mode_allowed(method, o) && n_cands > 0) {
        if ((e = ctx->pin_slot.ensure(sizeof(int) * (size_t)n_cands)) != cudaSuccess)
            return fail(LOC_E_NOMEM, std::string("ROI staging: ") + cudaGetErrorString(e));
        plan = plan_and_gather_rois(frames, n_frames, n_rows, n_cols, cands, n_cands, w0, o.max_half_width,
                                    o.host_roi_mode > 0, (int *)ctx->pin_slot.p, &ctx->pin_roi, &e);
        if (e != cudaSuccess) return fail(LOC_E_NOMEM, std::string("ROI staging: ") + cudaGetErrorString(e));
    }
    const size_t fbytes = plan.use ? (size_t)plan.px * sizeof(uint16_t)
                                   : (size_t)n_frames * n_rows * n_cols * sizeof(uint16_t);
    const size_t sbytes = plan.use ? sizeof(int) * (size_t)n_cands : 0;
    if ((e = ctx->frames.ensure(fbytes ? fbytes : 1)) != cudaSuccess ||
        (e = ctx->cands.ensure(cbytes ? cbytes : 1)) != cudaSuccess ||
        (e = ctx->out.ensure(obytes ? obytes : 1)) != cudaSuccess ||
        (e = ctx->flags.ensure(n_cands ? n_cands : 1)) != cudaSuccess ||
        (e = ctx->roi_slot.ensure(sbytes ? sbytes : 1)) != cudaSuccess)
        return fail(LOC_E_NOMEM, std::string("device buffers: ") + cudaGetErrorString(e));
    cudaStream_t st = 0;
    const void *fsrc = plan.use ? ctx->pin_roi.p : (const void *)frames;
    if (fbytes && (e = cudaMemcpyAsync(ctx->frames.p, fsrc, fbytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "frames upload");
    if (cbytes && (e = cudaMemcpyAsync(ctx->cands.p, cands, cbytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "candidates upload");
    if (sbytes &&
        (e = cudaMemcpyAsync(ctx->roi_slot.p, ctx->pin_slot.p, sbytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "ROI slots upload");
    ctx->h2d_bytes += fbytes + cbytes + sbytes;
    ctx->d2h_bytes += obytes + (size_t)n_cands;
    const RoiView view{(const int *)ctx->roi_slot.p, (const uint16_t *)ctx->frames.p, plan.px};
    rc = fit_impl(ctx, (const uint16_t *)ctx->frames.p, n_frames, n_rows, n_cols, (const loc_candidate *)ctx->cands.p,
                  n_cands, method, w0, sigma, opt, (double *)ctx->out.p, (uint8_t *)ctx->flags.p, st,
                  plan.use ? &view : nullptr);
    if (rc) return rc;
    if (obytes && (e = cudaMemcpyAsync(out, ctx->out.p, obytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "rows download");
    if (n_cands && (e = cudaMemcpyAsync(flags, ctx->flags.p, n_cands, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "flags download");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "fit");
    return LOC_OK;
}

LOC_API int loc_fit_host_async(loc_ctx *ctx, const uint16_t *frames, int n_frames, int n_rows, int n_cols,
                               const loc_candidate *cands, int n_cands, int method, double w0, double sigma,
                               const loc_options *opt, double *out, uint8_t *flags)
{
    int rc = validate(ctx, frames, n_frames, n_rows, n_cols, cands, n_cands, method, w0, sigma, out, flags);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    if (!ctx->s_in) {
        for (cudaStream_t *s : {&ctx->s_in, &ctx->s_fit, &ctx->s_out})
            if ((e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e, "stream");
        for (auto &sl : ctx->slot)
            for (cudaEvent_t *ev : {&sl.in_done, &sl.fit_done, &sl.out_done})
                if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess)
                    return cuda_fail(e, "event");
    }
    loc_ctx::HostSlot &sl = ctx->slot[ctx->next_slot];
    const size_t cbytes = (size_t)n_cands * sizeof(loc_candidate);
    const int ncol = loc_output_columns(method);
    const size_t obytes = (size_t)n_cands * ncol * sizeof(double);
    loc_options o;
    if (opt) o = *opt;
    else loc_default_options(&o);
    // ROI mode: the slot's staging buffers are refilled once its previous
    // upload has left them (the gather runs while earlier calls fit)
    RoiPlan plan;
    if (roi_mode_allowed(method, o) && n_cands > 0) {
        if ((e = cudaEventSynchronize(sl.in_done)) != cudaSuccess) return cuda_fail(e, "staging wait");
        if ((e = sl.pin_slot.ensure(sizeof(int) * (size_t)n_cands)) != cudaSuccess)
            return fail(LOC_E_NOMEM, std::string("ROI staging: ") + cudaGetErrorString(e));
        plan = plan_and_gather_rois(frames, n_frames, n_rows, n_cols, cands, n_cands, w0, o.max_half_width,
                                    o.host_roi_mode > 0, (int *)sl.pin_slot.p, &sl.pin_roi, &e);
        if (e != cudaSuccess) return fail(LOC_E_NOMEM, std::string("ROI staging: ") + cudaGetErrorString(e));
    }
    const size_t fbytes = plan.use ? (size_t)plan.px * sizeof(uint16_t)
                                   : (size_t)n_frames * n_rows * n_cols * sizeof(uint16_t);
    const size_t sbytes = plan.use ? sizeof(int) * (size_t)n_cands : 0;
    const size_t need = locb::scratch_bytes(method, n_cands, o.precision, o.fp64_rerun >= 0 ? 1 : 0,
                                            o.proposal ? 1 : 0);
    if (sl.frames.cap < fbytes || sl.cands.cap < cbytes || sl.out.cap < obytes || sl.flags.cap < (size_t)n_cands ||
        sl.roi_slot.cap < sbytes || ctx->scratch.cap < need) {
        // a buffer grows: the calls in flight may still use the old one
        if ((rc = loc_fit_host_wait(ctx)) != LOC_OK) return rc;
        if ((e = sl.frames.ensure(fbytes ? fbytes : 1)) != cudaSuccess ||
            (e = sl.cands.ensure(cbytes ? cbytes : 1)) != cudaSuccess ||
            (e = sl.out.ensure(obytes ? obytes : 1)) != cudaSuccess ||
            (e = sl.flags.ensure(n_cands ? n_cands : 1)) != cudaSuccess ||
            (e = sl.roi_slot.ensure(sbytes ? sbytes : 1)) != cudaSuccess)
            return fail(LOC_E_NOMEM, std::string("device buffers: ") + cudaGetErrorString(e));
    }
    // this slot's previous fit has read its frames and candidates
    if ((e = cudaStreamWaitEvent(ctx->s_in, sl.fit_done, 0)) != cudaSuccess) return cuda_fail(e, "stream wait");
    const void *fsrc = plan.use ? sl.pin_roi.p : (const void *)frames;
    if (fbytes && (e = cudaMemcpyAsync(sl.frames.p, fsrc, fbytes, cudaMemcpyHostToDevice, ctx->s_in)) != cudaSuccess)
        return cuda_fail(e, "frames upload");
    if (cbytes && (e = cudaMemcpyAsync(sl.cands.p, cands, cbytes, cudaMemcpyHostToDevice, ctx->s_in)) != cudaSuccess)
        return cuda_fail(e, "candidates upload");
    if (sbytes && (e = cudaMemcpyAsync(sl.roi_slot.p, sl.pin_slot.p, sbytes, cudaMemcpyHostToDevice, ctx->s_in)) !=
                      cudaSuccess)
        return cuda_fail(e, "ROI slots upload");
    if ((e = cudaEventRecord(sl.in_done, ctx->s_in)) != cudaSuccess) return cuda_fail(e, "event record");
    ctx->h2d_bytes += fbytes + cbytes + sbytes;
    ctx->d2h_bytes += obytes + (size_t)n_cands;
    // the fit waits for its upload and for the download of this slot's previous rows
    if ((e = cudaStreamWaitEvent(ctx->s_fit, sl.in_done, 0)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(ctx->s_fit, sl.out_done, 0)) != cudaSuccess)
        return cuda_fail(e, "stream wait");
    const RoiView view{(const int *)sl.roi_slot.p, (const uint16_t *)sl.frames.p, plan.px};
    if (n_cands > 0)
        rc = fit_impl(ctx, (const uint16_t *)sl.frames.p, n_frames, n_rows, n_cols, (const loc_candidate *)sl.cands.p,
                      n_cands, method, w0, sigma, opt, (double *)sl.out.p, (uint8_t *)sl.flags.p, ctx->s_fit,
                      plan.use ? &view : nullptr);
    if ((e = cudaEventRecord(sl.fit_done, ctx->s_fit)) != cudaSuccess) return cuda_fail(e, "event record");
    if (rc) return rc;
    if ((e = cudaStreamWaitEvent(ctx->s_out, sl.fit_done, 0)) != cudaSuccess) return cuda_fail(e, "stream wait");
    if (obytes && (e = cudaMemcpyAsync(out, sl.out.p, obytes, cudaMemcpyDeviceToHost, ctx->s_out)) != cudaSuccess)
        return cuda_fail(e, "rows download");
    if (n_cands && (e = cudaMemcpyAsync(flags, sl.flags.p, n_cands, cudaMemcpyDeviceToHost, ctx->s_out)) != cudaSuccess)
        return cuda_fail(e, "flags download");
    if ((e = cudaEventRecord(sl.out_done, ctx->s_out)) != cudaSuccess) return cuda_fail(e, "event record");
    ctx->next_slot ^= 1;
    return LOC_OK;
}

LOC_API int loc_host_bytes(const loc_ctx *ctx, uint64_t *h2d, uint64_t *d2h)
{
    if (!ctx) return fail(LOC_E_INVALID, "ctx is NULL");
    if (h2d) *h2d = ctx->h2d_bytes;
    if (d2h) *d2h = ctx->d2h_bytes;
    return LOC_OK;
}

LOC_API int loc_fit_host_wait(loc_ctx *ctx)
{
    if (!ctx) return fail(LOC_E_INVALID, "ctx is NULL");
    if (!ctx->s_in) return LOC_OK;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    for (cudaStream_t s : {ctx->s_in, ctx->s_fit, ctx->s_out})
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "host fit");
    return LOC_OK;
}

LOC_API int loc_compact_host(const double *out, const uint8_t *flags, int n_cands, int method, double *matrix,
                             int max_rows)
{
    const int rcols = loc_reference_columns(method);
    if (rcols < 0) return rcols;
    if (n_cands < 0 || (n_cands > 0 && (!out || !flags))) return fail(LOC_E_INVALID, "bad arguments");
    const int ncol = rcols + 2;
    int kept = 0;
    for (int i = 0; i < n_cands; ++i) kept += flags[i] == LOC_FLAG_KEPT;
    if (kept > max_rows || !matrix) return kept;
    int row = 0;
    for (int i = 0; i < n_cands; ++i) {
        if (flags[i] != LOC_FLAG_KEPT) continue;
        for (int c = 0; c < rcols; ++c) matrix[(size_t)c * kept + row] = out[(size_t)i * ncol + c];
        ++row;
    }
    return kept;
}

}  // extern "C"

// Record an error message without allocating (used by loc_fit_batch_static).
namespace locb {
int record_error_fixed(int code, const char *msg)
{
    std::snprintf(g_err_fixed, sizeof(g_err_fixed), "%s", msg);
    g_err_fixed_latest = true;
    return code;
}
}  // namespace locb

// ---- reference DLL compatibility (LocalizerDLL.h:53-56) ----

namespace {
std::mutex g_compat_mu;
loc_ctx *g_compat_ctx = nullptr;
}  // namespace

extern "C" {

LOC_API int LocalizerFitEmitters(unsigned short *imageData, int nRows, int nCols, int nImages, double psfWidth,
                                 double glrtInsensitivity, int *nEmitters, double **emitterCoordinates)
{
    try {
        if (!imageData || !nEmitters || !emitterCoordinates || nRows <= 0 || nCols <= 0 || nImages < 0) return -1;
        std::lock_guard<std::mutex> lk(g_compat_mu);
        if (!g_compat_ctx) {
            int dev = 0;
            cudaGetDevice(&dev);
            if (loc_ctx_create(&g_compat_ctx, dev) != LOC_OK) return -1;
        }
        // candidates: GLRT (PFA = glrtInsensitivity, width = psfWidth) + adjacent-8, as LocalizerDLL.cpp:99-103
        long cap = 1 << 16;
        std::vector<loc_candidate> cands;
        long n = 0;
        for (;;) {
            cands.resize((size_t)cap);
            n = loc_find_candidates_host(imageData, nImages, nRows, nCols, glrtInsensitivity, psfWidth, 0,
                                         cands.data(), cap);
            if (n < 0) return -1;
            if (n <= cap) break;
            cap = n;
        }
        cands.resize((size_t)n);
        const int method = LOC_METHOD_2DGAUSS_ELLIPSOIDAL_ASTIGMATISM;  // LocalizerDLL.cpp:107
        const int ncol = loc_output_columns(method);
        std::vector<double> out((size_t)n * ncol);
        std::vector<uint8_t> flags((size_t)n);
        if (n > 0 && loc_fit_host(g_compat_ctx, imageData, nImages, nRows, nCols, cands.data(), (int)n, method,
                                  psfWidth, 1.0, nullptr, out.data(), flags.data()) != LOC_OK)
            return -1;
        int kept = loc_compact_host(out.data(), flags.data(), (int)n, method, nullptr, 0);
        if (kept < 0) return -1;
        double *m = new double[(size_t)kept * 16 + 1];
        loc_compact_host(out.data(), flags.data(), (int)n, method, m, kept);
        *nEmitters = kept;
        *emitterCoordinates = m;
    } catch (...) {
        return -1;
    }
    return 0;
}

LOC_API void LocalizerFree(double *ptrToFree) { delete[] ptrToFree; }

}  // extern "C"
