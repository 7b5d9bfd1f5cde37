// Fit kernels of the B200 localization engine.
//
//   K0 classify / classes / scatter — validate candidates, apply the edge
//      reject of the reference (Localization.cpp:115-124), and build a work
//      queue grouped by ROI half-width (largest first).
//   K1 lm_fit — persistent solver: one thread per fit, a warp refills its
//      idle lanes from the queue with one atomic and stages their ROIs from
//      the HBM-resident uint16 frames with warp-cooperative loads into shared
//      memory; every loop trip is one model/Jacobian/normal-equation pass
//      for all active lanes (see loc_device.cuh).
//   K2 finalize — FP64: covariance (J^T J)^-1, uncertainty scaling, the
//      reference's accept/reject rules and output columns.
#include "loc_device.cuh"
#include "loc_fit.cuh"

#include <math_constants.h>

#include <cmath>
#include <cstdio>

namespace locb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int K = kMaxHalfWidth + 1;
constexpr int M_NCLS = 0, M_MAXR = 1;
// per ROI half-width r: queue start, count, dequeue cursor, histogram, fill cursor
__host__ __device__ constexpr int m_start(int r) { return 8 + 1 * K + r; }
__host__ __device__ constexpr int m_count(int r) { return 8 + 2 * K + r; }
__host__ __device__ constexpr int m_next(int r) { return 8 + 3 * K + r; }
__host__ __device__ constexpr int m_ccount(int r) { return 8 + 6 * K + r; }
__host__ __device__ constexpr int m_cnext(int r) { return 8 + 7 * K + r; }
__host__ __device__ constexpr int m_hist(int r) { return 8 + 4 * K + r; }
__host__ __device__ constexpr int m_fill(int r) { return 8 + 5 * K + r; }

__host__ __device__ constexpr int ref_cols(int method) { return method == 0 ? 12 : method == 1 ? 10 : 16; }

struct K0Args {
    const Cand *cands;
    int n;
    int n_frames, n_rows, n_cols;
    int r_default;
    int r_cap;        // candidates whose r exceeds it are rejected as bad input
    int method;
    int ncol_total;
    double *out;
    uint8_t *flags;
    int *cls;
    int *meta;
    int *cls2;   // optional: FP64 re-run marks, cleared here
    // ROI mode: a candidate that passes the edge rule must have its ROI
    // inside the packed ROI stack (else it is flagged as bad input: the
    // solver never reads outside the stack)
    const int *roi_slot;
    long long roi_px;
};

__device__ void write_reject_row(double *row, int ncol_total, int frame)
{
    row[0] = (double)frame;
    for (int k = 1; k < ncol_total - 2; ++k) row[k] = CUDART_NAN;
    row[ncol_total - 2] = 0.0;
    row[ncol_total - 1] = 0.0;
}

__global__ void k0_classify(K0Args a)
{
    __shared__ int hist[K];
    for (int r = threadIdx.x; r < K; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n) {
        const Cand c = a.cands[i];
        int cls = -1;
        uint8_t flag = F_PENDING;
        const bool finite = isfinite(c.x) && isfinite(c.y) && isfinite(c.intensity) && isfinite(c.background);
        const int r = c.half_width > 0 ? c.half_width : a.r_default;
        if (!finite || c.frame < 0 || c.frame >= a.n_frames || c.half_width < 0 || r < 1 || r > a.r_cap) {
            flag = F_BAD_INPUT;
        } else {
            // Localization.cpp:115-120, integer ROI origin and far corner
            const double xo = floor(c.x - (double)r), yo = floor(c.y - (double)r);
            const double xm = xo + 2 * r, ym = yo + 2 * r;
            if (xo < 0 || xm > a.n_rows - 1 || yo < 0 || ym > a.n_cols - 1) {
                flag = F_EDGE;
            } else if (a.roi_slot && (a.roi_slot[i] < 0 ||
                                      (long long)a.roi_slot[i] + (long long)(2 * r + 1) * (2 * r + 1) > a.roi_px)) {
                flag = F_BAD_INPUT;
            } else {
                cls = r;
                atomicAdd(&hist[r], 1);
            }
        }
        a.cls[i] = cls;
        if (a.cls2) a.cls2[i] = -1;
        a.flags[i] = flag;
        if (flag != F_PENDING) write_reject_row(a.out + (size_t)i * a.ncol_total, a.ncol_total, c.frame);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < K; r += blockDim.x)
        if (hist[r]) atomicAdd(&a.meta[m_hist(r)], hist[r]);
}

// One block: queue layout per half-width, largest ROIs first.
__global__ void k0_classes(int *meta)
{
    if (threadIdx.x != 0) return;
    int ncls = 0, start = 0, maxr = 0;
    for (int r = K - 1; r >= 1; --r) {
        const int cnt = meta[m_hist(r)];
        if (cnt == 0) continue;
        if (r > maxr) maxr = r;
        meta[m_start(r)] = start;
        meta[m_count(r)] = cnt;
        meta[m_next(r)] = 0;
        meta[m_fill(r)] = start;
        start += cnt;
        ++ncls;
    }
    meta[M_NCLS] = ncls;
    meta[M_MAXR] = maxr;
}

__global__ void k0_scatter(const int *cls, int n, int *meta, int *order)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = i < n ? cls[i] : -1;
    const unsigned active = __ballot_sync(kFull, c >= 0);
    if (c < 0) return;
    // warp-aggregated: one atomic per distinct class in the warp
    const unsigned peers = __match_any_sync(active, c);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(&meta[m_fill(c)], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    order[base + __popc(peers & ((1u << lane) - 1))] = i;
}

// Fits of the FP32 solver whose result could depend on its rounding go to an
// FP64 re-run: a branch decision of the trust-region method was within
// `margin` of its threshold, the undamped normal matrix had a pivot ratio
// below `pivot` (ill-conditioned), or the solver stopped for lack of
// progress.
template <int P>
__global__ void k3_flag(const float *state32, int stride, const int *cls, const uint8_t *flags, int n, float margin,
                        float pivot, int *cls2, int *meta2)
{
    using SL = StateLayout<P>;
    __shared__ int hist[K];
    for (int r = threadIdx.x; r < K; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        int c2 = -1;
        if (cls[i] >= 0 && flags[i] == F_PENDING) {
            const float *s = state32 + (size_t)i * stride;
            // fits stopped by the iteration cap are left alone: they have not
            // converged, are almost always rejected, and cost 200 iterations
            const float status = s[SL::STATUS];
            const bool risky = status != (float)T_MAX_ITER &&
                               (s[SL::MARGIN] < margin || s[SL::MINPIV] < pivot || status != 0.0f);
            if (risky) {
                c2 = cls[i];
                atomicAdd(&hist[c2], 1);
            }
        }
        cls2[i] = c2;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < K; r += blockDim.x)
        if (hist[r]) atomicAdd(&meta2[m_hist(r)], hist[r]);
}

// Per-class form of the flag pass: walks the queue of half-width r and
// appends the flagged fits to that class's FP64 queue (order2 / meta2), or,
// when their FP32 solve took more than long_iters iterations and a long
// queue exists (order3 / meta3), to that one: the long fits set the length
// of the re-run, so they get their own launch with more threads per fit.
template <int P>
__global__ void k3_flag_class(const float *state32, int stride, const int *order, const int *meta,
                              const uint8_t *flags, int r, float margin, float pivot, int warm_limit, int *cls2,
                              int *order2, int *meta2, int long_iters, int *order3, int *meta3, int capped,
                              float cond, int iters_min, float skip_rej, float w0)
{
    using SL = StateLayout<P>;
    constexpr int IX = P == 5 ? 2 : P == 4 ? 1 : 3;
    const int start = meta[m_start(r)], count = meta[m_count(r)];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        meta2[m_start(r)] = start;
        if (meta3) meta3[m_start(r)] = start;
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const int i = order[start + t];
        if (flags[i] != F_PENDING) continue;
        const float *s = state32 + (size_t)i * stride;
        const float status = s[SL::STATUS];
        // warm-started fits (warm_limit > 0) that needed many iterations may
        // stop elsewhere than the reference start's trajectory would
        // capped: fits the FP32 solver stopped at the iteration cap are
        // re-run too (the FP64 solve may converge where FP32 did not)
        const bool is_capped = status == (float)T_MAX_ITER;
        // cond > 0: a branch margin is also too small when it is within the
        // FP32 error the fit's conditioning allows (cond * eps32 / smallest
        // undamped pivot ratio)
        const float mthr = cond > 0.0f ? fmaxf(margin, cond * 5.96e-8f / fmaxf(s[SL::MINPIV], 1e-30f)) : margin;
        const bool risky = is_capped ? capped != 0
                                     : (s[SL::MARGIN] < mthr || s[SL::MINPIV] < pivot || status != 0.0f ||
                                        (warm_limit > 0 && s[SL::ITERS] > (float)warm_limit) ||
                                        (iters_min > 0 && s[SL::ITERS] >= (float)iters_min));
        // skip_rej > 0: a fit whose FP32 end point lies clearly inside a reject
        // rule of the finaliser (centre more than skip_rej px outside the ROI,
        // amplitude below zero by more than skip_rej of its start scale, or
        // every width more than the fraction skip_rej outside its accepted
        // range) is not re-run: only its reject code could change
        bool clear_reject = false;
        if (risky && skip_rej > 0.0f) {
            const float side = (float)(2 * r);
            const float x = s[IX], y = s[IX + 1], A = s[0];
            clear_reject = x < -skip_rej || x > side + skip_rej || y < -skip_rej || y > side + skip_rej ||
                           A < -skip_rej * fmaxf(fabsf(s[P - 1]), 1.0f);
            const float lo = 0.4f * w0 * (1.0f - skip_rej), hi = 1.5f * w0 * (1.0f + skip_rej);
            if constexpr (P == 5) {
                const float wd = fabsf(s[1]);
                clear_reject = clear_reject || wd < lo || wd > hi;
            } else if constexpr (P == 7) {
                // axes of the covariance [[sx^2, rho sx sy], [rho sx sy, sy^2]]
                const float sx = fabsf(s[1]), sy = fabsf(s[2]), rho = s[5];
                const float a = sx * sx, c = sy * sy, b = rho * sx * sy;
                const float ht = 0.5f * (a + c), rad = sqrtf(0.25f * (a - c) * (a - c) + b * b);
                const float s1 = sqrtf(fmaxf(ht - rad, 0.0f)), s2 = sqrtf(ht + rad);
                clear_reject = clear_reject || ((s1 < lo || s1 > hi) && (s2 < lo || s2 > hi));
            }
        }
        if (risky && !clear_reject) {
            cls2[i] = r;
            if (meta3 && s[SL::ITERS] > (float)long_iters) {
                const int slot = atomicAdd(&meta3[m_count(r)], 1);
                order3[start + slot] = i;
            } else {
                const int slot = atomicAdd(&meta2[m_count(r)], 1);
                order2[start + slot] = i;
            }
        }
    }
}

struct K1Args {
    const uint16_t *frames;
    long long frame_px;
    int n_rows;
    const Cand *cands;
    const int *order;
    int *meta;
    void *state;
    int state_stride;   // elements of the solver's precision per candidate
    float w0;
    float inv_s2, inv_abs_s;
    double inv_s2_d, inv_abs_s_d;
    int max_iter;
    float epsabs, epsrel;
    float pivot_thr;
    const float *init_params;
    unsigned long long *stats;
    int level;          // 0: fresh candidates, 1: fits suspended by level 0
    int budget;         // level-0 iteration budget (0: none)
    int *cont;          // continuation queue, laid out like order
    float *cont_state;  // saved solver state of suspended fits
    int cont_stride;
    int compensated;    // FP32 solver: sum the group's partial normal equations in FP64
    const int *roi_slot;  // ROI mode: first pixel of each candidate's packed ROI (row pitch 2r + 1)
};

template <int METHOD, int S, int TPF, typename T> struct Pass;
template <int S, int TPF, typename T> struct Pass<0, S, TPF, T> {
    __device__ __forceinline__ static void run(const float *roi, int s, int q, T, const T (&te)[5], const T (&dt)[5],
                                               T (&acc)[14], T (&vv)[5], T &chi2, T &dchi, T &dqmax)
    {
        pass_sym<S, TPF, T>(roi, 1, s, q, te, dt, acc, vv, chi2, dchi, dqmax);
    }
};
template <int S, int TPF, typename T> struct Pass<1, S, TPF, T> {
    __device__ __forceinline__ static void run(const float *roi, int s, int q, T w0, const T (&te)[4],
                                               const T (&dt)[4], T (&acc)[9], T (&vv)[4], T &chi2, T &dchi,
                                               T &dqmax)
    {
        pass_fixed<S, TPF, T>(roi, 1, s, q, w0, te, dt, acc, vv, chi2, dchi, dqmax);
    }
};
template <int S, int TPF, typename T> struct Pass<7, S, TPF, T> {
    __device__ __forceinline__ static void run(const float *roi, int s, int q, T, const T (&te)[7], const T (&dt)[7],
                                               T (&acc)[27], T (&vv)[7], T &chi2, T &dchi, T &dqmax)
    {
        pass_ell<S, TPF, T>(roi, 1, s, q, te, dt, acc, vv, chi2, dchi, dqmax);
    }
};

// Shared-memory words per fit for a ROI of npx pixels and TPF threads per
// fit: the smallest stride >= npx with stride = TPF (mod 2 TPF), so that the
// 32 lanes of a warp (32/TPF fits, TPF columns each) hit 32 distinct banks.
__host__ __device__ constexpr int roi_stride(int npx, int tpf)
{
    return npx + ((tpf - npx % (2 * tpf)) + 2 * tpf) % (2 * tpf);
}

template <typename T>
__device__ __forceinline__ T group_sum(T v, int tpf, unsigned mask)
{
    for (int o = tpf >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// Group sum of FP32 partial sums carried out in FP64 and rounded once: with
// TPF threads per fit each partial covers 1/TPF of the ROI, so the total is a
// two-level (pairwise) sum whose rounding error is that of n/TPF terms
// instead of n.
__device__ __forceinline__ float group_sum_wide(float v, int tpf, unsigned mask)
{
    double d = (double)v;
    for (int o = tpf >> 1; o > 0; o >>= 1) d += __shfl_xor_sync(mask, d, o);
    return (float)d;
}

template <typename T>
__device__ __forceinline__ T group_max(T v, int tpf, unsigned mask)
{
    for (int o = tpf >> 1; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o));
    return v;
}

// Saved solver state of a suspended fit (continuation level), floats:
// parameters, J^T J, J^T f, D, last step, then 11 scalars.
template <int P> struct ContLayout {
    static constexpr int NT = tri(P);
    static constexpr int TH = 0, A = P, V = P + NT, D = 2 * P + NT, DX = 3 * P + NT, SC = 4 * P + NT;
    static constexpr int STRIDE = ((SC + 11) + 3) / 4 * 4;
};


// Shared memory of the solver block: the ROIs, then (FP64 only) the
// per-fit normal equations.
template <typename T>
__host__ __device__ constexpr int state_smem_per_fit(int P) { return sizeof(T) == 8 ? (3 * tri(P) + 5 * P) * 8 : 0; }

// Process one queue of ROI half-width r: the fresh candidates (level 0) or
// the fits suspended there (level 1). TPF threads cooperate on each fit;
// S = 2r + 1 at compile time, or 0 for a runtime side.
template <int METHOD, typename T, int S, int TPF, bool ESC>
__device__ __forceinline__ void run_class(const K1Args &a, int r, float *smem, unsigned (&st)[ST_N])
{
    constexpr int P = Traits<METHOD>::P;
    constexpr int NT = tri(P);
    constexpr int IX = Traits<METHOD>::IX;
    using SL = StateLayout<P>;
    using CL = ContLayout<P>;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int q = lane % TPF;            // sub-lane within the fit's group
    const int glead = lane - q;          // lane of the group leader
    const bool leader = q == 0;
    const int s = S > 0 ? S : 2 * r + 1;
    const int npx = s * s;
    const int stride = roi_stride(npx, TPF);
    const float *myroi = smem + (tid / TPF) * stride;
    const bool cont = a.level == 1;
    const int *queue = cont ? a.cont : a.order;
    const int cstart = a.meta[m_start(r)];
    const int ccount = a.meta[cont ? m_ccount(r) : m_count(r)];
    int *next = a.meta + (cont ? m_cnext(r) : m_next(r));
    const T inv_s2 = sizeof(T) == 4 ? (T)a.inv_s2 : (T)a.inv_s2_d;
    const T inv_abs_s = sizeof(T) == 4 ? (T)a.inv_abs_s : (T)a.inv_abs_s_d;
    const T w0 = (T)a.w0;

    constexpr bool kSmemState = sizeof(T) == 8;
    T *sstate = nullptr;
    if constexpr (kSmemState) {
        const int roi_bytes = (blockDim.x / TPF) * stride * (int)sizeof(float);
        // one slot of state_smem_per_fit bytes per fit (the group's threads share it)
        sstate = (T *)((char *)smem + ((roi_bytes + 15) / 16) * 16) +
                 (tid / TPF) * (state_smem_per_fit<T>(P) / (int)sizeof(T));
    }
    // FP64: the normal equations, parameters, scaling, last step and the
    // scaled matrix of the damped solve live in the fit's shared-memory slot
    // (in registers they push the FP64 solver into spills); te, the
    // evaluation point, stays in registers
    StateArr<T, NT, kSmemState> A(sstate);
    StateArr<T, P, kSmemState> v(sstate ? sstate + NT : nullptr);
    StateArr<T, P, kSmemState> th(sstate ? sstate + NT + P : nullptr);
    StateArr<T, P, kSmemState> D(sstate ? sstate + NT + 2 * P : nullptr);
    StateArr<T, P, kSmemState> dx(sstate ? sstate + NT + 3 * P : nullptr);
    StateArr<T, P, kSmemState> te(sstate ? sstate + 3 * NT + 4 * P : nullptr);
    T fnorm = 0, delta = 0, par = 0, xnorm = 0, jdx2 = 0, pnorm = 0;
    int phase = 0, it_state = 0, iterations = 0, trial = 0, cidx = -1, xo = 0, yo = 0;
    T minpiv_fit = T(1);
    T margin_fit = T(1e30);
    unsigned esc_fit = 0;
    bool exhausted = false;
#pragma unroll
    for (int k = 0; k < P; ++k) th[k] = v[k] = D[k] = dx[k] = te[k] = T(0);
#pragma unroll
    for (int k = 0; k < NT; ++k) A[k] = T(0);

    auto theta_abs = [&](int k, auto &t) -> T {
        return k == IX ? t[k] + (T)xo : (k == IX + 1 ? t[k] + (T)yo : t[k]);
    };
    auto write_finish = [&](int status) {
        if (leader) {
            T *o = (T *)a.state + (size_t)cidx * a.state_stride;
#pragma unroll
            for (int k = 0; k < P; ++k) o[k] = th[k];
#pragma unroll
            for (int k = 0; k < NT; ++k) o[P + k] = A[k];
            o[SL::FNORM] = fnorm;
            o[SL::ITERS] = (T)iterations;
            o[SL::STATUS] = (T)status;
            o[SL::XOFF] = (T)xo;
            o[SL::YOFF] = (T)yo;
            T lastr = T(0);
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const T tol = (T)a.epsabs + (T)a.epsrel * fabs(theta_abs(k, th));
                const T qq = fdiv(fabs(dx[k]), tol);
                lastr = qq > lastr ? qq : lastr;
            }
            o[SL::MINPIV] = minpiv_fit;
            o[SL::LASTR] = lastr;
            o[SL::NESC] = (T)esc_fit;
            o[SL::MARGIN] = margin_fit;
            st[ST_FITS] += 1;
            st[ST_ITERS] += iterations;
        }
    };
    // park a fit that used up the first level's iteration budget
    auto write_suspend = [&]() {
        if (leader) {
            float *o = a.cont_state + (size_t)cidx * a.cont_stride;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                o[CL::TH + k] = (float)th[k];
                o[CL::V + k] = (float)v[k];
                o[CL::D + k] = (float)D[k];
                o[CL::DX + k] = (float)dx[k];
            }
#pragma unroll
            for (int k = 0; k < NT; ++k) o[CL::A + k] = (float)A[k];
            float *sc = o + CL::SC;
            sc[0] = (float)fnorm;
            sc[1] = (float)delta;
            sc[2] = (float)par;
            sc[3] = (float)xnorm;
            sc[4] = __int_as_float(it_state);
            sc[5] = __int_as_float(iterations);
            sc[6] = (float)minpiv_fit;
            sc[7] = (float)margin_fit;
            sc[8] = __uint_as_float(esc_fit);
            sc[9] = __int_as_float(xo);
            sc[10] = __int_as_float(yo);
            const int slot = atomicAdd(a.meta + m_ccount(r), 1);
            a.cont[cstart + slot] = cidx;
        }
    };
    // finish() and suspend() only mark the fit; its state is written at the
    // next flush(), before the lane is refilled (one inlined copy of each
    // write-out instead of one per call site)
    int done = -1;   // -1 nothing pending, -2 suspended, else the termination status
    auto finish = [&](int status) {
        done = status;
        phase = 0;
    };
    auto suspend = [&]() {
        done = -2;
        phase = 0;
    };
    auto flush = [&]() {
        if (done == -2) write_suspend();
        else if (done >= 0) write_finish(done);
        done = -1;
    };
    auto test_delta = [&]() -> bool {
        bool ok = true;
        T worst = T(0);
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const T tol = (T)a.epsabs + (T)a.epsrel * fabs(theta_abs(k, th));
            ok = ok && (fabs(dx[k]) < tol);
            const T qq = fdiv(fabs(dx[k]), tol);
            worst = qq > worst ? qq : worst;
        }
        margin_fit = fmin(margin_fit, fabs(worst - T(1)));
        return ok;
    };
    auto start_iteration = [&]() {
        if (!cont && a.budget > 0 && iterations >= a.budget) {
            suspend();
            return;
        }
        ++iterations;
        if (fnorm == T(0)) {  // iterate() returns at once; dx is unchanged
            if (test_delta()) finish(T_CONVERGED);
            else {
                iterations = a.max_iter;
                finish(T_MAX_ITER);
            }
            return;
        }
        trial = 0;
        phase = 2;
    };

    unsigned long long c_refill = 0, c_step = 0, c_pass = 0, c_decide = 0;
    long long t_mark = clock64();
    auto lap = [&](unsigned long long &acc_c) {
        const long long t = clock64();
        acc_c += (unsigned long long)(t - t_mark);
        t_mark = t;
    };
    while (true) {
        flush();
        // ---- refill idle groups from the queue: one atomic per warp ----
        const bool want = (phase == 0) && !exhausted;
        const unsigned need = __ballot_sync(kFull, want && leader);
        if (need) {
            const int first = __ffs(need) - 1;
            int base = 0;
            if (lane == first) base = atomicAdd(next, __popc(need));
            base = __shfl_sync(kFull, base, first);
            int my = -1;
            if (want) {
                const int qi = base + __popc(need & ((1u << glead) - 1));
                if (qi < ccount) my = queue[cstart + qi];
                else exhausted = true;
            }
            int fr = 0;
            long long rbase = 0;   // pixel offset of the ROI origin in the pixel array
            if (my >= 0) {
                const Cand cd = a.cands[my];
                const double cx = cd.x, cy = cd.y, cint = cd.intensity, cbg = cd.background;
                fr = cd.frame;
                cidx = my;
                if (cont) {
                    const float *o = a.cont_state + (size_t)my * a.cont_stride;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        th[k] = (T)o[CL::TH + k];
                        v[k] = (T)o[CL::V + k];
                        D[k] = (T)o[CL::D + k];
                        dx[k] = (T)o[CL::DX + k];
                    }
#pragma unroll
                    for (int k = 0; k < NT; ++k) A[k] = (T)o[CL::A + k];
                    const float *sc = o + CL::SC;
                    fnorm = (T)sc[0];
                    delta = (T)sc[1];
                    par = (T)sc[2];
                    xnorm = (T)sc[3];
                    it_state = __float_as_int(sc[4]);
                    iterations = __float_as_int(sc[5]);
                    minpiv_fit = (T)sc[6];
                    margin_fit = (T)sc[7];
                    esc_fit = __float_as_uint(sc[8]);
                    xo = __float_as_int(sc[9]);
                    yo = __float_as_int(sc[10]);
                    phase = 3;  // resume: start the next outer iteration after staging
                } else {
                    xo = (int)floor(cx - (double)r);
                    yo = (int)floor(cy - (double)r);
                    minpiv_fit = T(1);
                    margin_fit = T(1e30);
                    esc_fit = 0;
                    if (a.init_params && !isnan(a.init_params[(size_t)my * P])) {
                        const float *ip = a.init_params + (size_t)my * P;
#pragma unroll
                        for (int k = 0; k < P; ++k) {
                            const double off = k == IX ? (double)xo : (k == IX + 1 ? (double)yo : 0.0);
                            th[k] = (T)((double)ip[k] - off);
                        }
                    } else {
                        const T xl = (T)(cx - (double)xo), yl = (T)(cy - (double)yo);
                        if constexpr (METHOD == 0) {
                            th[0] = (T)cint; th[1] = w0; th[2] = xl; th[3] = yl; th[4] = (T)cbg;
                        } else if constexpr (METHOD == 1) {
                            th[0] = (T)cint; th[1] = xl; th[2] = yl; th[3] = (T)cbg;
                        } else {
                            th[0] = (T)cint; th[1] = w0; th[2] = w0; th[3] = xl; th[4] = yl;
                            th[5] = T(0); th[6] = (T)cbg;
                        }
                    }
                    phase = 1;
                }
                rbase = a.roi_slot ? (long long)a.roi_slot[my]
                                   : (long long)fr * a.frame_px + xo + (long long)yo * a.n_rows;
            }
            // warp-cooperative ROI staging: global uint16 -> shared float
            unsigned got = __ballot_sync(kFull, my >= 0 && leader);
            const int pitch = a.roi_slot ? s : a.n_rows;   // a packed ROI's rows are 2r + 1 pixels apart
            while (got) {
                const int src = __ffs(got) - 1;
                got &= got - 1;
                const long long sbase = __shfl_sync(kFull, rbase, src);
                const uint16_t *fb = a.frames + sbase;
                float *dst = smem + ((tid - lane + src) / TPF) * stride;
                for (int k = lane; k < npx; k += 32) {
                    const int j = k / s, i = k - j * s;
                    dst[k] = (float)__ldg(fb + i + (size_t)j * pitch);
                }
            }
            __syncwarp();
        }
        // fits resumed from level 0 and fits whose last step was accepted
        // start their next outer iteration here (one inlined copy of it)
        if (phase == 3) start_iteration();
        if (__ballot_sync(kFull, phase != 0) == 0) break;
        lap(c_refill);

        // ---- choose this fit's evaluation point (identical in every sub-lane) ----
        bool do_pass = false;
        if (phase == 1) {
#pragma unroll
            for (int k = 0; k < P; ++k) te[k] = th[k];
            do_pass = true;
        } else if (phase == 2) {
            ++trial;
            T invD[P], g[P], z[P];
            StateArr<T, NT, kSmemState> Ms(sstate ? sstate + NT + 4 * P : nullptr);
#pragma unroll
            for (int k = 0; k < P; ++k) {
                invD[k] = frcp(D[k]);
                g[k] = v[k] * invD[k];
            }
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = i; j < P; ++j) Ms[pku(P, i, j)] = A[pku(P, i, j)] * invD[i] * invD[j];
            unsigned nl = 0, ne = 0;
            bool sing = false;
            T npiv;
            lmpar_scaled<P, T, ESC>(Ms, g, delta, par, z, a.pivot_thr, nl, ne, sing, npiv, margin_fit,
                                    sstate ? sstate + 2 * NT + 4 * P : nullptr);
            if (leader) {
                st[ST_LAMBDA] += nl;
                st[ST_ESC] += ne;
            }
            esc_fit += ne;
            minpiv_fit = npiv < minpiv_fit ? npiv : minpiv_fit;
            if (sing) {
                finish(T_SINGULAR);
            } else {
                T pn2 = T(0);
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    dx[k] = -z[k] * invD[k];
                    te[k] = th[k] + dx[k];
                    pn2 += z[k] * z[k];
                }
                pnorm = fsqrt(pn2);
                if (it_state == 1 && pnorm < delta) delta = pnorm;
                T qf = T(0);
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    T row = T(0);
#pragma unroll
                    for (int j = 0; j < P; ++j) row += Ms[i <= j ? pku(P, i, j) : pku(P, j, i)] * z[j];
                    qf += z[i] * row;
                }
                jdx2 = qf;
                const bool bad = (METHOD == 0 && te[1] == T(0)) || (METHOD == 7 && (te[1] == T(0) || te[2] == T(0)));
                if (bad) finish(T_EBADFUNC);
                else do_pass = true;
            }
        }

        // ---- the pass: model, Jacobian and normal equations at te ----
        // All lanes reconverge here so that the pixel loop runs once for the
        // whole warp rather than once per divergent group.
        __syncwarp();
        lap(c_step);
        const unsigned pmask = __ballot_sync(kFull, do_pass);
        T acc[NT - 1], vv[P], chi2, dchi, dqmax;
        if (do_pass) {
            T dt[P], tev[P];
#pragma unroll
            for (int k = 0; k < P; ++k) {
                dt[k] = phase == 2 ? dx[k] : T(0);
                tev[k] = te[k];
            }
            Pass<METHOD, S, TPF, T>::run(myroi, s, q, w0, tev, dt, acc, vv, chi2, dchi, dqmax);
            if constexpr (TPF > 1 && sizeof(T) == 4) {
                if (a.compensated) {
#pragma unroll
                    for (int k = 0; k < NT - 1; ++k) acc[k] = group_sum_wide(acc[k], TPF, pmask);
#pragma unroll
                    for (int k = 0; k < P; ++k) vv[k] = group_sum_wide(vv[k], TPF, pmask);
                    chi2 = group_sum_wide(chi2, TPF, pmask);
                } else {
#pragma unroll
                    for (int k = 0; k < NT - 1; ++k) acc[k] = group_sum(acc[k], TPF, pmask);
#pragma unroll
                    for (int k = 0; k < P; ++k) vv[k] = group_sum(vv[k], TPF, pmask);
                    chi2 = group_sum(chi2, TPF, pmask);
                }
                dchi = group_sum(dchi, TPF, pmask);
                dqmax = group_max(dqmax, TPF, pmask);
            } else if constexpr (TPF > 1) {
#pragma unroll
                for (int k = 0; k < NT - 1; ++k) acc[k] = group_sum(acc[k], TPF, pmask);
#pragma unroll
                for (int k = 0; k < P; ++k) vv[k] = group_sum(vv[k], TPF, pmask);
                chi2 = group_sum(chi2, TPF, pmask);
                dchi = group_sum(dchi, TPF, pmask);
                dqmax = group_max(dqmax, TPF, pmask);
            }
            if (leader) {
                if (phase == 1) {
                    st[ST_J] += 1;
                    st[ST_PIXJ] += npx;
                } else {
                    st[ST_F] += 1;
                    st[ST_PIXF] += npx;
                }
            }
        }

        __syncwarp();
        lap(c_pass);
        // ---- decide ----
        if (do_pass) {
            const T fn1 = fsqrt(chi2) * inv_abs_s;
            if (phase == 1) {
                // gsl_multifit_fdfsolver_set for lmsder
#pragma unroll
                for (int k = 0; k < NT - 1; ++k) A[k] = acc[k] * inv_s2;
                A[NT - 1] = (T)npx * inv_s2;
#pragma unroll
                for (int k = 0; k < P; ++k) v[k] = vv[k] * inv_s2;
                fnorm = fn1;
                T xn2 = T(0);
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    const T cn = sqrt(A[pku(P, k, k)]);
                    D[k] = cn == T(0) ? T(1) : cn;
                    const T t = D[k] * theta_abs(k, th);
                    xn2 += t * t;
                    dx[k] = T(0);
                }
                xnorm = sqrt(xn2);
                delta = xnorm > T(0) ? T(100) * xnorm : T(100);
                par = T(0);
                it_state = 1;
                iterations = 0;
                phase = 3;  // next outer iteration, started after the refill
            } else {
                T actred = T(-1);
                if (T(0.1) * fn1 < fnorm) {
                    if (dqmax < T(0.25)) {
                        // accurate |f|^2 change from the per-pixel model differences
                        actred = fdiv(-(dchi * inv_s2), fnorm * fnorm);
                    } else {
                        const T u = fdiv(fn1, fnorm);
                        actred = T(1) - u * u;
                    }
                }
                const T if2 = frcp(fnorm * fnorm);
                const T t1s = jdx2 * if2;
                const T t2s = par * pnorm * pnorm * if2;
                const T prered = t1s + T(2) * t2s;
                const T dirder = -(t1s + t2s);
                const T ratio = prered > T(0) ? fdiv(actred, prered) : T(0);
                margin_fit = fmin(margin_fit, fmin(fabs(ratio - T(0.25)), fmin(fabs(ratio - T(0.75)),
                                                                              fabs(ratio - T(1e-4)))));
                if (ratio > T(0.25)) {
                    if (par == T(0) || ratio >= T(0.75)) {
                        delta = pnorm / T(0.5);
                        par *= T(0.5);
                    }
                } else {
                    T temp = (actred >= T(0)) ? T(0.5) : fdiv(T(0.5) * dirder, dirder + T(0.5) * actred);
                    if (T(0.1) * fn1 >= fnorm || temp < T(0.1)) temp = T(0.1);
                    const T lim = pnorm / T(0.1);
                    delta = temp * (delta < lim ? delta : lim);
                    par /= temp;
                }
                if (ratio >= T(1e-4)) {
                    T xn2 = T(0);
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        th[k] = te[k];
                        const T t = D[k] * theta_abs(k, th);
                        xn2 += t * t;
                        v[k] = vv[k] * inv_s2;
                    }
#pragma unroll
                    for (int k = 0; k < NT - 1; ++k) A[k] = acc[k] * inv_s2;
                    A[NT - 1] = (T)npx * inv_s2;
                    xnorm = sqrt(xn2);
                    fnorm = fn1;
                    ++it_state;
                    if (leader) {
                        st[ST_J] += 1;  // the accepted trial's Jacobian
                        st[ST_PIXJ] += npx;
                    }
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const T cn = sqrt(A[pku(P, k, k)]);
                        const T cnn = cn == T(0) ? T(1) : cn;
                        if (cnn > D[k]) D[k] = cnn;
                    }
                    if (test_delta()) finish(T_CONVERGED);
                    else if (iterations >= a.max_iter) finish(T_MAX_ITER);
                    else phase = 3;
                } else {
                    T gmax = T(0);
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const T gk = fabs(fdiv(v[k], D[k]));
                        if (gk > gmax) gmax = gk;
                    }
                    const T gnorm = fdiv(gmax, fnorm);
                    if (fabs(actred) <= (T)kDblEps && prered <= (T)kDblEps && T(0.5) * ratio <= T(1))
                        finish(T_ETOLF);
                    else if (delta <= (T)kDblEps * xnorm)
                        finish(T_ETOLX);
                    else if (gnorm <= (T)kDblEps)
                        finish(T_ETOLG);
                    else if (trial >= 10)
                        finish(T_ENOPROG);
                }
            }
        }
        __syncwarp();
        lap(c_decide);
    }
    flush();
    if (lane == 0) {
        st[ST_CYC_REFILL] += (unsigned)(c_refill >> 10);
        st[ST_CYC_STEP] += (unsigned)(c_step >> 10);
        st[ST_CYC_PASS] += (unsigned)(c_pass >> 10);
        st[ST_CYC_DECIDE] += (unsigned)(c_decide >> 10);
    }
}

// blocks of 128 threads resident per SM the register budget is sized for
// (FP64: one, i.e. the full 255 registers)
__host__ __device__ constexpr int k1_min_blocks(int method, int bytes) { return bytes == 8 ? 1 : (method == 7 ? 2 : 3); }

template <int METHOD, typename T, int S, int TPF, bool ESC>
__global__ void __launch_bounds__(128, k1_min_blocks(METHOD, sizeof(T))) k1_lm_fit(K1Args a, int r)
{
    extern __shared__ float smem[];
    unsigned st[ST_N];
#pragma unroll
    for (int k = 0; k < ST_N; ++k) st[k] = 0;
    if (a.meta[a.level == 1 ? m_ccount(r) : m_count(r)] > 0) run_class<METHOD, T, S, TPF, ESC>(a, r, smem, st);
    // warp-reduce the counters, one atomic per warp and counter
#pragma unroll
    for (int k = 0; k < ST_N; ++k) {
        unsigned long long vsum = st[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vsum += __shfl_xor_sync(kFull, vsum, o);
        if ((threadIdx.x & 31) == 0 && vsum) atomicAdd(&a.stats[k], vsum);
    }
}

struct K2Args {
    const Cand *cands;
    int n;
    int method;
    double w0;
    int r_default;
    const float *state32;   // FP32 solver state (NULL when the whole call ran in FP64)
    const double *state64;  // FP64 solver state of re-run fits (or of every fit)
    const int *rerun;       // >= 0 where the fit was re-run in FP64 (NULL: none)
    int state_stride;
    int ncol_total;
    double *out;
    uint8_t *flags;
    float *params_out;
    float *diag;
};

// Symmetric 2x2 eigen-decomposition with ascending eigenvalues (the
// reference uses Eigen::SelfAdjointEigenSolver, Localization.cpp:529-547);
// theta = atan(v00 / v10) of the eigenvector of the smaller eigenvalue.
__device__ bool eig2_theta(double a, double b, double c, double &l0, double &l1, double &theta)
{
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) return false;
    const double ht = 0.5 * (a + c), hd = 0.5 * (a - c);
    const double rad = hypot(hd, b);
    l0 = ht - rad;
    l1 = ht + rad;
    double v0, v1;
    if (b == 0.0) {
        if (a <= c) { v0 = 1.0; v1 = 0.0; } else { v0 = 0.0; v1 = 1.0; }
    } else {
        const double ua0 = b, ua1 = l0 - a, ub0 = l0 - c, ub1 = b;
        if (ua0 * ua0 + ua1 * ua1 >= ub0 * ub0 + ub1 * ub1) { v0 = ua0; v1 = ua1; }
        else { v0 = ub0; v1 = ub1; }
    }
    theta = (v1 == 0.0) ? 0.0 : atan(v0 / v1);
    return true;
}

// diag((J^T J)^-1) by Cholesky in FP64 (gsl_multifit_covar(J, 0.0, .) at
// Localization.cpp:185, 355, 556 forms the same inverse through QR).
template <int P>
__device__ bool inverse_diagonal(const double (&A)[tri(P)], double (&cd)[P])
{
    double L[tri(P)], inv[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        double d = A[pku(P, j, j)];
#pragma unroll
        for (int k = 0; k < j; ++k) d -= L[pkl(j, k)] * L[pkl(j, k)];
        if (!(d > 0.0)) return false;
        const double l = sqrt(d);
        L[pkl(j, j)] = l;
        inv[j] = 1.0 / l;
#pragma unroll
        for (int i = j + 1; i < P; ++i) {
            double s = A[pku(P, j, i)];
#pragma unroll
            for (int k = 0; k < j; ++k) s -= L[pkl(i, k)] * L[pkl(j, k)];
            L[pkl(i, j)] = s * inv[j];
        }
    }
    // columns of L^-1; diag(A^-1)_j = sum_k (L^-1)_{kj}^2
#pragma unroll
    for (int j = 0; j < P; ++j) cd[j] = 0.0;
#pragma unroll
    for (int col = 0; col < P; ++col) {
        double y[P];
#pragma unroll
        for (int i = 0; i < P; ++i) {
            if (i < col) { y[i] = 0.0; continue; }
            double s = (i == col) ? 1.0 : 0.0;
#pragma unroll
            for (int k = 0; k < i; ++k) s -= L[pkl(i, k)] * y[k];
            y[i] = s * inv[i];
        }
#pragma unroll
        for (int i = 0; i < P; ++i) cd[col] += y[i] * y[i];
    }
    return true;
}

template <int METHOD>
__global__ void k2_finalize(K2Args a)
{
    constexpr int P = Traits<METHOD == 5 ? 7 : METHOD>::P;
    constexpr int NT = tri(P);
    using SL = StateLayout<P>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    if (a.flags[i] != F_PENDING) return;
    const Cand cd = a.cands[i];
    const bool r64 = a.state32 == nullptr || (a.rerun && a.rerun[i] >= 0);
    const size_t base = (size_t)i * a.state_stride;
    auto sv = [&](int k) -> double { return r64 ? a.state64[base + k] : (double)a.state32[base + k]; };
    const int iterations = (int)sv(SL::ITERS);
    const int status = (int)sv(SL::STATUS);
    const int xo = (int)sv(SL::XOFF), yo = (int)sv(SL::YOFF);
    const int r = cd.half_width > 0 ? cd.half_width : a.r_default;
    const int xm = xo + 2 * r, ym = yo + 2 * r;
    const double w0 = a.w0;
    const int ncol = ref_cols(METHOD);
    double *row = a.out + (size_t)i * a.ncol_total;
    row[0] = (double)cd.frame;
    for (int k = 1; k < ncol; ++k) row[k] = CUDART_NAN;
    row[ncol] = (double)iterations;
    row[ncol + 1] = (double)status;

    double x[P];
#pragma unroll
    for (int k = 0; k < P; ++k) x[k] = sv(k);
    constexpr int IX = METHOD == 0 ? 2 : METHOD == 1 ? 1 : 3;
    x[IX] += xo;
    x[IX + 1] += yo;
    if constexpr (METHOD == 0) x[1] = fabs(x[1]);
    if constexpr (METHOD == 5 || METHOD == 7) {
        x[1] = fabs(x[1]);
        x[2] = fabs(x[2]);
    }
    if (a.params_out) {
#pragma unroll
        for (int k = 0; k < P; ++k) a.params_out[(size_t)i * P + k] = (float)x[k];
    }
    if (a.diag) {
        float *dg = a.diag + (size_t)i * 8;
        const size_t b32 = (size_t)i * a.state_stride;
        dg[0] = (float)sv(SL::MINPIV);
        dg[1] = (float)sv(SL::LASTR);
        dg[2] = (float)sv(SL::NESC);
        dg[3] = (float)sv(SL::MARGIN);
        dg[4] = r64 && a.state32 != nullptr ? 1.0f : 0.0f;
        dg[5] = a.state32 ? a.state32[b32 + SL::ITERS] : (float)iterations;
        dg[6] = a.state32 ? a.state32[b32 + SL::STATUS] : (float)status;
        dg[7] = 0.0f;
    }
    uint8_t flag = F_KEPT;
    if (x[0] <= 0) flag = F_AMPLITUDE;
    else if (x[IX] < xo || x[IX] > xm || x[IX + 1] < yo || x[IX + 1] > ym) flag = F_WINDOW;
    if (flag != F_KEPT) {
        a.flags[i] = flag;
        return;
    }
    double A[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) A[k] = sv(P + k);
    const double chi = sv(SL::FNORM);
    double cv[P];

    if constexpr (METHOD == 0) {
        if (x[1] < 0.4 * w0 || x[1] > w0 * 1.5) flag = F_WIDTH;
        else {
            const bool ok = inverse_diagonal<P>(A, cv);
            if (!ok)
                for (int k = 0; k < P; ++k) cv[k] = CUDART_NAN;
            const double dof = (double)((2 * r - 1) * (2 * r - 1) - 5);  // Localization.cpp:187 as written
            const double c = fmax(1.0, chi / sqrt(dof));
            const double pi = 3.1415926535897932384626433;
            const double width = x[1];
            const double widthDev = c * sqrt(cv[1]);
            const double integral = 2 * pi * width * width * x[0];
            const double relA = c * sqrt(cv[0]) / x[0];
            const double relW = widthDev / width;
            row[1] = integral;
            row[2] = width;
            row[3] = x[2];
            row[4] = x[3];
            row[5] = x[4];
            row[6] = 2 * pi * integral * sqrt(relA * relA + 2 * relW * relW);
            row[7] = widthDev;
            row[8] = c * sqrt(cv[2]);
            row[9] = c * sqrt(cv[3]);
            row[10] = c * sqrt(cv[4]);
            row[11] = 1.0;
        }
    } else if constexpr (METHOD == 1) {
        if (fabs(x[1] - cd.x) > 2.0 * w0 || fabs(x[2] - cd.y) > 2.0 * w0) flag = F_DRIFT;
        else {
            const bool ok = inverse_diagonal<P>(A, cv);
            if (!ok)
                for (int k = 0; k < P; ++k) cv[k] = CUDART_NAN;
            const double dof = (double)((2 * r - 1) * (2 * r - 1) - 4);
            const double c = fmax(1.0, chi / sqrt(dof));
            const double pi = 3.1415926535897932384626433;
            const double integral = 2 * pi * w0 * w0 * x[0];
            const double relA = c * sqrt(cv[0]) / x[0];
            row[1] = integral;
            row[2] = x[1];
            row[3] = x[2];
            row[4] = x[3];
            row[5] = 2 * pi * integral * w0 * w0 * sqrt(relA * relA);
            row[6] = c * sqrt(cv[1]);
            row[7] = c * sqrt(cv[2]);
            row[8] = c * sqrt(cv[3]);
            row[9] = 1.0;
        }
    } else {
        const double sx = x[1], sy = x[2], rho = x[5];
        double l0, l1, theta;
        if (!eig2_theta(sx * sx, rho * sx * sy, sy * sy, l0, l1, theta)) flag = F_EIGEN;
        else {
            const double s1 = sqrt(l0), s2 = sqrt(l1);
            if (!(((s1 >= 0.4 * w0) && (s1 <= 1.5 * w0)) || ((s2 >= 0.4 * w0) && (s2 <= 1.5 * w0)))) flag = F_NO_AXIS;
            else {
                const bool ok = inverse_diagonal<P>(A, cv);
                if (!ok)
                    for (int k = 0; k < P; ++k) cv[k] = CUDART_NAN;
                const double dof = (double)((2 * r - 1) * (2 * r - 1) - 7);
                const double c = fmax(1.0, chi / sqrt(dof));
                const double pi = 3.1415926535897932384626433;
                const double corrDev = c * sqrt(cv[5]);
                const double sxDev = c * sqrt(cv[1]), syDev = c * sqrt(cv[2]);
                double sn, cs;
                sincos(theta, &sn, &cs);
                const double s1Dev = sxDev * cs + syDev * sn;
                const double s2Dev = sxDev * sn + syDev * cs;
                const double ampDev = c * sqrt(cv[0]);
                const double omr = 1 - rho * rho;
                const double integral = 2.0 * pi * x[0] * sqrt(omr) * s1 * s2;
                row[1] = integral;
                row[2] = s1;
                row[3] = s2;
                row[4] = x[3];
                row[5] = x[4];
                row[6] = theta;
                row[7] = x[6];
                row[8] = integral * sqrt(ampDev * ampDev / x[0] / x[0] + rho * rho * corrDev * corrDev / omr / omr +
                                         s1Dev * s1Dev / s1 / s1 + s2Dev * s2Dev / s2 / s2);
                row[9] = s1Dev;
                row[10] = s2Dev;
                row[11] = c * sqrt(cv[3]);
                row[12] = c * sqrt(cv[4]);
                row[13] = 0.0;
                row[14] = c * sqrt(cv[6]);
                row[15] = 1.0;
                if constexpr (METHOD == 5) {
                    if ((0.75 * s1 > s2) || (1.25 * s1 < s2)) flag = F_SYM_RATIO;
                    else if (((s1 < w0 * 0.7) || (s1 > w0 * 1.3)) && ((s2 < w0 * 0.7) || (s2 > w0 * 1.3)))
                        flag = F_SYM_WIDTH;
                }
            }
        }
    }
    if (flag != F_KEPT) {
        for (int k = 1; k < ncol; ++k) row[k] = CUDART_NAN;
    }
    a.flags[i] = flag;
}

int solver_method(int method) { return method == 5 ? 7 : method; }

template <int METHOD, typename T, int S, int TPF, bool ESC = false>
cudaError_t launch_k1_s(const K1Args &ka, int r, int tpb, int bps_req, cudaStream_t stream)
{
    auto kern = k1_lm_fit<METHOD, T, S, TPF, ESC>;
    const int side = 2 * r + 1;
    const int per_fit = roi_stride(side * side, TPF) * (int)sizeof(float);
    constexpr int P = Traits<METHOD>::P;
    auto smem_of = [&](int t) { return ((t / TPF) * per_fit + 15) / 16 * 16 + (t / TPF) * state_smem_per_fit<T>(P); };
    // fewer threads per block when the block's shared memory would exceed 227 KB
    while (tpb > 32 && smem_of(tpb) > 227 * 1024) tpb -= 32;
    const int smem = smem_of(tpb);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, bps = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, tpb, smem);
    if (e != cudaSuccess) return e;
    if (bps < 1) return cudaErrorInvalidConfiguration;
    if (bps_req > 0 && bps_req < bps) bps = bps_req;
    kern<<<nsm * bps, tpb, smem, stream>>>(ka, r);
    return cudaGetLastError();
}

template <int METHOD, typename T, int TPF>
cudaError_t launch_k1_tpf(const K1Args &ka, int r, int tpb, int bps_req, cudaStream_t stream)
{
    if constexpr (sizeof(T) == 8) {
        return launch_k1_s<METHOD, T, 0, TPF>(ka, r, tpb, bps_req, stream);
    } else {
        // FP64 pivot escalation: one runtime-side instantiation per method
        // and threads per fit
        if (ka.pivot_thr > 0.0f) return launch_k1_s<METHOD, T, 0, TPF, true>(ka, r, tpb, bps_req, stream);
        switch (2 * r + 1) {
        case 5: return launch_k1_s<METHOD, T, 5, TPF>(ka, r, tpb, bps_req, stream);
        case 7: return launch_k1_s<METHOD, T, 7, TPF>(ka, r, tpb, bps_req, stream);
        case 9: return launch_k1_s<METHOD, T, 9, TPF>(ka, r, tpb, bps_req, stream);
        case 11: return launch_k1_s<METHOD, T, 11, TPF>(ka, r, tpb, bps_req, stream);
        case 13: return launch_k1_s<METHOD, T, 13, TPF>(ka, r, tpb, bps_req, stream);
        case 15: return launch_k1_s<METHOD, T, 15, TPF>(ka, r, tpb, bps_req, stream);
        case 17: return launch_k1_s<METHOD, T, 17, TPF>(ka, r, tpb, bps_req, stream);
        default: return launch_k1_s<METHOD, T, 0, TPF>(ka, r, tpb, bps_req, stream);
        }
    }
}

// One persistent solver launch for the queue of half-width r with tpf
// threads per fit (1, 4 or 8 for FP32; 1, 2, 4 or 8 for FP64).
template <int METHOD, typename T>
cudaError_t launch_k1(const K1Args &ka, int r, int tpb, int bps_req, int tpf, cudaStream_t stream)
{
    if constexpr (sizeof(T) == 8) {
        return tpf == 4 ? launch_k1_tpf<METHOD, T, 4>(ka, r, tpb, bps_req, stream)
             : tpf == 8 ? launch_k1_tpf<METHOD, T, 8>(ka, r, tpb, bps_req, stream)
             : tpf == 2 ? launch_k1_tpf<METHOD, T, 2>(ka, r, tpb, bps_req, stream)
                        : launch_k1_tpf<METHOD, T, 1>(ka, r, tpb, bps_req, stream);
    } else {
        switch (tpf) {
        case 4: return launch_k1_tpf<METHOD, T, 4>(ka, r, tpb, bps_req, stream);
        case 8: return launch_k1_tpf<METHOD, T, 8>(ka, r, tpb, bps_req, stream);
        // a half warp per fit (runtime ROI side only)
        case 16: return launch_k1_s<METHOD, T, 0, 16>(ka, r, tpb, bps_req, stream);
        default: return launch_k1_tpf<METHOD, T, 1>(ka, r, tpb, bps_req, stream);
        }
    }
}

int cont_stride_of(int m) { return m == 0 ? ContLayout<5>::STRIDE : m == 1 ? ContLayout<4>::STRIDE : ContLayout<7>::STRIDE; }

}  // namespace

int state_stride(int method)
{
    const int m = solver_method(method);
    return m == 0 ? StateLayout<5>::STRIDE : m == 1 ? StateLayout<4>::STRIDE : StateLayout<7>::STRIDE;
}

// Scratch layout (256-byte aligned pieces): cls, order, meta, stats, cont,
// cont_state, state (FP32 state, or FP64 state when the call runs in FP64),
// then for the FP64 re-run of flagged fits: cls2, order2, meta2, state64.
namespace {
size_t al256(size_t b) { return (b + 255) / 256 * 256; }
}

static_assert(kStatWords >= 2 * ST_N + 1, "statistics words");

size_t scratch_bytes(int method, int n, int precision, int rerun, int warm)
{
    const size_t el = precision == 1 ? sizeof(double) : sizeof(float);
    const int m = solver_method(method);
    size_t b = al256(sizeof(int) * (size_t)n) * 2 + al256(sizeof(int) * kMetaInts) +
               al256(sizeof(unsigned long long) * kStatWords) + al256(sizeof(int) * (size_t)n) +
               al256(sizeof(float) * (size_t)n * cont_stride_of(m)) + al256(el * (size_t)n * state_stride(method));
    if (precision != 1 && rerun)
        b += al256(sizeof(int) * (size_t)n) * 3 + al256(sizeof(int) * kMetaInts) * 2 +
             al256(sizeof(double) * (size_t)n * state_stride(method));
    if (warm) b += al256(sizeof(float) * (size_t)n * 8);
    return b;
}

void carve_scratch(void *base, int method, int n, int precision, int rerun, Scratch *s, int warm)
{
    const size_t el = precision == 1 ? sizeof(double) : sizeof(float);
    char *p = (char *)base;
    s->cls = (int *)p;
    p += al256(sizeof(int) * (size_t)n);
    s->order = (int *)p;
    p += al256(sizeof(int) * (size_t)n);
    s->meta = (int *)p;
    p += al256(sizeof(int) * kMetaInts);
    s->stats = (unsigned long long *)p;
    p += al256(sizeof(unsigned long long) * kStatWords);
    s->cont = (int *)p;
    p += al256(sizeof(int) * (size_t)n);
    s->cont_state = (float *)p;
    p += al256(sizeof(float) * (size_t)n * cont_stride_of(solver_method(method)));
    s->state = (void *)p;
    p += al256(el * (size_t)n * state_stride(method));
    if (precision != 1 && rerun) {
        s->cls2 = (int *)p;
        p += al256(sizeof(int) * (size_t)n);
        s->order2 = (int *)p;
        p += al256(sizeof(int) * (size_t)n);
        s->meta2 = (int *)p;
        p += al256(sizeof(int) * kMetaInts);
        s->order3 = (int *)p;
        p += al256(sizeof(int) * (size_t)n);
        s->meta3 = (int *)p;
        p += al256(sizeof(int) * kMetaInts);
        s->state64 = (double *)p;
        p += al256(sizeof(double) * (size_t)n * state_stride(method));
    } else {
        s->cls2 = s->order2 = s->meta2 = s->order3 = s->meta3 = nullptr;
        s->state64 = nullptr;
    }
    s->init = warm ? (float *)p : nullptr;
}

namespace {

template <typename T>
cudaError_t launch_queues(const FitParams &p, const K1Args &k1_in, const int *counts, int r_cap, int tpb,
                          bool two_level, int tpf_fixed, cudaStream_t stream, int *err_detail)
{
    K1Args k1 = k1_in;
    const int m = solver_method(p.method);
    cudaError_t e = cudaSuccess;
    for (int level = 0; level < (two_level ? 2 : 1); ++level) {
        k1.level = level;
        k1.budget = two_level ? p.level0_budget : 0;
        const int tpf = tpf_fixed > 0 ? tpf_fixed : (level == 0 ? p.threads_per_fit : p.tail_threads_per_fit);
        for (int r = r_cap; r >= 1; --r) {
            if (counts[r] <= 0) continue;
            e = m == 0 ? launch_k1<0, T>(k1, r, tpb, p.blocks_per_sm, tpf, stream)
              : m == 1 ? launch_k1<1, T>(k1, r, tpb, p.blocks_per_sm, tpf, stream)
                       : launch_k1<7, T>(k1, r, tpb, p.blocks_per_sm, tpf, stream);
            if (e == cudaErrorInvalidValue) *err_detail = 1;
            if (e != cudaSuccess) return e;
            if (p.launches) ++*p.launches;
        }
    }
    return e;
}

}  // namespace

cudaError_t enqueue_fit(const FitParams &p, const Scratch &s, cudaStream_t stream, int *err_detail)
{
    *err_detail = 0;
    const int n = p.n_cands;
    const int ncol_total = ref_cols(p.method) + 2;
    const int r_default = (int)std::ceil(p.w0 * 4.0);
    const bool rerun = p.precision != 1 && p.fp64_rerun && s.state64 != nullptr;
    cudaError_t e;
    e = cudaMemsetAsync(s.meta, 0, sizeof(int) * kMetaInts, stream);
    if (e != cudaSuccess) return e;
    if (rerun && (e = cudaMemsetAsync(s.meta2, 0, sizeof(int) * kMetaInts, stream)) != cudaSuccess) return e;
    const bool long_q = rerun && p.long_rerun_iters > 0;
    if (long_q && (e = cudaMemsetAsync(s.meta3, 0, sizeof(int) * kMetaInts, stream)) != cudaSuccess) return e;
    e = cudaMemsetAsync(s.stats, 0, sizeof(unsigned long long) * kStatWords, stream);
    if (e != cudaSuccess) return e;
    if (p.method == 6) {
        for (int k = 0; k < 4; ++k)
            if (p.ev[k]) cudaEventRecord(p.ev[k], stream);
        return enqueue_mlewg(p, s.stats, stream);
    }
    if (n == 0) {
        for (int k = 0; k < 4; ++k)
            if (p.ev[k]) cudaEventRecord(p.ev[k], stream);
        return cudaSuccess;
    }

    const int r_cap = p.max_half_width > 0 ? (p.max_half_width < kMaxHalfWidth ? p.max_half_width : kMaxHalfWidth)
                                           : kMaxHalfWidth;
    auto mark = [&](int k) {
        if (p.ev[k]) cudaEventRecord(p.ev[k], stream);
    };
    auto bump = [&]() {
        if (p.launches) ++*p.launches;
    };
    mark(0);
    // the pixel array the solver reads: the frames, or (ROI mode) the slots
    const bool roi_mode = p.roi_slot != nullptr;
    // the start proposal cuts its windows from whole frames
    if (roi_mode && p.warm) return cudaErrorInvalidValue;
    const uint16_t *px = roi_mode ? p.roi_stack : p.frames;
    const long long px_frame = roi_mode ? 0 : (long long)p.n_rows * p.n_cols;
    const int px_pitch = roi_mode ? 0 : p.n_rows;   // ROI mode: each ROI's own side
    K0Args k0{(const Cand *)p.cands, n, p.n_frames, p.n_rows, p.n_cols, r_default, r_cap, p.method, ncol_total,
              p.out, p.flags, s.cls, s.meta, rerun ? s.cls2 : nullptr, p.roi_slot, p.roi_px};
    const int nb = (n + 255) / 256;
    k0_classify<<<nb, 256, 0, stream>>>(k0);
    k0_classes<<<1, 32, 0, stream>>>(s.meta);
    k0_scatter<<<nb, 256, 0, stream>>>(s.cls, n, s.meta, s.order);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    bump();
    bump();
    bump();

    // which half-width queues exist: known bound from the caller, or the
    // histogram read back (one small synchronous copy)
    int counts[K];
    for (int r = 0; r < K; ++r) counts[r] = r <= r_cap ? 1 : 0;
    if (p.max_half_width <= 0) {
        e = cudaMemcpyAsync(counts, s.meta + m_count(0), sizeof(int) * K, cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return e;
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
    }
    mark(1);
    // learned start proposal and start check, before the solver chains fork
    if (p.warm) {
        e = enqueue_proposal(p.prop, p.frames, (long long)p.n_rows * p.n_cols, p.n_rows, p.n_cols, p.cands, s.cls, n,
                             p.method, (float)p.w0, s.init, s.stats + 2 * ST_N, p.prop.err, stream, p.launches);
        if (e != cudaSuccess) return e;
        if (p.ev_prop) cudaEventRecord(p.ev_prop, stream);
    }
    int tpb = p.threads_per_block > 0 ? p.threads_per_block : 128;
    tpb = (tpb + 31) / 32 * 32;
    if (tpb > 128) tpb = 128;
    const double s_abs = std::fabs(p.sigma);
    const int m = solver_method(p.method);
    K1Args k1{px, px_frame, px_pitch, (const Cand *)p.cands, s.order, s.meta,
              s.state, state_stride(p.method), (float)p.w0, (float)(1.0 / (p.sigma * p.sigma)),
              (float)(1.0 / s_abs), 1.0 / (p.sigma * p.sigma), 1.0 / s_abs, p.max_iter, (float)p.epsabs,
              (float)p.epsrel, p.precision == 1 ? 0.0f : p.pivot_thr, p.warm ? s.init : p.init_params, s.stats,
              0, 0, s.cont, s.cont_state, cont_stride_of(m), p.compensated, p.roi_slot};
    // Each ROI class is an independent chain -- level 0 (every candidate,
    // tpf0 threads per fit, up to `budget` iterations), level 1 (the fits
    // still running, tpf1 threads per fit), the flag pass and the FP64
    // re-run of flagged fits -- forked onto the auxiliary streams so that the
    // chains' tails overlap; the caller's stream joins them before the
    // finaliser.
    const bool two_level = p.precision != 1 && p.level0_budget > 0 && p.level0_budget < p.max_iter;
    int naux = 0;
    while (naux < kMaxAux && p.aux[naux]) ++naux;
    if (naux > 0) {
        e = cudaEventRecord(p.fork, stream);
        if (e != cudaSuccess) return e;
    }
    bool used[kMaxAux] = {false}, used_long[kMaxAux] = {false};
    int chain = 0;
    for (int r = r_cap; r >= 1; --r) {
        if (counts[r] <= 0) continue;
        cudaStream_t cs = stream;
        const int j = naux > 0 ? chain % naux : 0;
        if (naux > 0) {
            cs = p.aux[j];
            if (!used[j]) {
                if ((e = cudaStreamWaitEvent(cs, p.fork, 0)) != cudaSuccess) return e;
                used[j] = true;
            }
        }
        ++chain;
        int cnt1[K];
        for (int q = 0; q < K; ++q) cnt1[q] = q == r ? 1 : 0;
        if (p.precision == 1) {
            e = launch_queues<double>(p, k1, cnt1, r_cap, tpb, false, 1, cs, err_detail);
        } else {
            e = launch_queues<float>(p, k1, cnt1, r_cap, tpb, two_level, 0, cs, err_detail);
            if (e == cudaSuccess && rerun) {
                const int fb = 2 * 148;
                const int wl = p.warm ? p.warm_iter_limit : 0;
                const float *st32 = (const float *)s.state;
                const int sst = state_stride(p.method);
                int *o3 = long_q ? s.order3 : nullptr, *m3 = long_q ? s.meta3 : nullptr;
                const int li = p.long_rerun_iters;
                // a warm fit's reject says nothing about where the reference
                // start's path ends: with a proposal every flagged fit is re-run
                const float skip = p.warm ? 0.0f : p.rerun_skip_rejected;
                switch (m) {
                case 0: k3_flag_class<5><<<fb, 256, 0, cs>>>(st32, sst, s.order, s.meta, p.flags, r, p.rerun_margin,
                                                             p.rerun_pivot, wl, s.cls2, s.order2, s.meta2, li, o3,
                                                             m3, p.rerun_capped, p.rerun_cond, p.rerun_iters, skip, (float)p.w0); break;
                case 1: k3_flag_class<4><<<fb, 256, 0, cs>>>(st32, sst, s.order, s.meta, p.flags, r, p.rerun_margin,
                                                             p.rerun_pivot, wl, s.cls2, s.order2, s.meta2, li, o3,
                                                             m3, p.rerun_capped, p.rerun_cond, p.rerun_iters, skip, (float)p.w0); break;
                default: k3_flag_class<7><<<fb, 256, 0, cs>>>(st32, sst, s.order, s.meta, p.flags, r,
                                                              p.rerun_margin, p.rerun_pivot, wl, s.cls2, s.order2,
                                                              s.meta2, li, o3, m3, p.rerun_capped, p.rerun_cond, p.rerun_iters, skip, (float)p.w0); break;
                }
                if ((e = cudaGetLastError()) != cudaSuccess) return e;
                bump();
                K1Args k64 = k1;
                // warm-started fits fall back to the reference start
                if (p.warm) k64.init_params = nullptr;
                k64.order = s.order2;
                k64.meta = s.meta2;
                k64.state = s.state64;
                k64.pivot_thr = 0.0f;
                k64.stats = s.stats + ST_N;  // counters of the re-run kept apart
                if (long_q) {
                    // the long re-runs: their own stream (when the chain has
                    // one) and more threads per fit; launched first so that
                    // in a serial call they start at the head
                    K1Args kl = k64;
                    kl.order = s.order3;
                    kl.meta = s.meta3;
                    cudaStream_t ls = cs;
                    if (naux > 0 && p.aux_long[j]) {
                        ls = p.aux_long[j];
                        if ((e = cudaEventRecord(p.flagged[j], cs)) != cudaSuccess) return e;
                        if ((e = cudaStreamWaitEvent(ls, p.flagged[j], 0)) != cudaSuccess) return e;
                        used_long[j] = true;
                    }
                    e = launch_queues<double>(p, kl, cnt1, r_cap, tpb, false, p.long_rerun_threads_per_fit, ls,
                                              err_detail);
                    if (e != cudaSuccess) return e;
                }
                // the other flagged fits: fewer threads per fit, more fits in flight
                e = launch_queues<double>(p, k64, cnt1, r_cap, tpb, false, p.rerun_threads_per_fit, cs, err_detail);
            }
        }
        if (e != cudaSuccess) return e;
    }
    for (int j = 0; j < naux; ++j) {
        if (used[j]) {
            if ((e = cudaEventRecord(p.join[j], p.aux[j])) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(stream, p.join[j], 0)) != cudaSuccess) return e;
        }
        if (used_long[j]) {
            if ((e = cudaEventRecord(p.join_long[j], p.aux_long[j])) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(stream, p.join_long[j], 0)) != cudaSuccess) return e;
        }
    }
    if (e != cudaSuccess) return e;
    mark(2);
    K2Args k2{(const Cand *)p.cands, n, p.method, p.w0, r_default,
              p.precision == 1 ? nullptr : (const float *)s.state,
              p.precision == 1 ? (const double *)s.state : s.state64, rerun ? s.cls2 : nullptr,
              state_stride(p.method), ncol_total, p.out, p.flags, p.params_out, p.diag};
    bump();
    switch (p.method) {
    case 0: k2_finalize<0><<<nb, 256, 0, stream>>>(k2); break;
    case 1: k2_finalize<1><<<nb, 256, 0, stream>>>(k2); break;
    case 5: k2_finalize<5><<<nb, 256, 0, stream>>>(k2); break;
    default: k2_finalize<7><<<nb, 256, 0, stream>>>(k2); break;
    }
    mark(3);
    return cudaGetLastError();
}

}  // namespace locb
