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
__host__ __device__ constexpr int m_side(int c) { return 8 + 0 * K + c; }
__host__ __device__ constexpr int m_start(int c) { return 8 + 1 * K + c; }
__host__ __device__ constexpr int m_count(int c) { return 8 + 2 * K + c; }
__host__ __device__ constexpr int m_next(int c) { return 8 + 3 * K + c; }
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
            } else {
                cls = r;
                atomicAdd(&hist[r], 1);
            }
        }
        a.cls[i] = cls;
        a.flags[i] = flag;
        if (flag != F_PENDING) write_reject_row(a.out + (size_t)i * a.ncol_total, a.ncol_total, c.frame);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < K; r += blockDim.x)
        if (hist[r]) atomicAdd(&a.meta[m_hist(r)], hist[r]);
}

// One block: class table in descending half-width order.
__global__ void k0_classes(int *meta)
{
    if (threadIdx.x != 0) return;
    int ncls = 0, start = 0, maxr = 0;
    for (int r = K - 1; r >= 1; --r) {
        const int cnt = meta[m_hist(r)];
        if (cnt == 0) continue;
        if (r > maxr) maxr = r;
        meta[m_side(ncls)] = 2 * r + 1;
        meta[m_start(ncls)] = start;
        meta[m_count(ncls)] = cnt;
        meta[m_next(ncls)] = 0;
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
};

template <int METHOD, int S, typename T> struct Pass;
template <int S, typename T> struct Pass<0, S, T> {
    __device__ __forceinline__ static void run(const float *roi, int ld, int s, T, const T (&te)[5], const T (&dt)[5],
                                               T (&acc)[14], T (&vv)[5], T &chi2, T &dchi, T &dqmax)
    {
        pass_sym<S, T>(roi, ld, s, te, dt, acc, vv, chi2, dchi, dqmax);
    }
};
template <int S, typename T> struct Pass<1, S, T> {
    __device__ __forceinline__ static void run(const float *roi, int ld, int s, T w0, const T (&te)[4],
                                               const T (&dt)[4], T (&acc)[9], T (&vv)[4], T &chi2, T &dchi,
                                               T &dqmax)
    {
        pass_fixed<S, T>(roi, ld, s, w0, te, dt, acc, vv, chi2, dchi, dqmax);
    }
};
template <int S, typename T> struct Pass<7, S, T> {
    __device__ __forceinline__ static void run(const float *roi, int ld, int s, T, const T (&te)[7], const T (&dt)[7],
                                               T (&acc)[27], T (&vv)[7], T &chi2, T &dchi, T &dqmax)
    {
        pass_ell<S, T>(roi, ld, s, te, dt, acc, vv, chi2, dchi, dqmax);
    }
};

// Process one ROI class with the whole warp; S > 0 compile-time side.
template <int METHOD, typename T, int S>
__device__ __noinline__ void run_class(const K1Args &a, int c, float *smem, unsigned (&st)[ST_N])
{
    constexpr int P = Traits<METHOD>::P;
    constexpr int NT = tri(P);
    constexpr int IX = Traits<METHOD>::IX;
    using SL = StateLayout<P>;
    const int ld = blockDim.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wbase = tid - lane;
    const int s = S > 0 ? S : a.meta[m_side(c)];
    const int r = (s - 1) / 2;
    const int npx = s * s;
    const int cstart = a.meta[m_start(c)];
    const int ccount = a.meta[m_count(c)];
    int *next = a.meta + m_next(c);
    const float *myroi = smem + tid;
    const T inv_s2 = sizeof(T) == 4 ? (T)a.inv_s2 : (T)a.inv_s2_d;
    const T inv_abs_s = sizeof(T) == 4 ? (T)a.inv_abs_s : (T)a.inv_abs_s_d;
    const T w0 = (T)a.w0;

    T th[P], A[NT], v[P], D[P], dx[P], te[P];
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

    auto theta_abs = [&](int k, const T (&t)[P]) -> T {
        return k == IX ? t[k] + (T)xo : (k == IX + 1 ? t[k] + (T)yo : t[k]);
    };
    auto finish = [&](int status) {
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
            const T q = fabs(dx[k]) / tol;
            lastr = q > lastr ? q : lastr;
        }
        o[SL::MINPIV] = minpiv_fit;
        o[SL::LASTR] = lastr;
        o[SL::NESC] = (T)esc_fit;
        o[SL::MARGIN] = margin_fit;
        st[ST_FITS] += 1;
        st[ST_ITERS] += iterations;
        phase = 0;
    };
    auto test_delta = [&]() -> bool {
        bool ok = true;
        T worst = T(0);
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const T tol = (T)a.epsabs + (T)a.epsrel * fabs(theta_abs(k, th));
            ok = ok && (fabs(dx[k]) < tol);
            const T q = fabs(dx[k]) / tol;
            worst = q > worst ? q : worst;
        }
        margin_fit = fmin(margin_fit, fabs(worst - T(1)));
        return ok;
    };
    auto start_iteration = [&]() {
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

    while (true) {
        // ---- refill idle lanes from the class queue ----
        const bool want = (phase == 0) && !exhausted;
        const unsigned need = __ballot_sync(kFull, want);
        if (need) {
            const int leader = __ffs(need) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(next, __popc(need));
            base = __shfl_sync(kFull, base, leader);
            int my = -1;
            if (want) {
                const int q = base + __popc(need & ((1u << lane) - 1));
                if (q < ccount) my = a.order[cstart + q];
                else exhausted = true;
            }
            int fr = 0;
            if (my >= 0) {
                const Cand cd = a.cands[my];
                xo = (int)floor(cd.x - (double)r);
                yo = (int)floor(cd.y - (double)r);
                fr = cd.frame;
                cidx = my;
                minpiv_fit = T(1);
                margin_fit = T(1e30);
                esc_fit = 0;
                if (a.init_params) {
                    const float *ip = a.init_params + (size_t)my * P;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const double off = k == IX ? (double)xo : (k == IX + 1 ? (double)yo : 0.0);
                        th[k] = (T)((double)ip[k] - off);
                    }
                } else {
                    const T xl = (T)(cd.x - (double)xo), yl = (T)(cd.y - (double)yo);
                    if constexpr (METHOD == 0) {
                        th[0] = (T)cd.intensity; th[1] = w0; th[2] = xl; th[3] = yl; th[4] = (T)cd.background;
                    } else if constexpr (METHOD == 1) {
                        th[0] = (T)cd.intensity; th[1] = xl; th[2] = yl; th[3] = (T)cd.background;
                    } else {
                        th[0] = (T)cd.intensity; th[1] = w0; th[2] = w0; th[3] = xl; th[4] = yl;
                        th[5] = T(0); th[6] = (T)cd.background;
                    }
                }
                phase = 1;
            }
            // warp-cooperative ROI staging: global uint16 -> shared float
            unsigned got = __ballot_sync(kFull, my >= 0);
            while (got) {
                const int src = __ffs(got) - 1;
                got &= got - 1;
                const int sxo = __shfl_sync(kFull, xo, src);
                const int syo = __shfl_sync(kFull, yo, src);
                const int sfr = __shfl_sync(kFull, fr, src);
                const uint16_t *fb = a.frames + (size_t)sfr * (size_t)a.frame_px + sxo + (size_t)syo * a.n_rows;
                float *dst = smem + wbase + src;
                for (int k = lane; k < npx; k += 32) {
                    const int j = k / s, i = k - j * s;
                    dst[k * ld] = (float)__ldg(fb + i + (size_t)j * a.n_rows);
                }
            }
            __syncwarp();
        }
        if (__ballot_sync(kFull, phase != 0) == 0) break;

        // ---- choose this lane's evaluation point ----
        bool do_pass = false;
        if (phase == 1) {
#pragma unroll
            for (int k = 0; k < P; ++k) te[k] = th[k];
            do_pass = true;
        } else if (phase == 2) {
            ++trial;
            T invD[P], g[P], Ms[NT], z[P];
#pragma unroll
            for (int k = 0; k < P; ++k) {
                invD[k] = T(1) / D[k];
                g[k] = v[k] * invD[k];
            }
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = i; j < P; ++j) Ms[pku(P, i, j)] = A[pku(P, i, j)] * invD[i] * invD[j];
            unsigned nl = 0, ne = 0;
            bool sing = false;
            T npiv;
            lmpar_scaled<P, T>(Ms, g, delta, par, z, a.pivot_thr, nl, ne, sing, npiv, margin_fit);
            st[ST_LAMBDA] += nl;
            st[ST_ESC] += ne;
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
                pnorm = sqrt(pn2);
                if (it_state == 1 && pnorm < delta) delta = pnorm;
                T q = T(0);
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    T row = T(0);
#pragma unroll
                    for (int j = 0; j < P; ++j) row += Ms[i <= j ? pku(P, i, j) : pku(P, j, i)] * z[j];
                    q += z[i] * row;
                }
                jdx2 = q;
                const bool bad = (METHOD == 0 && te[1] == T(0)) || (METHOD == 7 && (te[1] == T(0) || te[2] == T(0)));
                if (bad) finish(T_EBADFUNC);
                else do_pass = true;
            }
        }

        // ---- the pass: model, Jacobian and normal equations at te ----
        T acc[NT - 1], vv[P], chi2, dchi, dqmax;
        if (do_pass) {
            T dt[P];
#pragma unroll
            for (int k = 0; k < P; ++k) dt[k] = phase == 2 ? dx[k] : T(0);
            Pass<METHOD, S, T>::run(myroi, ld, s, w0, te, dt, acc, vv, chi2, dchi, dqmax);
            if (phase == 1) {
                st[ST_J] += 1;
                st[ST_PIXJ] += npx;
            } else {
                st[ST_F] += 1;
                st[ST_PIXF] += npx;
            }
        }

        // ---- decide ----
        if (do_pass) {
            const T fn1 = sqrt(chi2) * inv_abs_s;
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
                start_iteration();
            } else {
                T actred = T(-1);
                if (T(0.1) * fn1 < fnorm) {
                    if (dqmax < T(0.25)) {
                        // accurate |f|^2 change from the per-pixel model differences
                        actred = -(dchi * inv_s2) / (fnorm * fnorm);
                    } else {
                        const T u = fn1 / fnorm;
                        actred = T(1) - u * u;
                    }
                }
                const T if2 = T(1) / (fnorm * fnorm);
                const T t1s = jdx2 * if2;
                const T t2s = par * pnorm * pnorm * if2;
                const T prered = t1s + T(2) * t2s;
                const T dirder = -(t1s + t2s);
                const T ratio = prered > T(0) ? actred / prered : T(0);
                margin_fit = fmin(margin_fit, fmin(fabs(ratio - T(0.25)), fmin(fabs(ratio - T(0.75)),
                                                                              fabs(ratio - T(1e-4)))));
                if (ratio > T(0.25)) {
                    if (par == T(0) || ratio >= T(0.75)) {
                        delta = pnorm / T(0.5);
                        par *= T(0.5);
                    }
                } else {
                    T temp = (actred >= T(0)) ? T(0.5) : T(0.5) * dirder / (dirder + T(0.5) * actred);
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
                    st[ST_J] += 1;  // the accepted trial's Jacobian
                    st[ST_PIXJ] += npx;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const T cn = sqrt(A[pku(P, k, k)]);
                        const T cnn = cn == T(0) ? T(1) : cn;
                        if (cnn > D[k]) D[k] = cnn;
                    }
                    if (test_delta()) finish(T_CONVERGED);
                    else if (iterations >= a.max_iter) finish(T_MAX_ITER);
                    else start_iteration();
                } else {
                    T gmax = T(0);
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const T gk = fabs(v[k] / D[k]);
                        if (gk > gmax) gmax = gk;
                    }
                    const T gnorm = gmax / fnorm;
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
    }
}

template <int METHOD, typename T>
__global__ void __launch_bounds__(128) k1_lm_fit(K1Args a)
{
    extern __shared__ float smem[];
    unsigned st[ST_N];
#pragma unroll
    for (int k = 0; k < ST_N; ++k) st[k] = 0;
    const int ncls = a.meta[M_NCLS];
    for (int c = 0; c < ncls; ++c) {
        const int s = a.meta[m_side(c)];
        if constexpr (sizeof(T) == 8) {
            run_class<METHOD, T, 0>(a, c, smem, st);
            continue;
        } else {
        switch (s) {
        case 5: run_class<METHOD, T, 5>(a, c, smem, st); break;
        case 7: run_class<METHOD, T, 7>(a, c, smem, st); break;
        case 9: run_class<METHOD, T, 9>(a, c, smem, st); break;
        case 11: run_class<METHOD, T, 11>(a, c, smem, st); break;
        case 13: run_class<METHOD, T, 13>(a, c, smem, st); break;
        case 15: run_class<METHOD, T, 15>(a, c, smem, st); break;
        case 17: run_class<METHOD, T, 17>(a, c, smem, st); break;
        default: run_class<METHOD, T, 0>(a, c, smem, st); break;
        }
        }
    }
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
    const void *state;
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

template <int METHOD, typename ST>
__global__ void k2_finalize(K2Args a)
{
    constexpr int P = Traits<METHOD == 5 ? 7 : METHOD>::P;
    constexpr int NT = tri(P);
    using SL = StateLayout<P>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    if (a.flags[i] != F_PENDING) return;
    const Cand cd = a.cands[i];
    const ST *s = (const ST *)a.state + (size_t)i * a.state_stride;
    const int iterations = (int)s[SL::ITERS];
    const int status = (int)s[SL::STATUS];
    const int xo = (int)s[SL::XOFF], yo = (int)s[SL::YOFF];
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
    for (int k = 0; k < P; ++k) x[k] = (double)s[k];
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
        dg[0] = (float)s[SL::MINPIV];
        dg[1] = (float)s[SL::LASTR];
        dg[2] = (float)s[SL::NESC];
        dg[3] = (float)s[SL::MARGIN];
        dg[4] = 0.0f;
        dg[5] = (float)iterations;
        dg[6] = (float)status;
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
    for (int k = 0; k < NT; ++k) A[k] = (double)s[P + k];
    const double chi = (double)s[SL::FNORM];
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

template <int METHOD, typename T>
cudaError_t launch_k1(const K1Args &ka, int tpb, int bps_req, int smem, cudaStream_t stream)
{
    auto kern = k1_lm_fit<METHOD, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, bps = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, tpb, smem);
    if (e != cudaSuccess) return e;
    if (bps < 1) return cudaErrorInvalidConfiguration;
    if (bps_req > 0 && bps_req < bps) bps = bps_req;
    kern<<<nsm * bps, tpb, smem, stream>>>(ka);
    return cudaGetLastError();
}

}  // namespace

int state_stride(int method)
{
    const int m = solver_method(method);
    return m == 0 ? StateLayout<5>::STRIDE : m == 1 ? StateLayout<4>::STRIDE : StateLayout<7>::STRIDE;
}

size_t scratch_bytes(int method, int n, int precision)
{
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t el = precision == 1 ? sizeof(double) : sizeof(float);
    return al(sizeof(int) * (size_t)n) * 2 + al(sizeof(int) * kMetaInts) +
           al(el * (size_t)n * state_stride(method)) + al(sizeof(unsigned long long) * ST_N);
}

void carve_scratch(void *base, int method, int n, Scratch *s)
{
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    char *p = (char *)base;
    s->cls = (int *)p;
    p += al(sizeof(int) * (size_t)n);
    s->order = (int *)p;
    p += al(sizeof(int) * (size_t)n);
    s->meta = (int *)p;
    p += al(sizeof(int) * kMetaInts);
    s->stats = (unsigned long long *)p;
    p += al(sizeof(unsigned long long) * ST_N);
    s->state = (void *)p;
}

cudaError_t enqueue_fit(const FitParams &p, const Scratch &s, cudaStream_t stream, int *err_detail)
{
    *err_detail = 0;
    const int n = p.n_cands;
    const int ncol_total = ref_cols(p.method) + 2;
    const int r_default = (int)std::ceil(p.w0 * 4.0);
    cudaError_t e;
    e = cudaMemsetAsync(s.meta, 0, sizeof(int) * kMetaInts, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s.stats, 0, sizeof(unsigned long long) * ST_N, stream);
    if (e != cudaSuccess) return e;
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
    mark(0);
    K0Args k0{(const Cand *)p.cands, n, p.n_frames, p.n_rows, p.n_cols, r_default, r_cap, p.method, ncol_total,
              p.out, p.flags, s.cls, s.meta};
    const int nb = (n + 255) / 256;
    k0_classify<<<nb, 256, 0, stream>>>(k0);
    k0_classes<<<1, 32, 0, stream>>>(s.meta);
    k0_scatter<<<nb, 256, 0, stream>>>(s.cls, n, s.meta, s.order);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    int maxr = p.max_half_width;
    if (maxr <= 0) {
        // the solver's shared memory is sized by the largest ROI present
        int mr = 0;
        e = cudaMemcpyAsync(&mr, s.meta + M_MAXR, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return e;
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        maxr = mr;
    }
    if (maxr > r_cap) maxr = r_cap;
    mark(1);
    if (maxr >= 1) {
        const int side = 2 * maxr + 1;
        int tpb = p.threads_per_block > 0 ? p.threads_per_block : 128;
        tpb = (tpb + 31) / 32 * 32;
        if (tpb > 128) tpb = 128;
        // shrink the block until the per-lane ROIs fit the 227 KB shared memory limit
        while (tpb > 32 && (size_t)tpb * side * side * sizeof(float) > 227u * 1024u) tpb -= 32;
        const size_t smem = (size_t)tpb * side * side * sizeof(float);
        if (smem > 227u * 1024u) {
            *err_detail = 1;
            return cudaErrorInvalidValue;
        }
        const double s_abs = std::fabs(p.sigma);
        K1Args k1{p.frames, (long long)p.n_rows * p.n_cols, p.n_rows, (const Cand *)p.cands, s.order, s.meta,
                  s.state, state_stride(p.method), (float)p.w0, (float)(1.0 / (p.sigma * p.sigma)),
                  (float)(1.0 / s_abs), 1.0 / (p.sigma * p.sigma), 1.0 / s_abs, p.max_iter, (float)p.epsabs,
                  (float)p.epsrel, p.precision == 1 ? 0.0f : p.pivot_thr, p.init_params, s.stats};
        const int m = solver_method(p.method);
        if (p.precision == 1) {
            e = m == 0 ? launch_k1<0, double>(k1, tpb, p.blocks_per_sm, (int)smem, stream)
              : m == 1 ? launch_k1<1, double>(k1, tpb, p.blocks_per_sm, (int)smem, stream)
                       : launch_k1<7, double>(k1, tpb, p.blocks_per_sm, (int)smem, stream);
        } else {
            e = m == 0 ? launch_k1<0, float>(k1, tpb, p.blocks_per_sm, (int)smem, stream)
              : m == 1 ? launch_k1<1, float>(k1, tpb, p.blocks_per_sm, (int)smem, stream)
                       : launch_k1<7, float>(k1, tpb, p.blocks_per_sm, (int)smem, stream);
        }
        if (e != cudaSuccess) return e;
    }
    mark(2);
    K2Args k2{(const Cand *)p.cands, n, p.method, p.w0, r_default, s.state, state_stride(p.method), ncol_total,
              p.out, p.flags, p.params_out, p.diag};
    if (p.precision == 1) {
        switch (p.method) {
        case 0: k2_finalize<0, double><<<nb, 256, 0, stream>>>(k2); break;
        case 1: k2_finalize<1, double><<<nb, 256, 0, stream>>>(k2); break;
        case 5: k2_finalize<5, double><<<nb, 256, 0, stream>>>(k2); break;
        default: k2_finalize<7, double><<<nb, 256, 0, stream>>>(k2); break;
        }
    } else {
        switch (p.method) {
        case 0: k2_finalize<0, float><<<nb, 256, 0, stream>>>(k2); break;
        case 1: k2_finalize<1, float><<<nb, 256, 0, stream>>>(k2); break;
        case 5: k2_finalize<5, float><<<nb, 256, 0, stream>>>(k2); break;
        default: k2_finalize<7, float><<<nb, 256, 0, stream>>>(k2); break;
        }
    }
    mark(3);
    return cudaGetLastError();
}

}  // namespace locb
