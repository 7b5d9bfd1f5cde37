// Device building blocks of the B200 Levenberg-Marquardt fit engine.
//
// One CUDA thread owns one emitter fit ("lane"); a warp advances 32 fits in
// lock step, one model evaluation pass per loop trip. The iteration is the
// scaled trust-region Levenberg-Marquardt method that the reference runs
// through GSL's lmsder (source/Localization.cpp:145-155; GSL 1.16, MINPACK
// lmder/lmpar of More 1978), restated on the normal equations: every pass
// accumulates J^T J, J^T f and |f|^2 of the ROI, and the damped step
// (J^T J + par D^2) p = -J^T f of MINPACK's lmpar is solved by an in-register
// Cholesky factorisation of the D-scaled matrix. In exact arithmetic this
// is the same sequence of steps, trust radii and Levenberg parameters as the
// QR-based lmsder; FP32 pivots that fall below a conditioning threshold are
// refactorised in FP64.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace locb {

struct Cand {
    double x, y, intensity, background;
    int32_t frame;
    int32_t half_width;
};
static_assert(sizeof(Cand) == 40, "candidate layout");


// Parameter vectors per method (reference Localization.cpp:138-142, 318-321,
// 485-491): symmetric (A, s, x0, y0, b); fixed width (A, x0, y0, b);
// ellipsoidal (A, sx, sy, x0, y0, rho, b). IX = index of x0.
template <int METHOD> struct Traits;
template <> struct Traits<0> { static constexpr int P = 5; static constexpr int IX = 2; };
template <> struct Traits<1> { static constexpr int P = 4; static constexpr int IX = 1; };
template <> struct Traits<7> { static constexpr int P = 7; static constexpr int IX = 3; };

__host__ __device__ constexpr int tri(int P) { return P * (P + 1) / 2; }
// packed upper triangle (row-major, i <= j)
__host__ __device__ constexpr int pku(int P, int i, int j) { return i * P - i * (i - 1) / 2 + (j - i); }
// packed lower triangle (row-major, j <= i)
__host__ __device__ constexpr int pkl(int i, int j) { return i * (i + 1) / 2 + j; }

// Per-candidate fit state handed from the solver kernel to the finaliser, in
// the solver's precision: [0,P) parameters (ROI-local positions), [P, P+NT)
// scaled J^T J, then fnorm, iterations, status, x_off, y_off (small integers,
// exact in either precision).
template <int P> struct StateLayout {
    static constexpr int NT = tri(P);
    static constexpr int FNORM = P + NT;
    static constexpr int ITERS = FNORM + 1;
    static constexpr int STATUS = FNORM + 2;
    static constexpr int XOFF = FNORM + 3;
    static constexpr int YOFF = FNORM + 4;
    static constexpr int MINPIV = FNORM + 5;   // smallest undamped pivot ratio over the fit
    static constexpr int LASTR = FNORM + 6;    // last step / test_delta tolerance (max over parameters)
    static constexpr int NESC = FNORM + 7;     // FP64 pivot escalations in the fit
    static constexpr int MARGIN = FNORM + 8;   // smallest relative distance of a branch decision to its threshold
    static constexpr int STRIDE = ((FNORM + 9) + 3) / 4 * 4;
};

// Reject codes and termination codes (public header LOC_FLAG_*, LOC_TERM_*).
enum : uint8_t {
    F_KEPT = 0, F_EDGE = 1, F_AMPLITUDE = 2, F_WINDOW = 3, F_WIDTH = 4, F_DRIFT = 5,
    F_EIGEN = 6, F_NO_AXIS = 7, F_SYM_RATIO = 8, F_SYM_WIDTH = 9, F_BAD_INPUT = 10,
    F_PENDING = 255
};
enum : int { T_CONVERGED = 0, T_MAX_ITER = 1, T_EBADFUNC = 9, T_ENOPROG = 27, T_ETOLF = 29,
             T_ETOLX = 30, T_ETOLG = 31, T_SINGULAR = 64 };

// stats slots; the last four accumulate SM clock cycles per warp (lane 0)
// spent in each phase of the solver loop
enum { ST_F = 0, ST_J = 1, ST_LAMBDA = 2, ST_ESC = 3, ST_FITS = 4, ST_ITERS = 5, ST_PIXF = 6,
       ST_PIXJ = 7, ST_CYC_REFILL = 8, ST_CYC_STEP = 9, ST_CYC_PASS = 10, ST_CYC_DECIDE = 11, ST_N = 12 };

constexpr double kDblEps = 2.2204460492503131e-16;   // GSL_DBL_EPSILON
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// exp(-c*q) in the precision of T. For float the constant is pre-multiplied
// by log2(e) and the hardware exp2 unit is used; for double, exp().
template <typename T> struct Expo;
template <> struct Expo<float> {
    static constexpr float scale = kLog2e;
    __device__ __forceinline__ static float ex(float a) { return ex2_approx(a); }
};
template <> struct Expo<double> {
    static constexpr double scale = 1.0;
    __device__ __forceinline__ static double ex(double a) { return exp(a); }
};

// Division, reciprocal and square roots of the solver's control path. In
// FP32 they use the hardware approximations (about 2 ulp), which shortens
// the serial dependency chains of the step solve and the accept/reject logic
// (the FP32 path's accuracy is set elsewhere: by the accumulated normal
// equations); the FP64 path keeps correctly rounded operations.
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float frcp(float a) { return __fdividef(1.0f, a); }
__device__ __forceinline__ double frcp(double a) { return 1.0 / a; }
__device__ __forceinline__ float frsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ double frsqrt(double a) { return rsqrt(a); }
__device__ __forceinline__ float fsqrt(float a) { return a > 0.0f ? a * rsqrtf(a) : sqrtf(a); }
__device__ __forceinline__ double fsqrt(double a) { return sqrt(a); }

// Per-fit array in registers, or (InSmem) in a shared-memory slot of the
// fit's group; the FP64 solver keeps its normal equations, state vectors and
// Cholesky factor there so that they are not live in registers.
template <typename T, int N, bool InSmem> struct StateArr;
template <typename T, int N> struct StateArr<T, N, false> {
    T r[N];
    __device__ __forceinline__ explicit StateArr(T *) {}
    __device__ __forceinline__ T &operator[](int k) { return r[k]; }
    __device__ __forceinline__ const T &operator[](int k) const { return r[k]; }
};
template <typename T, int N> struct StateArr<T, N, true> {
    T *p;
    __device__ __forceinline__ explicit StateArr(T *slot) : p(slot) {}
    __device__ __forceinline__ T &operator[](int k) { return p[k]; }
    __device__ __forceinline__ const T &operator[](int k) const { return p[k]; }
};

template <typename T> __device__ __forceinline__ T tiny_pos();
template <> __device__ __forceinline__ float tiny_pos<float>() { return FLT_MIN; }
template <> __device__ __forceinline__ double tiny_pos<double>() { return DBL_MIN; }

// ---------------------------------------------------------------------------
// Model + Jacobian + normal-equation accumulation over one ROI.
//
// roi: the fit's pixels in shared memory, pixel k = i + j*S at roi[k*ld]
// (i along x). With TPF threads per fit, sub-lane q visits the columns
// i = q, q + TPF, ... of every row and the caller sums the partial results
// over the group. Parameters are ROI-local (x0 measured from the ROI origin).
// acc receives the packed upper triangle of J^T J without its last entry
// (the offset column is identically 1, so that entry is the pixel count),
// vv = J^T r and chi2 = |r|^2, with r = model - data (unit noise weight;
// the caller rescales). Expressions follow the reference callbacks:
// symmetric Localization.cpp:1007-1048 / 1128-1181 (width column scaled by
// 1/sqrt(2) as in the reference), fixed width :1050-1076 / 1183-1225,
// ellipsoidal :1078-1126 / 1227-1295 (correlation column as written there).
// ---------------------------------------------------------------------------

template <typename T, typename R>
__device__ __forceinline__ T load_px(const R *roi, int k, int ld);
template <>
__device__ __forceinline__ float load_px<float, float>(const float *roi, int k, int ld) { return roi[k * ld]; }
template <>
__device__ __forceinline__ double load_px<double, float>(const float *roi, int k, int ld) { return (double)roi[k * ld]; }

// Accurate change of |r|^2 between the current point th and the evaluated
// point te = th + dth. The actual-reduction ratio of the trust-region test
// needs fnorm(te)^2 - fnorm(th)^2 to a precision that an FP32 model value
// (~600 photons, 24-bit mantissa) cannot give once steps shrink below about
// 1e-3 px. The pass therefore also forms, per pixel, the model difference
//   delta = m(te) - m(th) = e' (dA - A expm1(q - q')) + db
// from the exponent difference q - q', which is written analytically in the
// parameter step (no cancellation), and accumulates
//   dchi = sum delta (2 r' - delta) = |r(te)|^2 - |r(th)|^2.
// expm1 is a degree-6 series, exact to FP32 for |q - q'| < 0.25 (truncation
// below 5e-8 relative); dqmax reports the largest |q - q'| so the caller can
// fall back to the direct difference for larger steps, whose reduction is
// large enough for FP32 to resolve directly.
template <typename T>
__device__ __forceinline__ T expm1_series(T y)
{
    T p = fma(y, T(1.0 / 720.0), T(1.0 / 120.0));
    p = fma(y, p, T(1.0 / 24.0));
    p = fma(y, p, T(1.0 / 6.0));
    p = fma(y, p, T(0.5));
    p = fma(y, p, T(1));
    return y * p;
}

// S > 0: compile-time ROI side (rows fully unrolled); S == 0: runtime side s_rt.
template <int S, int TPF, typename T>
__device__ __forceinline__ void pass_sym(const float *__restrict__ roi, int ld, int s_rt, int q, const T (&th)[5],
                                         const T (&dth)[5], T (&acc)[14], T (&vv)[5], T &chi2, T &dchi, T &dqmax)
{
    const int s = S > 0 ? S : s_rt;
    const T A = th[0], w = th[1], x0 = th[2], y0 = th[3], b = th[4];
    const T dA = dth[0], dw = dth[1], dxs = dth[2], dys = dth[3], db = dth[4];
    const T A0 = A - dA, w0c = w - dw;                         // current point
    const T w2i = T(1) / (w * w);
    const T c1 = -T(0.5) * w2i * (T)Expo<T>::scale;
    const T ka_x = A * w2i;                                   // dfdx0 = u e A / w^2
    const T ka_r = ka_x / (w * T(1.4142135623730950488));      // dfdr = d2 e A / (sqrt2 w^3)
    // exponent q = -c d2, c = 1/(2 w^2); q' - q = -(d2' (c' - c) + c (d2' - d2))
    const T cc = T(0.5) / (w0c * w0c);
    const T cpr = T(0.5) * w2i;
    const T dc = -T(2) * dw * (T(2) * w0c + dw) * cc * cpr;   // c' - c
    const T m2dx = -T(2) * dxs;
#pragma unroll
    for (int k = 0; k < 14; ++k) acc[k] = T(0);
#pragma unroll
    for (int k = 0; k < 5; ++k) vv[k] = T(0);
    chi2 = T(0);
    dchi = T(0);
    dqmax = T(0);
    auto body = [&](int i, T wy, T wy2, T krow, const float *row) {
        const T u = (T)i - x0;
        const T d2 = fma(u, u, wy2);
        const T e = Expo<T>::ex(d2 * c1);
        const T dat = load_px<T, float>(row, i, ld);
        const T r = fma(A, e, b - dat);
        // accurate |r|^2 change
        const T dd = fma(m2dx, u, krow);                      // d2' - d2
        const T ydq = fma(d2, dc, cc * dd);                   // q - q'
        dqmax = fmax(dqmax, fabs(ydq));
        const T del = fma(e, fma(-A0, expm1_series(ydq), dA), db);
        dchi = fma(del, fma(T(2), r, -del), dchi);
        // Jacobian and normal equations at the evaluated point
        const T jr = d2 * (e * ka_r);
        const T ex = e * ka_x;
        const T jx = u * ex, jy = wy * ex;
        acc[0] = fma(e, e, acc[0]);   acc[1] = fma(e, jr, acc[1]);   acc[2] = fma(e, jx, acc[2]);
        acc[3] = fma(e, jy, acc[3]);  acc[4] += e;
        acc[5] = fma(jr, jr, acc[5]); acc[6] = fma(jr, jx, acc[6]); acc[7] = fma(jr, jy, acc[7]);
        acc[8] += jr;
        acc[9] = fma(jx, jx, acc[9]); acc[10] = fma(jx, jy, acc[10]); acc[11] += jx;
        acc[12] = fma(jy, jy, acc[12]); acc[13] += jy;
        vv[0] = fma(e, r, vv[0]); vv[1] = fma(jr, r, vv[1]); vv[2] = fma(jx, r, vv[2]);
        vv[3] = fma(jy, r, vv[3]); vv[4] += r;
        chi2 = fma(r, r, chi2);
    };
    if constexpr (TPF >= 16) {
        // a half or whole warp per fit: the flattened ROI is dealt out over
        // the lanes (row-wise dealing would idle the lanes past a row's end)
#pragma unroll 1
        for (int k = q; k < s * s; k += TPF) {
            const int j = k / s, i = k - j * s;
            const T wy = (T)j - y0;
            body(i, wy, wy * wy, -dxs * dxs - dys * (T(2) * wy + dys), roi + j * s * ld);
        }
    } else {
#pragma unroll 1
    for (int j = 0; j < s; ++j) {
        const T wy = (T)j - y0;
        const T wy2 = wy * wy;
        const T krow = -dxs * dxs - dys * (T(2) * wy + dys);  // (d2' - d2) minus its u term
        const float *row = roi + j * s * ld;
        if (S > 0) {
            // two columns per trip: unrolling all of them made the per-class
            // solver large enough to miss in the instruction cache
#pragma unroll 2
            for (int t = 0; t < (S > 0 ? (S + TPF - 1) / TPF : 1); ++t) {
                const int i = q + TPF * t;
                if (TPF == 1 || i < S) body(i, wy, wy2, krow, row);
            }
        } else {
#pragma unroll 1
            for (int i = q; i < s; i += TPF) body(i, wy, wy2, krow, row);
        }
    }
    }
}

template <int S, int TPF, typename T>
__device__ __forceinline__ void pass_fixed(const float *__restrict__ roi, int ld, int s_rt, int q, T w0,
                                           const T (&th)[4],
                                           const T (&dth)[4], T (&acc)[9], T (&vv)[4], T &chi2, T &dchi, T &dqmax)
{
    const int s = S > 0 ? S : s_rt;
    const T A = th[0], x0 = th[1], y0 = th[2], b = th[3];
    const T dA = dth[0], dxs = dth[1], dys = dth[2], db = dth[3];
    const T A0 = A - dA;
    const T w2i = T(1) / (w0 * w0);
    const T c1 = -T(0.5) * w2i * (T)Expo<T>::scale;
    const T ka_x = A * w2i;
    const T cc = T(0.5) * w2i;
    const T m2dx = -T(2) * dxs;
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = T(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) vv[k] = T(0);
    chi2 = T(0);
    dchi = T(0);
    dqmax = T(0);
    auto body = [&](int i, T wy, T wy2, T krow, const float *row) {
        const T u = (T)i - x0;
        const T d2 = fma(u, u, wy2);
        const T e = Expo<T>::ex(d2 * c1);
        const T dat = load_px<T, float>(row, i, ld);
        const T r = fma(A, e, b - dat);
        const T ydq = cc * fma(m2dx, u, krow);                // q - q' = c (d2' - d2)
        dqmax = fmax(dqmax, fabs(ydq));
        const T del = fma(e, fma(-A0, expm1_series(ydq), dA), db);
        dchi = fma(del, fma(T(2), r, -del), dchi);
        const T ex = e * ka_x;
        const T jx = u * ex, jy = wy * ex;
        acc[0] = fma(e, e, acc[0]); acc[1] = fma(e, jx, acc[1]); acc[2] = fma(e, jy, acc[2]); acc[3] += e;
        acc[4] = fma(jx, jx, acc[4]); acc[5] = fma(jx, jy, acc[5]); acc[6] += jx;
        acc[7] = fma(jy, jy, acc[7]); acc[8] += jy;
        vv[0] = fma(e, r, vv[0]); vv[1] = fma(jx, r, vv[1]); vv[2] = fma(jy, r, vv[2]); vv[3] += r;
        chi2 = fma(r, r, chi2);
    };
    if constexpr (TPF >= 16) {
#pragma unroll 1
        for (int k = q; k < s * s; k += TPF) {
            const int j = k / s, i = k - j * s;
            const T wy = (T)j - y0;
            body(i, wy, wy * wy, -dxs * dxs - dys * (T(2) * wy + dys), roi + j * s * ld);
        }
    } else {
#pragma unroll 1
    for (int j = 0; j < s; ++j) {
        const T wy = (T)j - y0;
        const T wy2 = wy * wy;
        const T krow = -dxs * dxs - dys * (T(2) * wy + dys);
        const float *row = roi + j * s * ld;
        if (S > 0) {
            // two columns per trip: unrolling all of them made the per-class
            // solver large enough to miss in the instruction cache
#pragma unroll 2
            for (int t = 0; t < (S > 0 ? (S + TPF - 1) / TPF : 1); ++t) {
                const int i = q + TPF * t;
                if (TPF == 1 || i < S) body(i, wy, wy2, krow, row);
            }
        } else {
#pragma unroll 1
            for (int i = q; i < s; i += TPF) body(i, wy, wy2, krow, row);
        }
    }
    }
}

template <int S, int TPF, typename T>
__device__ __forceinline__ void pass_ell(const float *__restrict__ roi, int ld, int s_rt, int q, const T (&th)[7],
                                         const T (&dth)[7], T (&acc)[27], T (&vv)[7], T &chi2, T &dchi, T &dqmax)
{
    const int s = S > 0 ? S : s_rt;
    const T A = th[0], sx = th[1], sy = th[2], x0 = th[3], y0 = th[4], rho = th[5], b = th[6];
    const T dA = dth[0], dsx = dth[1], dsy = dth[2], dxs = dth[3], dys = dth[4], drho = dth[5], db = dth[6];
    const T A0 = A - dA, sx0 = sx - dsx, sy0 = sy - dsy, rho0 = rho - drho;
    const T isx = T(1) / sx, isy = T(1) / sy;
    const T a = isx * isx, c = isy * isy, bb = isx * isy;
    const T rb = rho * bb;
    const T k = T(1) / (T(1) - rho * rho);
    const T cexp = -T(0.5) * k * (T)Expo<T>::scale;
    const T AK = A * k;
    const T ABK = AK * bb;
    const T rk = rho * k;
    const T tr = T(2) * rho;
    // current-point coefficients and their exact differences to the evaluated point
    const T isx0 = T(1) / sx0, isy0 = T(1) / sy0;
    const T a0 = isx0 * isx0, c0 = isy0 * isy0, bb0 = isx0 * isy0;
    const T k0 = T(1) / (T(1) - rho0 * rho0);
    const T da = -dsx * (T(2) * sx0 + dsx) * a0 * a;          // a' - a
    const T dcq = -dsy * (T(2) * sy0 + dsy) * c0 * c;         // c' - c
    const T dbb = -(dsx * sy0 + sx * dsy) * bb0 * bb;          // bb' - bb
    const T drb = drho * bb + rho0 * dbb;                      // rb' - rb
    const T dk = drho * (T(2) * rho0 + drho) * k0 * k;         // k' - k
    const T rb0 = rho0 * bb0;
    const T hk = -T(0.5) * k, hdk = -T(0.5) * dk;
    const T dx2 = dxs * dxs;
#pragma unroll
    for (int q = 0; q < 27; ++q) acc[q] = T(0);
#pragma unroll
    for (int q = 0; q < 7; ++q) vv[q] = T(0);
    chi2 = T(0);
    dchi = T(0);
    dqmax = T(0);
    auto body = [&](int i, T wy, T wy2, T wc, T wrb, T brow, T crow, const float *row) {
        const T u = (T)i - x0;
        const T P1 = fma(u, a, -wrb);            // u/sx^2 - rho w/(sx sy)
        const T P2 = fma(-rb, u, wc);            // w/sy^2 - rho u/(sx sy)
        const T q = fma(u, P1, wy * P2);         // the quadratic form Q'
        const T e = Expo<T>::ex(q * cexp);
        const T dat = load_px<T, float>(row, i, ld);
        const T r = fma(A, e, b - dat);
        // q' - q = -(k' Q' - k Q)/2 with Q' - Q a quadratic in u (per-row coefficients)
        const T dQ = fma(fma(da, u, brow), u, crow);
        const T ydq = -fma(hk, dQ, hdk * (q - dQ));           // q - q'
        dqmax = fmax(dqmax, fabs(ydq));
        const T del = fma(e, fma(-A0, expm1_series(ydq), dA), db);
        dchi = fma(del, fma(T(2), r, -del), dchi);
        const T ek = e * AK;
        const T jx = ek * P1, jy = ek * P2;      // dfdx0, dfdy0
        const T jsx = (jx * u) * isx;            // dfdsigmaX
        const T jsy = (jy * wy) * isy;           // dfdsigmaY
        const T uw = u * wy;
        const T d2 = fma(u, u, wy2);
        const T inner = fma(-tr, uw, d2);
        const T t = fma(-rk, inner, uw);
        const T jrho = (e * ABK) * t;            // dfdcorr as in the reference
        const T col[6] = {e, jsx, jsy, jx, jy, jrho};
        int o = 0;
#pragma unroll
        for (int m = 0; m < 6; ++m) {
#pragma unroll
            for (int n = m; n < 6; ++n) acc[o + n - m] = fma(col[m], col[n], acc[o + n - m]);
            acc[o + 6 - m] += col[m];
            o += 7 - m;
        }
#pragma unroll
        for (int m = 0; m < 6; ++m) vv[m] = fma(col[m], r, vv[m]);
        vv[6] += r;
        chi2 = fma(r, r, chi2);
    };
    auto row_terms = [&](int j, T &wy, T &wy2, T &wc, T &wrb, T &brow, T &crow) {
        wy = (T)j - y0;
        wy2 = wy * wy;
        wc = wy * c;
        wrb = wy * rb;
        const T wcur = wy + dys;
        brow = T(2) * (dxs * (da - a) - drb * wy + rb0 * dys);
        crow = (da - a) * dx2 - c * dys * (T(2) * wy + dys) + dcq * wcur * wcur + T(2) * rb0 * dxs * wcur;
    };
    if constexpr (TPF >= 16) {
#pragma unroll 1
        for (int k = q; k < s * s; k += TPF) {
            const int j = k / s, i = k - j * s;
            T wy, wy2, wc, wrb, brow, crow;
            row_terms(j, wy, wy2, wc, wrb, brow, crow);
            body(i, wy, wy2, wc, wrb, brow, crow, roi + j * s * ld);
        }
    } else {
#pragma unroll 1
    for (int j = 0; j < s; ++j) {
        const T wy = (T)j - y0;
        const T wy2 = wy * wy;
        const T wc = wy * c;
        const T wrb = wy * rb;
        // Q' - Q = da u^2 + brow u + crow, u and w at the evaluated point
        const T wcur = wy + dys;
        const T brow = T(2) * (dxs * (da - a) - drb * wy + rb0 * dys);
        const T crow = (da - a) * dx2 - c * dys * (T(2) * wy + dys) + dcq * wcur * wcur +
                       T(2) * rb0 * dxs * wcur;
        const float *row = roi + j * s * ld;
        if (S > 0) {
            // two columns per trip: unrolling all of them made the per-class
            // solver large enough to miss in the instruction cache
#pragma unroll 2
            for (int t = 0; t < (S > 0 ? (S + TPF - 1) / TPF : 1); ++t) {
                const int i = q + TPF * t;
                if (TPF == 1 || i < S) body(i, wy, wy2, wc, wrb, brow, crow, row);
            }
        } else {
#pragma unroll 1
            for (int i = q; i < s; i += TPF) body(i, wy, wy2, wc, wrb, brow, crow, row);
        }
    }
    }
}

// ---------------------------------------------------------------------------
// Damped solve in D-scaled coordinates. With M = D^-1 J^T J D^-1 and
// g = D^-1 J^T f, the lmpar step x (J x ~ f, reference step dx = -x) is
// D x = z with (M + par I) z = g. Returns z, |z| and |L^-1 z|^2 / |z|^2
// (the quantity MINPACK's lmpar forms as |w|^2 through R or S), and the
// smallest pivot ratio d_k / (M_kk + par) met in the factorisation.
// Result codes: 0 ok, 1 an FP32 pivot fell below thr * diagonal (redo in
// FP64), 2 not positive definite (in the precision T).
// ---------------------------------------------------------------------------
// The triangular loops run over 0..P-1 with the bound as a condition
// (same operations, same order): with trip counts that depend on the outer
// index the compiler kept the factor and solve vectors in local memory for
// P = 7.
template <int P, typename T, typename MS, typename MA>
__device__ __forceinline__ int chol_solve(const MA &Ms, MS par, const MS (&g)[P], T thr,
                                          MS (&z)[P], MS &znorm, MS &w2, MS &minpiv, T *lslot = nullptr)
{
    // the all-FP64 solve keeps its factor in the fit's shared-memory slot
    constexpr bool kSm = sizeof(T) == 8 && sizeof(MS) == 8;
    StateArr<T, tri(P), kSm> L(lslot);
    T inv[P];
    // smallest pivot ratio d / djj, kept as a fraction (one division at the
    // end instead of one per pivot: FP64 division is long-latency)
    T mpn = T(1), mpd = T(1);
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const T djj = (T)Ms[pku(P, j, j)] + (T)par;
        T d = djj;
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (k < j) d -= L[pkl(j, k)] * L[pkl(j, k)];
        if (d * mpd < mpn * djj) {
            mpn = d;
            mpd = djj;
        }
        if (!(d > thr * djj)) {
            minpiv = (MS)(mpn / mpd);
            return thr > T(0) ? 1 : 2;
        }
        const T il = frsqrt(d);
        inv[j] = il;
        L[pkl(j, j)] = d * il;
#pragma unroll
        for (int i = 0; i < P; ++i) {
            if (i <= j) continue;
            T sacc = (T)Ms[pku(P, j, i)];
#pragma unroll
            for (int k = 0; k < P; ++k)
                if (k < j) sacc -= L[pkl(i, k)] * L[pkl(j, k)];
            L[pkl(i, j)] = sacc * inv[j];
        }
    }
    minpiv = (MS)(mpn / mpd);
    T y[P];
#pragma unroll
    for (int i = 0; i < P; ++i) {
        T sacc = (T)g[i];
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (k < i) sacc -= L[pkl(i, k)] * y[k];
        y[i] = sacc * inv[i];
    }
    T zz[P];
#pragma unroll
    for (int ii = P - 1; ii >= 0; --ii) {
        T sacc = y[ii];
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (k > ii) sacc -= L[pkl(k, ii)] * zz[k];
        zz[ii] = sacc * inv[ii];
    }
    T n2 = T(0);
#pragma unroll
    for (int i = 0; i < P; ++i) n2 += zz[i] * zz[i];
    const T zn = fsqrt(n2);
    T q2 = T(0);
    if (zn > T(0)) {
        const T izn = frcp(zn);
        T qv[P];
#pragma unroll
        for (int i = 0; i < P; ++i) {
            T sacc = zz[i] * izn;
#pragma unroll
            for (int k = 0; k < P; ++k)
                if (k < i) sacc -= L[pkl(i, k)] * qv[k];
            qv[i] = sacc * inv[i];
            q2 += qv[i] * qv[i];
        }
    }
#pragma unroll
    for (int i = 0; i < P; ++i) z[i] = (MS)zz[i];
    znorm = (MS)zn;
    w2 = (MS)q2;
    return 0;
}

// FP64 refactorisation of an FP32 system whose pivot fell below threshold.
// Kept out of line: it is rare, and inlined its double-precision working set
// would raise the register budget of the whole solver loop.
template <int P>
__device__ __noinline__ int chol_solve_fp64(const float *Ms, float par, const float *g, float *z, float *out)
{
    float msl[tri(P)], gl[P], zl[P];
#pragma unroll
    for (int k = 0; k < tri(P); ++k) msl[k] = Ms[k];
#pragma unroll
    for (int k = 0; k < P; ++k) gl[k] = g[k];
    float zn, w2, mp;
    const int rc = chol_solve<P, double, float>(msl, par, gl, 0.0, zl, zn, w2, mp);
#pragma unroll
    for (int k = 0; k < P; ++k) z[k] = zl[k];
    out[0] = zn;
    out[1] = w2;
    return rc;
}

// One damped solve in working precision T; with ESC (FP32 only), pivots
// below thr * diagonal are refactorised in FP64. ESC is a separate kernel
// instantiation: the out-of-line FP64 call costs the solver loop a stack
// frame and register spills even when it never runs.
template <int P, typename T, bool ESC, typename MA>
__device__ __forceinline__ int damped_solve(const MA &Ms, T par, const T (&g)[P], float thr,
                                            T (&z)[P], T &znorm, T &w2, T &minpiv, unsigned &n_esc,
                                            T *lslot)
{
    // FP64 solves take no pivot threshold (there is no higher precision to
    // escalate to), so only FP32 solves can return 1
    int rc = chol_solve<P, T, T>(Ms, par, g, (ESC && sizeof(T) == 4) ? (T)thr : T(0), z, znorm, w2, minpiv,
                                 lslot);
    if constexpr (ESC && sizeof(T) == 4) {
        if (rc == 1) {
            ++n_esc;
            float msl[tri(P)], gl[P], zl[P], o2[2];
#pragma unroll
            for (int k = 0; k < tri(P); ++k) msl[k] = Ms[k];
#pragma unroll
            for (int k = 0; k < P; ++k) gl[k] = g[k];
            rc = chol_solve_fp64<P>(msl, par, gl, zl, o2);
#pragma unroll
            for (int k = 0; k < P; ++k) z[k] = zl[k];
            znorm = o2[0];
            w2 = o2[1];
        }
    }
    return rc;
}

// MINPACK/GSL lmpar in scaled coordinates (see chol_solve). On return z is
// the accepted scaled step and par the Levenberg parameter it was solved
// with; newton_piv is the smallest pivot ratio of the undamped factorisation
// (a conditioning measure of the scaled normal matrix). A damped system that
// is not positive definite (possible only when rounding has made the
// accumulated J^T J indefinite) raises par until it factorises.
//
// margin receives the smallest distance, relative to delta, between a
// quantity and the threshold of a branch it decided (the Newton acceptance
// fp <= 0.1 delta, the |fp| <= 0.1 delta stop, the fp <= fp_old stop): a
// small margin means a rounding difference could have taken the other branch.
template <int P, typename T, bool ESC, typename MA>
__device__ __forceinline__ void lmpar_scaled(const MA &Ms, const T (&g)[P], T delta, T &par,
                                             T (&z)[P], float thr, unsigned &n_lambda, unsigned &n_esc,
                                             bool &singular, T &newton_piv, T &margin, T *lslot = nullptr)
{
    const T idelta = frcp(delta);
    T dxnorm, w2, mp;
    singular = false;
    // One call site for the damped solve: the first trip is the undamped
    // (Newton) solve, the others the lambda search (an inlined solve per call
    // site would double the solver's code).
    T fp = T(0), par_l = T(0), par_u = T(0), gnorm = T(0), pr = T(0);
    bool first = true;
    int fails = 0, it = 1;
#pragma unroll 1
    for (;;) {
        if (!first && pr == T(0)) {
            const T t = T(0.001) * par_u;
            pr = t > tiny_pos<T>() ? t : tiny_pos<T>();
        }
        ++n_lambda;
        const int rc = damped_solve<P, T, ESC>(Ms, pr, g, thr, z, dxnorm, w2, mp, n_esc, lslot);
        if (first) {
            first = false;
            newton_piv = mp;
            bool rank_def = false;
            if (rc != 0) {  // Newton step undefined: treat as infinitely long, no lower bound
                rank_def = true;
                dxnorm = (T)INFINITY;
                w2 = T(0);
                newton_piv = T(0);
            }
            fp = dxnorm - delta;
            if (!rank_def) margin = fmin(margin, fabs(fp - T(0.1) * delta) * idelta);
            if (!rank_def && fp <= T(0.1) * delta) {
                par = T(0);
                return;
            }
            par_l = (!rank_def && w2 > T(0)) ? fdiv(fp * idelta, w2) : T(0);
            T gn2 = T(0);
#pragma unroll
            for (int i = 0; i < P; ++i) gn2 += g[i] * g[i];
            gnorm = fsqrt(gn2);
            par_u = gnorm * idelta;
            if (par_u == T(0)) par_u = tiny_pos<T>() / (delta < T(0.1) ? delta : T(0.1));
            pr = par;
            if (pr > par_u) pr = par_u;
            else if (pr < par_l) pr = par_l;
            if (pr == T(0)) pr = fdiv(gnorm, dxnorm);
            continue;
        }
        if (rc != 0) {
            // the unit-diagonal scaled matrix plus a larger shift factorises
            if (++fails > 16) {
                singular = true;
                break;
            }
            pr = pr * T(4) > T(1e-6) ? pr * T(4) : T(1e-6);
            continue;
        }
        const T fp_old = fp;
        fp = dxnorm - delta;
        margin = fmin(margin, fabs(fabs(fp) - T(0.1) * delta) * idelta);
        if (fabs(fp) <= T(0.1) * delta) break;
        if (par_l == T(0) && fp_old < T(0)) margin = fmin(margin, fabs(fp - fp_old) * idelta);
        if (par_l == T(0) && fp <= fp_old && fp_old < T(0)) break;
        if (it == 10) break;
        const T par_c = fdiv(fp * idelta, w2);
        if (fp > T(0)) {
            if (pr > par_l) par_l = pr;
        } else if (fp < T(0)) {
            if (pr < par_u) par_u = pr;
        }
        pr = (par_l > pr + par_c) ? par_l : pr + par_c;
        ++it;
    }
    par = pr;
}

}  // namespace locb
