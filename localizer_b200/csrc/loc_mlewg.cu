// MLEwG fits on the GPU: maximum-likelihood Gaussian localization with a
// Nelder-Mead simplex (reference FitPositions_MLEwG::fit_positions,
// source/Localization.cpp:633-789; objective MinimizationFunction_MLEwG
// :1333-1362, position deviation CalculateMLEwGVariance :1364-1374).
//
// One thread per candidate, in FP64 and in the reference's operation order:
// this file is compiled without fused multiply-add contraction, the objective
// sums the pixels row by row as the reference does, and the simplex follows
// the same restated minimiser as the CPU oracle (GSL nmsimplex2: reflect,
// expand by 2, contract by 0.5, shrink to the best corner; centre and squared
// size updated incrementally; BLAS-style norm, dot and axpy). Start: centre at
// the candidate, width w0, background from the candidate, integral
// 2 pi w0^2 x intensity, unit steps; stop when the simplex size falls below
// 1e-2 or after 200 iterations. Rejects, in the reference's order: integral
// <= 0, centre outside the ROI, centre moved by more than 2 w0, integral
// outside [1/2, 3/2] of the start, width outside [1/2, 3/2] w0.
#include "../../include/localizer_b200.h"
#include "loc_fit.cuh"

#include <cuda_runtime.h>
#include <math_constants.h>

#include <cmath>
#include <cstdint>

namespace locb {

namespace {

constexpr int N = 5, NP = 6;
constexpr double kPi = 3.1415926535897932384626433;   // the reference's PI (Defines.h:97)

struct MlCand {
    double x, y, intensity, background;
    int32_t frame, half_width;
};

struct Roi {
    const uint16_t *base;  // pixel (0, 0) of the ROI
    int n_rows;            // frame row stride
    int s;                 // ROI side
    double xoff, yoff;
};

__device__ double objective(const double *p, const Roi &roi)
{
    const double x0 = p[0], y0 = p[1], sd = p[2], bg = p[3], nph = p[4];
    double sum = 0.0;
    for (int j = 0; j < roi.s; ++j) {
        const uint16_t *row = roi.base + (size_t)j * roi.n_rows;
        for (int i = 0; i < roi.s; ++i) {
            const double x = roi.xoff + (double)i, y = roi.yoff + (double)j;
            const double d = (double)row[i];
            const double e = nph / (2 * kPi * sd * sd) * exp(-((x - x0) * (x - x0) + (y - y0) * (y - y0)) / sd / sd) + bg;
            if (d >= 0.0) sum += -e + d * log(e) - lgamma(d + 1.0);
        }
    }
    return -1.0 * sum;
}

__device__ double dnrm2(const double *x)
{
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < N; i++) {
        if (x[i] != 0.0) {
            const double ax = fabs(x[i]);
            if (scale < ax) {
                ssq = 1.0 + ssq * (scale / ax) * (scale / ax);
                scale = ax;
            } else {
                ssq += (ax / scale) * (ax / scale);
            }
        }
    }
    return scale * sqrt(ssq);
}

struct Simplex {
    double x1[NP * N];
    double y1[NP];
    double center[N];
    double S2;
};

__device__ void compute_center(Simplex &s)
{
    for (int j = 0; j < N; j++) s.center[j] = 0.0;
    for (int i = 0; i < NP; i++)
        for (int j = 0; j < N; j++) s.center[j] += 1.0 * s.x1[i * N + j];
    const double a = 1.0 / NP;
    for (int j = 0; j < N; j++) s.center[j] *= a;
}

__device__ double compute_size(Simplex &s)
{
    double ss = 0.0, w[N];
    for (int i = 0; i < NP; i++) {
        for (int j = 0; j < N; j++) w[j] = s.x1[i * N + j];
        for (int j = 0; j < N; j++) w[j] += -1.0 * s.center[j];
        const double t = dnrm2(w);
        ss += t * t;
    }
    s.S2 = ss / NP;
    return sqrt(ss / NP);
}

__device__ double try_corner(double coeff, const Simplex &s, int corner, double *xc, const Roi &roi)
{
    const double alpha = (1 - coeff) * NP / (NP - 1.0);
    const double beta = (NP * coeff - 1.0) / (NP - 1.0);
    for (int j = 0; j < N; j++) xc[j] = s.center[j] * alpha;
    for (int j = 0; j < N; j++) xc[j] += beta * s.x1[corner * N + j];
    return objective(xc, roi);
}

__device__ void update_point(Simplex &s, int i, const double *x, double val)
{
    double delta[N], xmc[N];
    const double *xo = s.x1 + i * N;
    for (int j = 0; j < N; j++) delta[j] = x[j];
    for (int j = 0; j < N; j++) delta[j] += -1.0 * xo[j];
    for (int j = 0; j < N; j++) xmc[j] = xo[j];
    for (int j = 0; j < N; j++) xmc[j] += -1.0 * s.center[j];
    const double d = dnrm2(delta);
    double xmcd = 0.0;
    for (int j = 0; j < N; j++) xmcd += xmc[j] * delta[j];
    s.S2 += (2.0 / NP) * xmcd + ((NP - 1.0) / NP) * (d * d / NP);
    const double a = 1.0 / NP;
    for (int j = 0; j < N; j++) s.center[j] += -a * xo[j];
    for (int j = 0; j < N; j++) s.center[j] += a * x[j];
    for (int j = 0; j < N; j++) s.x1[i * N + j] = x[j];
    s.y1[i] = val;
}

// 0 ok, 5 failed contraction (non-finite values)
__device__ int nm_iterate(Simplex &s, const Roi &roi, double *x, double &size)
{
    double xc[N], xc2[N];
    int hi = 0, lo = 0, s_hi = 1;
    double dhi = s.y1[0], dlo = s.y1[0], ds_hi = s.y1[1];
    for (int i = 1; i < NP; i++) {
        const double v = s.y1[i];
        if (v < dlo) {
            dlo = v;
            lo = i;
        } else if (v > dhi) {
            ds_hi = dhi;
            s_hi = hi;
            dhi = v;
            hi = i;
        } else if (v > ds_hi) {
            ds_hi = v;
            s_hi = i;
        }
    }
    const double val = try_corner(-1.0, s, hi, xc, roi);
    if (isfinite(val) && val < s.y1[lo]) {
        const double val2 = try_corner(-2.0, s, hi, xc2, roi);
        if (isfinite(val2) && val2 < s.y1[lo]) update_point(s, hi, xc2, val2);
        else update_point(s, hi, xc, val);
    } else if (!isfinite(val) || val > s.y1[s_hi]) {
        if (isfinite(val) && val <= s.y1[hi]) update_point(s, hi, xc, val);
        const double val2 = try_corner(0.5, s, hi, xc2, roi);
        if (isfinite(val2) && val2 <= s.y1[hi]) {
            update_point(s, hi, xc2, val2);
        } else {
            bool bad = false;
            for (int i = 0; i < NP; i++) {
                if (i == lo) continue;
                for (int j = 0; j < N; j++) s.x1[i * N + j] = 0.5 * (s.x1[i * N + j] + s.x1[lo * N + j]);
                const double v = objective(s.x1 + i * N, roi);
                s.y1[i] = v;
                if (!isfinite(v)) bad = true;
            }
            compute_center(s);
            compute_size(s);
            if (bad) return 5;
        }
    } else {
        // better than the second-worst corner: replace the worst by the reflection
        update_point(s, hi, xc, val);
    }
    lo = 0;
    for (int i = 1; i < NP; i++)
        if (s.y1[i] < s.y1[lo]) lo = i;
    for (int j = 0; j < N; j++) x[j] = s.x1[lo * N + j];
    size = s.S2 > 0 ? sqrt(s.S2) : compute_size(s);
    return 0;
}

struct MlArgs {
    const uint16_t *frames;
    int n_frames, n_rows, n_cols;
    const MlCand *cands;
    int n;
    double w0;
    int r_default, r_cap;
    double *out;      // n x 10
    uint8_t *flags;
    float *params_out;
    unsigned long long *stats;
};

__global__ void __launch_bounds__(64) k_mlewg(MlArgs a)
{
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= a.n) return;
    constexpr int ncol = 10;
    double *row = a.out + (size_t)ci * ncol;
    const MlCand c = a.cands[ci];
    auto reject = [&](uint8_t flag) {
        row[0] = (double)c.frame;
        for (int k = 1; k < ncol - 2; ++k) row[k] = CUDART_NAN;
        a.flags[ci] = flag;
    };
    row[ncol - 2] = 0.0;
    row[ncol - 1] = 0.0;
    const bool finite = isfinite(c.x) && isfinite(c.y) && isfinite(c.intensity) && isfinite(c.background);
    const int r = c.half_width > 0 ? c.half_width : a.r_default;
    if (!finite || c.frame < 0 || c.frame >= a.n_frames || c.half_width < 0 || r < 1 || r > a.r_cap) {
        reject(10);
        return;
    }
    const int s = 2 * r + 1;
    // Localization.cpp:694-704
    const int xo = (int)floor(c.x - (double)r), yo = (int)floor(c.y - (double)r);
    const int xm = xo + s - 1, ym = yo + s - 1;
    if (xo < 0 || xm > a.n_rows - 1 || yo < 0 || ym > a.n_cols - 1) {
        reject(1);
        return;
    }
    Roi roi{a.frames + (size_t)c.frame * a.n_rows * a.n_cols + xo + (size_t)yo * a.n_rows, a.n_rows, s, (double)xo,
            (double)yo};
    const double integral = c.intensity * 2.0 * CUDART_PI * a.w0 * a.w0;
    double x[N] = {c.x, c.y, a.w0, c.background, integral};
    // set: corner 0 at the start, corner i+1 one unit further along axis i
    Simplex sp;
    int status = 0;
    double v = objective(x, roi);
    if (!isfinite(v)) status = 9;
    for (int j = 0; j < N; j++) sp.x1[j] = x[j];
    sp.y1[0] = v;
    for (int i = 0; i < N && status == 0; i++) {
        double t[N];
        for (int j = 0; j < N; j++) t[j] = x[j];
        t[i] = x[i] + 1.0;
        v = objective(t, roi);
        if (!isfinite(v)) status = 9;
        for (int j = 0; j < N; j++) sp.x1[(i + 1) * N + j] = t[j];
        sp.y1[i + 1] = v;
    }
    long iterations = 0;
    if (status == 0) {
        compute_center(sp);
        double size = compute_size(sp);
        int test = 1;
        do {
            iterations++;
            const int st = nm_iterate(sp, roi, x, size);
            if (st != 0) {
                status = st;
                break;
            }
            test = size < 1e-2 ? 0 : 1;
        } while (test == 1 && iterations < 200);
        if (status == 0) status = test;   // 0 converged, 1 iteration cap
    }
    if (a.stats) {
        atomicAdd(&a.stats[4], 1ull);
        atomicAdd(&a.stats[5], (unsigned long long)iterations);
    }
    row[ncol - 2] = (double)iterations;
    row[ncol - 1] = (double)status;
    if (a.params_out)
        for (int k = 0; k < N; ++k) a.params_out[(size_t)ci * N + k] = (float)x[k];
    if (status == 9) {   // non-finite objective at the start: the simplex was never set up
        reject(10);
        return;
    }
    // Localization.cpp:739-768
    if (x[4] <= 0) {
        reject(2);
        return;
    }
    if (x[0] < xo || x[0] > xm || x[1] < yo || x[1] > ym) {
        reject(3);
        return;
    }
    if (fabs(x[0] - c.x) > 2.0 * a.w0 || fabs(x[1] - c.y) > 2.0 * a.w0) {
        reject(5);
        return;
    }
    if (x[4] < integral / 2.0 || x[4] > integral * 1.5) {
        reject(11);
        return;
    }
    if (x[2] < a.w0 / 2.0 || x[2] > a.w0 * 1.5) {
        reject(4);
        return;
    }
    // CalculateMLEwGVariance (Localization.cpp:1364-1374)
    const double sigmaA = a.w0 * a.w0 + 1.0 / 12.0;
    const double var = sigmaA * sigmaA / x[4] * (16.0 / 9.0 + 8 * CUDART_PI * a.w0 * a.w0 * x[3] / x[4]);
    row[0] = (double)c.frame;
    row[1] = x[4];
    row[2] = x[2];
    row[3] = x[0];
    row[4] = x[1];
    row[5] = x[3];
    row[6] = sqrt(var);
    row[7] = 1.0;
    a.flags[ci] = 0;
}

}  // namespace

cudaError_t enqueue_mlewg(const FitParams &p, unsigned long long *stats, cudaStream_t stream)
{
    if (p.n_cands == 0) return cudaSuccess;
    MlArgs a{p.frames, p.n_frames, p.n_rows, p.n_cols, static_cast<const MlCand *>(p.cands), p.n_cands, p.w0,
             (int)std::ceil(p.w0 * 4.0),
             p.max_half_width > 0 ? (p.max_half_width < kMaxHalfWidth ? p.max_half_width : kMaxHalfWidth)
                                  : kMaxHalfWidth,
             p.out, p.flags, p.params_out, stats};
    k_mlewg<<<(p.n_cands + 63) / 64, 64, 0, stream>>>(a);
    if (p.launches) ++*p.launches;
    return cudaGetLastError();
}

}  // namespace locb
