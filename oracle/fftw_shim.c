/*
 * TEST INFRASTRUCTURE ONLY — the subset of the FFTW 3 API that the
 * reference's Convolver.cpp imports (fftw_plan_dft_r2c_2d,
 * fftw_plan_dft_c2r_2d, fftw_execute, fftw_destroy_plan, fftw_malloc,
 * fftw_free; Convolver.cpp:205-256), so that the reference's own GLRT
 * segmentation (Segmentation.cpp:241-430) can be compiled unmodified into
 * oracle/_ref. FFTW itself is not in the reference tree (only its header,
 * include/fftw3.h, is vendored).
 *
 * Semantics follow FFTW's documentation: a 2-D transform of n0 x n1 values in
 * row-major order (n1 fastest); r2c writes the n0 x (n1/2 + 1) non-redundant
 * half of the forward transform (exponent sign -1); c2r takes such a half
 * spectrum, treats it as the half of a Hermitian array, and writes the
 * n0 x n1 real backward transform (sign +1). Neither is normalised.
 *
 * Algorithm: separable 1-D complex transforms, each computed by the
 * iterative radix-2 Cooley-Tukey FFT (bit-reversal permutation, then log2 n
 * butterfly stages) when the length is a power of two, and by the direct
 * O(n^2) DFT sum otherwise. Twiddle factors are cos/sin of 2 pi k / n in
 * double precision. The values agree with FFTW's to rounding (about 1e-15
 * relative), not bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double fftw_complex[2];

struct fftw_plan_s {
    int kind;  /* 0: r2c, 1: c2r */
    int n0, n1;
    double *rin;          /* r2c input / c2r output (real, n0 x n1) */
    fftw_complex *cbuf;   /* r2c output / c2r input (n0 x (n1/2 + 1)) */
};
typedef struct fftw_plan_s *fftw_plan;

void *fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void *p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* in-place 1-D complex transform of n values (re, im interleaved), sign = -1
 * forward, +1 backward */
static void fft1d(double *a, int n, int sign)
{
    if (n <= 1) return;
    if (is_pow2(n)) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double tr = a[2 * i], ti = a[2 * i + 1];
                a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
                a[2 * j] = tr; a[2 * j + 1] = ti;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1;
            for (int k = 0; k < half; ++k) {
                const double ang = sign * 2.0 * M_PI * (double)k / (double)len;
                const double wr = cos(ang), wi = sin(ang);
                for (int s = 0; s < n; s += len) {
                    double *u = a + 2 * (s + k), *v = a + 2 * (s + k + half);
                    const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                    v[0] = u[0] - vr; v[1] = u[1] - vi;
                    u[0] += vr; u[1] += vi;
                }
            }
        }
        return;
    }
    double *t = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) {
            const double ang = sign * 2.0 * M_PI * (double)(((long long)j * k) % n) / (double)n;
            const double wr = cos(ang), wi = sin(ang);
            sr += a[2 * j] * wr - a[2 * j + 1] * wi;
            si += a[2 * j] * wi + a[2 * j + 1] * wr;
        }
        t[2 * k] = sr; t[2 * k + 1] = si;
    }
    memcpy(a, t, sizeof(double) * 2 * (size_t)n);
    free(t);
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->kind = 0; p->n0 = n0; p->n1 = n1; p->rin = in; p->cbuf = out;
    return p;
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->kind = 1; p->n0 = n0; p->n1 = n1; p->rin = out; p->cbuf = in;
    return p;
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

void fftw_execute(const fftw_plan p)
{
    const int n0 = p->n0, n1 = p->n1, h = n1 / 2 + 1;
    const int nmax = n0 > n1 ? n0 : n1;
    double *row = (double *)malloc(sizeof(double) * 2 * (size_t)nmax);
    if (p->kind == 0) {
        /* rows: full complex transform of each real row, keep the first h bins */
        for (int i = 0; i < n0; ++i) {
            for (int j = 0; j < n1; ++j) { row[2 * j] = p->rin[(size_t)i * n1 + j]; row[2 * j + 1] = 0.0; }
            fft1d(row, n1, -1);
            for (int k = 0; k < h; ++k) {
                p->cbuf[(size_t)i * h + k][0] = row[2 * k];
                p->cbuf[(size_t)i * h + k][1] = row[2 * k + 1];
            }
        }
        /* columns of the half spectrum */
        for (int k = 0; k < h; ++k) {
            for (int i = 0; i < n0; ++i) {
                row[2 * i] = p->cbuf[(size_t)i * h + k][0];
                row[2 * i + 1] = p->cbuf[(size_t)i * h + k][1];
            }
            fft1d(row, n0, -1);
            for (int i = 0; i < n0; ++i) {
                p->cbuf[(size_t)i * h + k][0] = row[2 * i];
                p->cbuf[(size_t)i * h + k][1] = row[2 * i + 1];
            }
        }
    } else {
        /* columns of the half spectrum, backward */
        fftw_complex *tmp = (fftw_complex *)malloc(sizeof(fftw_complex) * (size_t)n0 * h);
        for (int k = 0; k < h; ++k) {
            for (int i = 0; i < n0; ++i) {
                row[2 * i] = p->cbuf[(size_t)i * h + k][0];
                row[2 * i + 1] = p->cbuf[(size_t)i * h + k][1];
            }
            fft1d(row, n0, +1);
            for (int i = 0; i < n0; ++i) {
                tmp[(size_t)i * h + k][0] = row[2 * i];
                tmp[(size_t)i * h + k][1] = row[2 * i + 1];
            }
        }
        /* rows: Hermitian extension X[n1 - k] = conj(X[k]), backward, real part */
        for (int i = 0; i < n0; ++i) {
            for (int k = 0; k < h; ++k) {
                row[2 * k] = tmp[(size_t)i * h + k][0];
                row[2 * k + 1] = tmp[(size_t)i * h + k][1];
            }
            for (int k = h; k < n1; ++k) {
                row[2 * k] = tmp[(size_t)i * h + (n1 - k)][0];
                row[2 * k + 1] = -tmp[(size_t)i * h + (n1 - k)][1];
            }
            fft1d(row, n1, +1);
            for (int j = 0; j < n1; ++j) p->rin[(size_t)i * n1 + j] = row[2 * j];
        }
        free(tmp);
    }
    free(row);
}
