/*
 * TEST INFRASTRUCTURE ONLY — the GSL 1.16 entry points that the reference's
 * Segmentation.cpp imports besides those of gsl_shim.c: the histogram
 * functions (used by its Isodata and triangle thresholders,
 * Segmentation.cpp:56-236, 759-800) and gsl_sort_vector (its median
 * filter, :588). The GLRT thresholder the fit path's candidates come from
 * uses none of them; they are here so that Segmentation.cpp links
 * unmodified. Compiled against the reference's vendored GSL headers for the
 * struct layouts; behaviour per GSL's documentation: uniform bins
 * [range[i], range[i+1]), values outside [range[0], range[n]) ignored, ties of
 * the maximum resolved to the first bin, ascending in-place sort.
 */
#include <gsl/gsl_errno.h>
#include <gsl/gsl_histogram.h>
#include <gsl/gsl_vector.h>

#include <stdlib.h>

gsl_histogram *gsl_histogram_alloc(size_t n)
{
    if (n == 0) return NULL;
    gsl_histogram *h = (gsl_histogram *)malloc(sizeof(gsl_histogram));
    h->n = n;
    h->range = (double *)calloc(n + 1, sizeof(double));
    h->bin = (double *)calloc(n, sizeof(double));
    return h;
}

void gsl_histogram_free(gsl_histogram *h)
{
    if (!h) return;
    free(h->range);
    free(h->bin);
    free(h);
}

int gsl_histogram_set_ranges_uniform(gsl_histogram *h, double xmin, double xmax)
{
    if (!(xmin < xmax)) return GSL_EINVAL;
    for (size_t i = 0; i <= h->n; ++i) h->range[i] = xmin + ((double)i / (double)h->n) * (xmax - xmin);
    for (size_t i = 0; i < h->n; ++i) h->bin[i] = 0.0;
    return GSL_SUCCESS;
}

int gsl_histogram_increment(gsl_histogram *h, double x)
{
    const size_t n = h->n;
    if (!(x >= h->range[0]) || !(x < h->range[n])) return GSL_EDOM;
    /* uniform estimate, then step to the bin whose range holds x */
    size_t i = (size_t)((x - h->range[0]) / (h->range[n] - h->range[0]) * (double)n);
    if (i >= n) i = n - 1;
    while (i > 0 && x < h->range[i]) --i;
    while (i + 1 < n && x >= h->range[i + 1]) ++i;
    h->bin[i] += 1.0;
    return GSL_SUCCESS;
}

double gsl_histogram_get(const gsl_histogram *h, size_t i) { return i < h->n ? h->bin[i] : 0.0; }

int gsl_histogram_get_range(const gsl_histogram *h, size_t i, double *lower, double *upper)
{
    if (i >= h->n) return GSL_EDOM;
    *lower = h->range[i];
    *upper = h->range[i + 1];
    return GSL_SUCCESS;
}

double gsl_histogram_max_val(const gsl_histogram *h)
{
    double m = h->bin[0];
    for (size_t i = 1; i < h->n; ++i)
        if (h->bin[i] > m) m = h->bin[i];
    return m;
}

size_t gsl_histogram_max_bin(const gsl_histogram *h)
{
    size_t k = 0;
    for (size_t i = 1; i < h->n; ++i)
        if (h->bin[i] > h->bin[k]) k = i;
    return k;
}

static int cmp_double(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

void gsl_sort_vector(gsl_vector *v)
{
    if (v->stride == 1) {
        qsort(v->data, v->size, sizeof(double), cmp_double);
        return;
    }
    double *t = (double *)malloc(sizeof(double) * (v->size ? v->size : 1));
    for (size_t i = 0; i < v->size; ++i) t[i] = v->data[i * v->stride];
    qsort(t, v->size, sizeof(double), cmp_double);
    for (size_t i = 0; i < v->size; ++i) v->data[i * v->stride] = t[i];
    free(t);
}

/* GSL's error hook (GSL_ERROR in the vendored headers): the reference's
 * segmentation code reports through it; here the message is printed and
 * control returns to the caller, which then sees the error code. */
#include <stdio.h>
void gsl_error(const char *reason, const char *file, int line, int gsl_errno)
{
    fprintf(stderr, "gsl: %s:%d: %s (%d)\n", file, line, reason, gsl_errno);
}
