/*
 * TEST INFRASTRUCTURE ONLY — drives the reference's own fitter and finder
 * classes (compiled unmodified from the reference tree into oracle/_ref by
 * oracle/Makefile) on one stack of uint16 frames, so that the restatement in
 * loc_oracle.c and the CUDA path can be checked against the reference code.
 *
 * The ROI half-width of a reference fitter is fixed at construction as
 * ceil(4*w0) (Localization.h:68,84,97); the harness sets the protected
 * cutoff_radius member directly to honour per-candidate half-widths.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <list>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <Eigen/Eigen>
#include <gsl/gsl_histogram.h>
#include <gsl/gsl_matrix.h>
#include <gsl/gsl_vector.h>

/* Only the reference's own headers see this; the standard library and the
 * vendored third-party headers above are already included. */
#define protected public
#include "Localization.h"
#include "ParticleFinding.h"
#undef protected

extern "C" {
void lmshim_log_reset(void);
long lmshim_log_count(void);
void lmshim_log_get(long i, int *iters, int *status);
}

namespace {

struct Cand {
    double x, y, intensity, background;
    int32_t frame;
    int32_t half_width;
};

ImagePtr frame_image(const uint16_t *frames, int frame, int n_rows, int n_cols)
{
    ImagePtr img(new Image(n_rows, n_cols));
    const uint16_t *src = frames + (size_t)frame * n_rows * n_cols;
    for (int j = 0; j < n_cols; j++)
        for (int i = 0; i < n_rows; i++) (*img)(i, j) = (double)src[i + (size_t)j * n_rows];
    return img;
}

std::shared_ptr<FitPositions> make_fitter(int method, double w0, double sigma, size_t r)
{
    switch (method) {
    case 0: {
        auto f = std::make_shared<FitPositions_SymmetricGaussian>(w0, sigma);
        f->cutoff_radius = r;
        return f;
    }
    case 1: {
        auto f = std::make_shared<FitPositions_FixedWidthGaussian>(w0, sigma);
        f->cutoff_radius = r;
        return f;
    }
    case 7: {
        auto f = std::make_shared<FitPositions_EllipsoidalGaussian>(w0, sigma);
        f->cutoff_radius = r;
        return f;
    }
    case 5: {
        auto f = std::make_shared<FitPositions_EllipsoidalGaussian_SymmetricPSF>(w0, sigma);
        f->ellipsoidalFitter.cutoff_radius = r;
        return f;
    }
    case 6: {
        auto f = std::make_shared<FitPositions_MLEwG>(w0);   /* no noise weight */
        f->cutoff_radius = r;
        return f;
    }
    }
    return nullptr;
}

int ref_cols(int method)
{
    return method == 0 ? 12 : method == 1 ? 10 : method == 6 ? 8 : 16;
}

} // namespace

extern "C" {

/*
 * Fit the candidates with the reference classes. Candidates must be grouped
 * so that each run of equal (frame, half_width) is contiguous; each run is
 * one fit_positions() call, as one frame is in PALMAnalysis.cpp:234.
 * out: nc rows of ref_cols(method) doubles (rows of kept candidates only are
 * written); kept[i] = 1 if candidate i produced an output row; iters[i] =
 * iterate() calls (-1 if the solver never ran, i.e. the edge reject);
 * status[i] = last iterate() status.
 */
int ref_fit(const uint16_t *frames, int n_frames, int n_rows, int n_cols, const void *cands_v,
            int nc, int method, double w0, double sigma, double *out, int32_t *kept,
            int32_t *iters, int32_t *status)
{
    const Cand *cands = (const Cand *)cands_v;
    const int ncol = ref_cols(method);
    for (int i = 0; i < nc; i++) {
        kept[i] = 0;
        iters[i] = -1;
        status[i] = 0;
    }
    try {
        int start = 0;
        while (start < nc) {
            int end = start + 1;
            while (end < nc && cands[end].frame == cands[start].frame &&
                   cands[end].half_width == cands[start].half_width)
                end++;
            int fr = cands[start].frame;
            if (fr < 0 || fr >= n_frames) return -2;
            size_t r = cands[start].half_width > 0 ? (size_t)cands[start].half_width
                                                   : (size_t)std::ceil(w0 * 4.0);
            ImagePtr img = frame_image(frames, fr, n_rows, n_cols);

            auto make_list = [&]() {
                auto lst = std::make_shared<std::list<Particle>>();
                for (int i = start; i < end; i++) {
                    Particle p;
                    p.x = cands[i].x;
                    p.y = cands[i].y;
                    p.intensity = cands[i].intensity;
                    p.background = cands[i].background;
                    lst->push_back(p);
                }
                return lst;
            };

            /* raw fit: for method 5 this is the ellipsoidal fit it wraps */
            int raw_method = method == 5 ? 7 : method;
            auto lst = make_list();
            lmshim_log_reset();
            auto fitter = make_fitter(raw_method, w0, sigma, r);
            auto res = fitter->fit_positions(img, lst);
            ImagePtr m = res->getLocalizedPositionsAsMatrix();

            /* edge-rejected candidates never reach the solver: map log entries */
            long nlog = lmshim_log_count();
            long li = 0;
            for (int i = start; i < end; i++) {
                double x0 = cands[i].x, y0 = cands[i].y;
                long xo = (long)std::floor(x0 - (double)r), yo = (long)std::floor(y0 - (double)r);
                long xm = xo + 2 * (long)r, ym = yo + 2 * (long)r;
                bool edge = xo < 0 || xm > n_rows - 1 || yo < 0 || ym > n_cols - 1;
                if (edge) continue;
                if (li < nlog) {
                    int it, st;
                    lmshim_log_get(li, &it, &st);
                    iters[i] = it;
                    status[i] = st;
                }
                li++;
            }

            /* the surviving list is the kept subsequence, in order */
            std::vector<int> kept_idx;
            auto it = lst->begin();
            for (int i = start; i < end && it != lst->end(); i++) {
                if (it->x == cands[i].x && it->y == cands[i].y &&
                    it->intensity == cands[i].intensity && it->background == cands[i].background) {
                    kept_idx.push_back(i);
                    ++it;
                }
            }
            if ((long)kept_idx.size() != (long)m->rows()) return -3;

            if (method != 5) {
                for (size_t k = 0; k < kept_idx.size(); k++) {
                    int i = kept_idx[k];
                    kept[i] = 1;
                    for (int c = 0; c < ncol; c++) out[(size_t)i * ncol + c] = (*m)((int)k, c);
                    out[(size_t)i * ncol + 0] = (double)fr;
                }
            } else {
                auto lst2 = make_list();
                auto f5 = make_fitter(5, w0, sigma, r);
                auto res5 = f5->fit_positions(img, lst2);
                ImagePtr m5 = res5->getLocalizedPositionsAsMatrix();
                /* rows of the filtered container are a subsequence of the raw rows */
                long k5 = 0;
                for (size_t k = 0; k < kept_idx.size() && k5 < m5->rows(); k++) {
                    bool same = true;
                    for (int c = 0; c < ncol; c++) {
                        double a = (*m)((int)k, c), b = (*m5)((int)k5, c);
                        if (!(a == b || (std::isnan(a) && std::isnan(b)))) {
                            same = false;
                            break;
                        }
                    }
                    if (same) {
                        int i = kept_idx[k];
                        kept[i] = 1;
                        for (int c = 0; c < ncol; c++) out[(size_t)i * ncol + c] = (*m5)((int)k5, c);
                        out[(size_t)i * ncol + 0] = (double)fr;
                        k5++;
                    }
                }
                if (k5 != m5->rows()) return -4;
            }
            start = end;
        }
    } catch (...) {
        return -1;
    }
    return 0;
}

/*
 * The reference's own text writer: fit one frame's candidates (all with the
 * same frame and ROI half-width) with the reference fitter of `method`, set
 * the frame numbers as the controller does (PALMAnalysis.cpp:238) and write
 * them with writePositionsToFile (Storage.cpp:292-345, 427-470, 642-700).
 * Returns the number of positions written, or a negative code.
 */
int ref_write_positions(const uint16_t *frames, int n_frames, int n_rows, int n_cols, const void *cands_v, int nc,
                        int method, double w0, double sigma, const char *path, const char *header)
{
    const Cand *cands = (const Cand *)cands_v;
    if (nc <= 0) return -2;
    for (int i = 1; i < nc; i++)
        if (cands[i].frame != cands[0].frame || cands[i].half_width != cands[0].half_width) return -2;
    const int fr = cands[0].frame;
    if (fr < 0 || fr >= n_frames) return -2;
    /* make sure the stream library (and its locale) of this library is set up */
    static std::ios_base::Init ios_init;
    try {
        size_t r = cands[0].half_width > 0 ? (size_t)cands[0].half_width : (size_t)std::ceil(w0 * 4.0);
        ImagePtr img = frame_image(frames, fr, n_rows, n_cols);
        auto lst = std::make_shared<std::list<Particle>>();
        for (int i = 0; i < nc; i++) {
            Particle p;
            p.x = cands[i].x;
            p.y = cands[i].y;
            p.intensity = cands[i].intensity;
            p.background = cands[i].background;
            lst->push_back(p);
        }
        auto fitter = make_fitter(method, w0, sigma, r);
        auto res = fitter->fit_positions(img, lst);
        res->setFrameNumbers((size_t)fr);
        res->writePositionsToFile(std::string(path), std::string(header));
        return (int)res->getNPositions();
    } catch (...) {
        return -1;
    }
}

/* The reference's own GLRT detector (ThresholdImage_GLRT_FFT,
 * Segmentation.cpp:241-430, with its FFT-based Gaussian correlation running
 * on fftw_shim.c) on one frame: mask_out receives 255 / 0 per pixel,
 * column-major like the frame. */
int ref_glrt_mask(const uint16_t *frame, int n_rows, int n_cols, double pfa, double psf_width, int32_t *mask_out)
{
    try {
        ImagePtr img = frame_image(frame, 0, n_rows, n_cols);
        ThresholdImage_GLRT_FFT th(pfa, psf_width);
        auto m = th.do_thresholding(img);
        for (int j = 0; j < n_cols; j++)
            for (int i = 0; i < n_rows; i++) mask_out[i + (size_t)j * n_rows] = (*m)(i, j);
        return 0;
    } catch (...) {
        return -1;
    }
}

/* The reference's candidate pipeline over a stack, as its analysis
 * controller runs it per frame (PALMAnalysis.cpp:214-227, one thresholder
 * and one finder for the whole stack): GLRT + adjacent-8. out receives
 * (x, y, intensity, background, frame) per particle in frame order; returns
 * the number found (only max_out are written) or -1. */
long ref_find_candidates(const uint16_t *frames, int n_frames, int n_rows, int n_cols, double pfa,
                         double psf_width, double *out, long max_out)
{
    try {
        ThresholdImage_GLRT_FFT th(pfa, psf_width);
        ParticleFinder_adjacent8 finder;
        long k = 0;
        for (int f = 0; f < n_frames; f++) {
            ImagePtr img = frame_image(frames, f, n_rows, n_cols);
            auto m = th.do_thresholding(img);
            auto parts = finder.findPositions(img, m);
            for (auto &p : *parts) {
                if (k < max_out) {
                    out[5 * k + 0] = p.x;
                    out[5 * k + 1] = p.y;
                    out[5 * k + 2] = p.intensity;
                    out[5 * k + 3] = p.background;
                    out[5 * k + 4] = (double)f;
                }
                k++;
            }
        }
        return k;
    } catch (...) {
        return -1;
    }
}

/* The reference's adjacent-8 finder on a given mask (255 = detected). */
int ref_find_adjacent8(const uint16_t *frame, int n_rows, int n_cols, const int32_t *mask,
                       double *out, int max_out)
{
    try {
        ImagePtr img = frame_image(frame, 0, n_rows, n_cols);
        auto th = std::make_shared<Eigen::Matrix<int, Eigen::Dynamic, Eigen::Dynamic>>(n_rows, n_cols);
        for (int j = 0; j < n_cols; j++)
            for (int i = 0; i < n_rows; i++) (*th)(i, j) = mask[i + (size_t)j * n_rows];
        ParticleFinder_adjacent8 finder;
        auto parts = finder.findPositions(img, th);
        int k = 0;
        for (auto &p : *parts) {
            if (k < max_out) {
                out[4 * k + 0] = p.x;
                out[4 * k + 1] = p.y;
                out[4 * k + 2] = p.intensity;
                out[4 * k + 3] = p.background;
            }
            k++;
        }
        return k;
    } catch (...) {
        return -1;
    }
}

} // extern "C"
