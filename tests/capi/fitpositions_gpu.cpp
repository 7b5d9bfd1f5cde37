/*
 * TEST INFRASTRUCTURE — the C++ drop-in of the fitting path, compiled
 * against the reference's own headers (source/Localization.h,
 * source/Storage.h) by oracle/Makefile (target `capi`), together with the
 * reference's fitter classes, into oracle/_ref/libfitpositions_gpu.so.
 *
 * FitPositions_GPU is the subclass a maintainer adds next to the reference's
 * fitters: it overrides the virtual FitPositions::fit_positions
 * (Localization.h:55-61), forwards the frame and its particles to the C ABI
 * (loc_fit_host of include/localizer_b200.h), erases the rejected particles
 * from the caller's list as the reference's fitters do
 * (Localization.cpp:107-212) and returns the method's
 * LocalizedPositionsContainer. fpgpu_compare drives it and the reference's
 * own fitter through the reference's worker pattern (one fit_positions call
 * per frame, then setFrameNumbers, then a merge into one container,
 * PALMAnalysis.cpp:196-240) so a test can compare both results.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <vector>

#include <Eigen/Eigen>

#include "Localization.h"
#include "Storage.h"
#include "localizer_b200.h"

class FitPositions_GPU : public FitPositions {
public:
    FitPositions_GPU(int method_rhs, double initialPSFWidth, double sigma_rhs = 1.0, int device = 0)
        : method(method_rhs), w0(initialPSFWidth), sigma(sigma_rhs)
    {
        if (loc_ctx_create(&ctx, device) != LOC_OK) throw std::runtime_error(loc_last_error());
    }
    ~FitPositions_GPU() { loc_ctx_destroy(ctx); }

    std::shared_ptr<LocalizedPositionsContainer> fit_positions(const ImagePtr image,
                                                               std::shared_ptr<std::list<Particle> > particles)
    {
        std::lock_guard<std::mutex> lock(mutex);  // a loc_ctx serves one thread at a time
        const int nRows = (int)image->rows(), nCols = (int)image->cols();
        std::vector<uint16_t> frame((size_t)nRows * nCols);  // column-major, x fastest (FileIO.cpp:195)
        for (int j = 0; j < nCols; ++j)
            for (int i = 0; i < nRows; ++i) frame[i + (size_t)j * nRows] = (uint16_t)(*image)(i, j);
        std::vector<loc_candidate> cands;
        for (const Particle &p : *particles) cands.push_back({p.x, p.y, p.intensity, p.background, 0, 0});
        const int n = (int)cands.size();
        const int ncol = loc_output_columns(method);
        std::vector<double> rows((size_t)n * ncol);
        std::vector<uint8_t> flags((size_t)n);
        loc_options opt;
        loc_default_options(&opt);
        if (n > 0 && loc_fit_host(ctx, frame.data(), 1, nRows, nCols, cands.data(), n, method, w0, sigma, &opt,
                                  rows.data(), flags.data()) != LOC_OK)
            throw std::runtime_error(loc_last_error());
        // erase the rejects from the caller's list as the reference's fitters
        // do; the symmetric-PSF filter of method 5 drops positions from the
        // container but leaves their particles in the list
        // (Localization.cpp:606-631)
        auto it = particles->begin();
        for (int k = 0; k < n; ++k) {
            const bool erase = flags[k] != LOC_FLAG_KEPT && flags[k] != LOC_FLAG_SYMPSF_RATIO &&
                               flags[k] != LOC_FLAG_SYMPSF_WIDTH;
            it = erase ? particles->erase(it) : std::next(it);
        }
        return makeContainer(rows, flags, ncol);
    }

private:
    int method;
    double w0, sigma;
    loc_ctx *ctx = nullptr;
    std::mutex mutex;

    // kept rows -> the method's container, fields in the order of the
    // reference's LocalizedPosition_* classes (Storage.h:117-186, 233-249)
    std::shared_ptr<LocalizedPositionsContainer> makeContainer(const std::vector<double> &rows,
                                                               const std::vector<uint8_t> &flags, int ncol)
    {
        const size_t n = flags.size();
        if (method == LOC_METHOD_2DGAUSS) {
            auto c = std::make_shared<LocalizedPositionsContainer_2DGauss>();
            for (size_t k = 0; k < n; ++k) {
                if (flags[k]) continue;
                const double *r = &rows[k * ncol];
                auto p = std::make_shared<LocalizedPosition_2DGauss>();
                p->frameNumber = (size_t)r[0];
                p->integral = r[1]; p->width = r[2]; p->xPosition = r[3]; p->yPosition = r[4];
                p->background = r[5]; p->integralDeviation = r[6]; p->widthDeviation = r[7];
                p->xPositionDeviation = r[8]; p->yPositionDeviation = r[9]; p->backgroundDeviation = r[10];
                c->addPosition(p);
            }
            return c;
        }
        if (method == LOC_METHOD_2DGAUSS_FIXEDWIDTH) {
            auto c = std::make_shared<LocalizedPositionsContainer_2DGaussFixedWidth>();
            for (size_t k = 0; k < n; ++k) {
                if (flags[k]) continue;
                const double *r = &rows[k * ncol];
                auto p = std::make_shared<LocalizedPosition_2DGaussFixedWidth>();
                p->frameNumber = (size_t)r[0];
                p->integral = r[1]; p->xPosition = r[2]; p->yPosition = r[3]; p->background = r[4];
                p->integralDeviation = r[5]; p->xPositionDeviation = r[6]; p->yPositionDeviation = r[7];
                p->backgroundDeviation = r[8];
                c->addPosition(p);
            }
            return c;
        }
        if (method == LOC_METHOD_MLEWG) {
            auto c = std::make_shared<LocalizedPositionsContainer_MLEwG>();
            for (size_t k = 0; k < n; ++k) {
                if (flags[k]) continue;
                const double *r = &rows[k * ncol];
                auto p = std::make_shared<LocalizedPosition_MLEwG>();
                p->frameNumber = (size_t)r[0];
                p->integral = r[1]; p->width = r[2]; p->xPosition = r[3]; p->yPosition = r[4];
                p->background = r[5]; p->positionDeviation = r[6];
                c->addPosition(p);
            }
            return c;
        }
        auto c = std::make_shared<LocalizedPositionsContainer_Ellipsoidal2DGaussian>();
        for (size_t k = 0; k < n; ++k) {
            if (flags[k]) continue;
            const double *r = &rows[k * ncol];
            auto p = std::make_shared<LocalizedPosition_Ellipsoidal2DGauss>();
            p->frameNumber = (size_t)r[0];
            p->integral = r[1]; p->stdDev1 = r[2]; p->stdDev2 = r[3]; p->xPosition = r[4]; p->yPosition = r[5];
            p->theta = r[6]; p->background = r[7]; p->integralDeviation = r[8]; p->stdDev1Deviation = r[9];
            p->stdDev2Deviation = r[10]; p->xPositionDeviation = r[11]; p->yPositionDeviation = r[12];
            p->thetaDeviation = r[13]; p->backgroundDeviation = r[14];
            c->addPosition(p);
        }
        return c;
    }
};

namespace {

std::shared_ptr<FitPositions> reference_fitter(int method, double w0, double sigma)
{
    switch (method) {
    case 0: return std::make_shared<FitPositions_SymmetricGaussian>(w0, sigma);
    case 1: return std::make_shared<FitPositions_FixedWidthGaussian>(w0, sigma);
    case 5: return std::make_shared<FitPositions_EllipsoidalGaussian_SymmetricPSF>(w0, sigma);
    case 6: return std::make_shared<FitPositions_MLEwG>(w0);
    case 7: return std::make_shared<FitPositions_EllipsoidalGaussian>(w0, sigma);
    default: throw std::runtime_error("method");
    }
}

int copy_matrix(const std::shared_ptr<LocalizedPositionsContainer> &c, double *dst, int max_rows)
{
    ImagePtr m = c->getLocalizedPositionsAsMatrix();
    const int rows = (int)m->rows(), cols = (int)m->cols();
    if (rows > max_rows) return -1;
    // row-major copy of the column-major N x C matrix
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j) dst[(size_t)i * cols + j] = (*m)(i, j);
    return rows;
}

}  // namespace

extern "C" {

/*
 * For each frame f in [0, n_frames): the particles of that frame (x, y,
 * intensity, background rows of `particles` whose frame_of is f, in order)
 * go through FitPositions_GPU(method, w0, sigma) and through the
 * reference's fitter of that method, each on its own copy of the list; the
 * returned containers get setFrameNumbers(f) and are merged into one
 * container per side. Writes both merged matrices (row-major, at most
 * max_rows rows each) and the (x, y) of the particles each side left in its
 * list. Returns 0, or -1 on an error (message in loc_last_error for the GPU
 * side).
 */
int fpgpu_compare(const uint16_t *frames, int n_frames, int n_rows, int n_cols, const double *particles,
                  const int *frame_of, int n, int method, double w0, double sigma, int device, double *gpu_matrix,
                  int *gpu_rows, double *ref_matrix, int *ref_rows, int max_rows, double *gpu_left, int *n_gpu_left,
                  double *ref_left, int *n_ref_left)
{
    try {
        FitPositions_GPU gpu(method, w0, sigma, device);
        std::shared_ptr<FitPositions> ref = reference_fitter(method, w0, sigma);
        std::shared_ptr<LocalizedPositionsContainer> all_gpu, all_ref;
        int ng = 0, nr = 0;
        for (int f = 0; f < n_frames; ++f) {
            ImagePtr img(new Image(n_rows, n_cols));
            const uint16_t *src = frames + (size_t)f * n_rows * n_cols;
            for (int j = 0; j < n_cols; ++j)
                for (int i = 0; i < n_rows; ++i) (*img)(i, j) = (double)src[i + (size_t)j * n_rows];
            auto lg = std::make_shared<std::list<Particle> >();
            for (int k = 0; k < n; ++k) {
                if (frame_of[k] != f) continue;
                Particle p(particles[4 * k], particles[4 * k + 1], particles[4 * k + 2]);
                p.background = particles[4 * k + 3];
                lg->push_back(p);
            }
            auto lr = std::make_shared<std::list<Particle> >(*lg);
            auto cg = gpu.fit_positions(img, lg);
            auto cr = ref->fit_positions(img, lr);
            cg->setFrameNumbers(f);
            cr->setFrameNumbers(f);
            if (!all_gpu) all_gpu = cg; else all_gpu->addPositions(cg);
            if (!all_ref) all_ref = cr; else all_ref->addPositions(cr);
            for (const Particle &p : *lg) { gpu_left[2 * ng] = p.x; gpu_left[2 * ng + 1] = p.y; ++ng; }
            for (const Particle &p : *lr) { ref_left[2 * nr] = p.x; ref_left[2 * nr + 1] = p.y; ++nr; }
        }
        *n_gpu_left = ng;
        *n_ref_left = nr;
        *gpu_rows = all_gpu ? copy_matrix(all_gpu, gpu_matrix, max_rows) : 0;
        *ref_rows = all_ref ? copy_matrix(all_ref, ref_matrix, max_rows) : 0;
        if (*gpu_rows < 0 || *ref_rows < 0) return -1;
    } catch (...) {
        return -1;
    }
    return 0;
}

}  // extern "C"
