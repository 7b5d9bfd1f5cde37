// Host candidate finder: GLRT detection + adjacent-8 particle grouping.
//
// Restates ThresholdImage_GLRT_FFT (reference source/Segmentation.cpp:241-430)
// and ParticleFinder_adjacent8 (source/ParticleFinding.cpp:283-427). The
// reference correlates with the zero-mean Gaussian window through an FFT of
// the whole frame; on the interior pixels the test visits that equals the
// direct sum used here. Window sums of the pixel values and their squares are
// exact integer sums in double. Frames are processed in parallel on host
// threads, one frame per task, as PALMAnalysisController does
// (source/PALMAnalysis.cpp:96-130).
#include "../../include/localizer_b200.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Particle {
    double x, y, intensity, background;
};

void glrt_mask(const uint16_t *frame, int n_rows, int n_cols, double pfa, double w, std::vector<int32_t> &mask)
{
    int ws = (int)std::ceil(4 * w);
    if (ws % 2 == 0) ws += 1;
    const int half = ws / 2;
    const double npix = (double)ws * (double)ws;
    const int xs = n_rows - (n_rows % 2), ys = n_cols - (n_cols % 2);
    mask.assign((size_t)n_rows * n_cols, 0);
    if (xs < ws + 2 || ys < ws + 2) return;
    std::vector<double> g((size_t)ws * ws);
    double sum = 0.0;
    for (int j = -half; j <= half; ++j)
        for (int i = -half; i <= half; ++i) {
            double v = 1.0 / (1.77245385 * w) * std::exp(-1.0 / (2.0 * w * w) * ((double)i * i + (double)j * j));
            g[(i + half) + (j + half) * ws] = v;
            sum += v;
        }
    sum /= npix;
    double sumsq = 0.0;
    for (auto &v : g) {
        v -= sum;
        sumsq += v * v;
    }
    const double thr = 1.0 - std::exp(-pfa / npix);
    for (int l = half + 1; l < ys - half; l++) {
        for (int k = half + 1; k < xs - half; k++) {
            double s1 = 0.0, s2 = 0.0, conv = 0.0;
            for (int b = -half; b <= half; b++) {
                const uint16_t *rowp = frame + (size_t)(l + b) * n_rows + (k - half);
                const double *gr = &g[(size_t)(b + half) * ws];
                for (int a = 0; a < ws; a++) {
                    const double v = (double)rowp[a];
                    s1 += v;
                    s2 += v * v;
                    conv += v * gr[a];
                }
            }
            const double avg = s1 / npix;
            const double null_h = s2 - avg * avg * npix;
            const double alpha = conv / sumsq;
            const double test = alpha * alpha / null_h * sumsq;
            if (test < 1.0 && test > thr) mask[(size_t)k + (size_t)l * n_rows] = 255;
        }
    }
}

void adjacent8(const uint16_t *frame, int n_rows, int n_cols, const std::vector<int32_t> &mask,
               std::vector<Particle> &out)
{
    const size_t npx = (size_t)n_rows * n_cols;
    std::vector<int32_t> mapped(npx, -1);
    std::vector<int> queue;
    queue.reserve(1024);
    double bg = 0.0;
    size_t nbg = 0;
    int pidx = 0;
    out.clear();
    for (int j = 0; j < n_cols; j++) {
        for (int i = 0; i < n_rows; i++) {
            const size_t at = (size_t)i + (size_t)j * n_rows;
            if (mask[at] < 128) {
                bg += (double)frame[at];
                ++nbg;
                continue;
            }
            if (mapped[at] != -1) continue;
            mapped[at] = pidx;
            queue.clear();
            queue.push_back((int)at);
            size_t qh = 0;
            double sx = 0.0, sy = 0.0, mx = 0.0;
            long cnt = 0;
            while (qh < queue.size()) {
                const int cur = queue[qh++];
                const int cx = cur % n_rows, cy = cur / n_rows;
                const int lx = std::max(cx - 1, 0), ux = std::min(cx + 1, n_rows - 1);
                const int ly = std::max(cy - 1, 0), uy = std::min(cy + 1, n_cols - 1);
                for (int b = ly; b <= uy; b++)
                    for (int a = lx; a <= ux; a++) {
                        if (a == cx && b == cy) continue;
                        const size_t nat = (size_t)a + (size_t)b * n_rows;
                        if (mask[nat] < 128 || mapped[nat] != -1) continue;
                        mapped[nat] = pidx;
                        queue.push_back((int)nat);
                    }
                sx += (double)cx;
                sy += (double)cy;
                const double v = (double)frame[cur];
                if (v > mx) mx = v;
                cnt++;
            }
            ++pidx;
            out.push_back({sx / (double)cnt, sy / (double)cnt, mx, 0.0});
        }
    }
    bg /= (double)nbg;
    for (auto &p : out) {
        p.intensity -= bg;
        p.background = bg;
    }
}

}  // namespace

extern "C" LOC_API long loc_find_candidates_host(const uint16_t *frames, int n_frames, int n_rows, int n_cols,
                                                 double pfa, double psf_width, int n_threads, loc_candidate *cands,
                                                 long max_cands)
{
    if (!frames || n_frames < 0 || n_rows <= 0 || n_cols <= 0 || !(psf_width > 0) || max_cands < 0 ||
        (max_cands > 0 && !cands))
        return LOC_E_INVALID;
    int nt = n_threads > 0 ? n_threads : (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if (nt > n_frames) nt = n_frames > 0 ? n_frames : 1;
    std::vector<std::vector<Particle>> per((size_t)n_frames);
    std::atomic<int> next{0};
    auto worker = [&]() {
        std::vector<int32_t> mask;
        for (;;) {
            const int f = next.fetch_add(1);
            if (f >= n_frames) break;
            const uint16_t *fr = frames + (size_t)f * n_rows * n_cols;
            glrt_mask(fr, n_rows, n_cols, pfa, psf_width, mask);
            adjacent8(fr, n_rows, n_cols, mask, per[(size_t)f]);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(worker);
    worker();
    for (auto &t : th) t.join();
    long total = 0;
    for (int f = 0; f < n_frames; ++f) {
        for (const auto &p : per[(size_t)f]) {
            if (total < max_cands) {
                loc_candidate &c = cands[total];
                c.x = p.x;
                c.y = p.y;
                c.intensity = p.intensity;
                c.background = p.background;
                c.frame = f;
                c.half_width = 0;
            }
            ++total;
        }
    }
    return total;
}
