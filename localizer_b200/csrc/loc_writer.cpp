// Localized-positions text writer in the reference's format
// (LocalizedPositionsContainer_*::writePositionsToFile, reference
// source/Storage.cpp:292-345 symmetric, 427-470 fixed width, 642-700
// ellipsoidal, 1128-1175 MLEwG): a title line naming the fit, the caller's header line,
// "DATA FOLLOWS", the column titles, then one tab-separated line per kept
// position. Frame numbers and the frames-present count are integers; every
// other value is written as a default-formatted C++ stream writes a double
// (printf "%g": 6 significant digits), so files are byte-identical to the
// reference's for the same positions. Rows are formatted in parallel on
// host threads and written in order.
#include "../../include/localizer_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace locb {
int record_error_fixed(int code, const char *msg);
}

namespace {

const char *const kTitle[4] = {
    "Localized positions using symmetric 2D Gauss fitting",
    "Localized positions using symmetric 2D Gauss fitting with fixed PSF width",
    "Localized positions using ellipsoidal 2D Gauss fitting",
    "Localized positions using MLEwG estimation",
};

const char *const kCols0[] = {"First frame", "Integrated intensity", "Fitted PSF standard deviation (pixel)",
                              "X position (pixel)", "Y position (pixel)", "Background", "Intensity deviation",
                              "PSF width deviation (pixel)", "X position deviation (pixel)",
                              "Y position deviation (pixel)", "Background deviation (pixel)",
                              "Number of frames where this emitter is present"};
const char *const kCols1[] = {"First frame", "Integrated intensity", "X position (pixel)", "Y position (pixel)",
                              "Background", "Intensity deviation", "X position deviation (pixel)",
                              "Y position deviation (pixel)", "Background deviation",
                              "Number of frames where this emitter is present"};
const char *const kCols7[] = {"First frame", "Integrated intensity",
                              "Fitted PSF standard deviation along first principal axis (pixel)",
                              "Fitted PSF standard deviation along second principal axis (pixel)",
                              "X position (pixel)", "Y position (pixel)", "Angular rotation (radians)", "Background",
                              "Intensity deviation", "PSF width deviation along first principal axis (pixel)",
                              "PSF width deviation along second principal axis (pixel)",
                              "X position deviation (pixel)", "Y position deviation (pixel)", "Rotation deviation",
                              "Background deviation", "Number of frames where this emitter is present"};

const char *const kCols6[] = {"First frame", "Integrated intensity", "Fitted PSF standard deviation (pixel)",
                              "X position (pixel)", "Y position (pixel)", "Background", "Position deviation (pixel)",
                              "Number of frames where this emitter is present"};

void format_row(std::string &s, const double *row, int ncol)
{
    char buf[64];
    for (int c = 0; c < ncol; ++c) {
        int len;
        if (c == 0 || c == ncol - 1)  // frame number, frames present: size_t in the reference
            len = std::snprintf(buf, sizeof buf, "%llu", (unsigned long long)row[c]);
        else
            len = std::snprintf(buf, sizeof buf, "%g", row[c]);
        s.append(buf, (size_t)len);
        s.push_back(c == ncol - 1 ? '\n' : '\t');
    }
}

}  // namespace

extern "C" LOC_API long loc_write_positions_text(const double *rows, const uint8_t *flags, long n, int method,
                                                 const char *path, const char *header)
{
    if (!path || n < 0 || (n > 0 && !rows))
        return locb::record_error_fixed(LOC_E_INVALID, "bad argument");
    if (!(method == 0 || method == 1 || method == 5 || method == 6 || method == 7))
        return locb::record_error_fixed(LOC_E_UNSUPPORTED, "unsupported method code");
    const int ref_cols = method == 0 ? 12 : method == 1 ? 10 : method == 6 ? 8 : 16;
    const int stride = ref_cols + 2;  // rows as the fit calls write them
    const char *const *cols = method == 0 ? kCols0 : method == 1 ? kCols1 : method == 6 ? kCols6 : kCols7;
    std::vector<long> kept;
    kept.reserve((size_t)n);
    for (long i = 0; i < n; ++i)
        if (!flags || flags[i] == 0) kept.push_back(i);
    if (kept.empty()) return locb::record_error_fixed(LOC_E_INVALID, "No positions localized!");

    FILE *f = std::fopen(path, "wb");
    if (!f) return locb::record_error_fixed(LOC_E_INVALID, "Unable to create the output file");
    std::string head;
    head += kTitle[method == 0 ? 0 : method == 1 ? 1 : method == 6 ? 3 : 2];
    head += "\n";
    head += header ? header : "";
    head += "\nDATA FOLLOWS\n";
    for (int c = 0; c < ref_cols; ++c) {
        head += cols[c];
        head += c == ref_cols - 1 ? "\n" : "\t";
    }
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();

    const long nk = (long)kept.size();
    int nt = (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, (int)(nk / 20000) + 1));
    const long block = 1 << 16;  // rows formatted per task, written in order
    std::vector<std::string> parts((size_t)nt);
    for (long base = 0; base < nk && ok; base += block * nt) {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) {
            const long a = base + (long)t * block, b = std::min(nk, a + block);
            parts[(size_t)t].clear();
            if (a >= b) continue;
            auto job = [&, t, a, b]() {
                std::string &s = parts[(size_t)t];
                s.reserve((size_t)(b - a) * (size_t)ref_cols * 12);
                for (long k = a; k < b; ++k) format_row(s, rows + (size_t)kept[(size_t)k] * stride, ref_cols);
            };
            if (t == nt - 1 || b == nk) job();
            else th.emplace_back(job);
        }
        for (auto &x : th) x.join();
        for (int t = 0; t < nt && ok; ++t)
            ok = std::fwrite(parts[(size_t)t].data(), 1, parts[(size_t)t].size(), f) == parts[(size_t)t].size();
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) return locb::record_error_fixed(LOC_E_INVALID, "Error writing to the localized positions file");
    return nk;
}
