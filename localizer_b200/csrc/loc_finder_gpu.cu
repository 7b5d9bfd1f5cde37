// GPU candidate finder: GLRT detection + adjacent-8 particle grouping,
// restating ThresholdImage_GLRT_FFT (reference source/Segmentation.cpp:241-430)
// and ParticleFinder_adjacent8 (source/ParticleFinding.cpp:283-427) with the
// same results, bit for bit, as the host finder in loc_finder.cpp:
//
// * The GLRT statistic of every interior pixel uses the reference's zero-mean
//   Gaussian window (computed on the host in double, as the host finder does)
//   and the same floating-point operation sequence: window sums of values and
//   squares are exact integers, the correlation is accumulated row by row in
//   double with separate multiply and add (no fused multiply-add), and the
//   test value is formed in the host's order.
// * Connected components (8-neighbourhood) by union-find with links always
//   pointing to the smaller raster index, so every component's root is its
//   first pixel in raster order; particles are numbered in that order, which
//   is the order in which the reference's raster scan discovers them.
// * Particle position = unweighted mean of the component's pixel coordinates,
//   intensity = brightest pixel minus the frame background, background =
//   mean of the frame's pixels outside the mask: integer sums, exact in
//   double, divided once, as on the host.
//
// Frames are processed in chunks so that the per-pixel working arrays (mask,
// labels, particle ids: 9 bytes per pixel) stay within a bounded scratch.
#include "../../include/localizer_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace locb {
int record_error_fixed(int code, const char *msg);
}

namespace {

constexpr int kMaxWin = 33;                 // window side up to ceil(4 w) = 33 (w <= 8)
__constant__ double c_g[kMaxWin * kMaxWin];  // zero-mean Gaussian window, row-major (b, a)

constexpr int kTX = 32, kTY = 8;            // GLRT output tile
constexpr int kLinkLimit = 1 << 24;

// GLRT mask of every pixel of a chunk of frames, plus per-frame sums of the
// pixels outside the mask (the background).
__global__ void k_glrt(const uint16_t *frames, int n_rows, int n_cols, int ws, double npix, double sumsq,
                       double thr, uint8_t *mask, int *label, unsigned long long *bg_sum,
                       unsigned long long *bg_cnt)
{
    extern __shared__ uint16_t tile[];
    const int half = ws / 2;
    const int f = blockIdx.z;
    const int tx0 = blockIdx.x * kTX, ty0 = blockIdx.y * kTY;
    const int tw = kTX + 2 * half, th = kTY + 2 * half;
    const uint16_t *fr = frames + (size_t)f * n_rows * n_cols;
    const int tid = threadIdx.y * kTX + threadIdx.x;
    for (int k = tid; k < tw * th; k += kTX * kTY) {
        const int yy = ty0 - half + k / tw, xx = tx0 - half + k % tw;
        tile[k] = (xx >= 0 && xx < n_rows && yy >= 0 && yy < n_cols) ? fr[xx + (size_t)yy * n_rows] : 0;
    }
    __syncthreads();
    const int k = tx0 + threadIdx.x, l = ty0 + threadIdx.y;
    bool in = false;
    uint16_t pv = 0;
    if (k < n_rows && l < n_cols) {
        pv = tile[(threadIdx.y + half) * tw + threadIdx.x + half];
        const int xs = n_rows - (n_rows % 2), ys = n_cols - (n_cols % 2);
        if (xs >= ws + 2 && ys >= ws + 2 && l >= half + 1 && l < ys - half && k >= half + 1 && k < xs - half) {
            long long s1 = 0, s2 = 0;
            double conv = 0.0;
            for (int b = 0; b < ws; ++b) {
                const uint16_t *rowp = tile + (threadIdx.y + b) * tw + threadIdx.x;
                const double *gr = c_g + b * ws;
                for (int a = 0; a < ws; ++a) {
                    const long long v = rowp[a];
                    s1 += v;
                    s2 += v * v;
                    conv = __dadd_rn(conv, __dmul_rn((double)v, gr[a]));
                }
            }
            const double avg = __ddiv_rn((double)s1, npix);
            const double null_h = __dsub_rn((double)s2, __dmul_rn(__dmul_rn(avg, avg), npix));
            const double alpha = __ddiv_rn(conv, sumsq);
            const double test = __dmul_rn(__ddiv_rn(__dmul_rn(alpha, alpha), null_h), sumsq);
            in = test < 1.0 && test > thr;
        }
        const size_t at = (size_t)f * n_rows * n_cols + k + (size_t)l * n_rows;
        mask[at] = in ? 255 : 0;
        label[at] = in ? (int)at : -1;
    }
    // background sums of the pixels outside the mask, one atomic per warp
    const unsigned full = 0xffffffffu;
    unsigned long long s = (k < n_rows && l < n_cols && !in) ? (unsigned long long)pv : 0ull;
    unsigned long long c = (k < n_rows && l < n_cols && !in) ? 1ull : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(full, s, o);
        c += __shfl_xor_sync(full, c, o);
    }
    if ((tid & 31) == 0 && c) {
        atomicAdd(&bg_sum[f], s);
        atomicAdd(&bg_cnt[f], c);
    }
}

__device__ __forceinline__ int find_root(const int *L, int x)
{
    int n = 0;
    int y = L[x];
    while (y != x && n < kLinkLimit) {
        x = y;
        y = L[x];
        ++n;
    }
    return x;
}

// link two pixels' components; roots always keep the smaller index
__device__ void unite(int *L, int a, int b, int *err)
{
    for (int n = 0; n < kLinkLimit; ++n) {
        a = find_root(L, a);
        b = find_root(L, b);
        if (a == b) return;
        if (a < b) {
            const int old = atomicMin(&L[b], a);
            if (old == b) return;
            b = old;
        } else {
            const int old = atomicMin(&L[a], b);
            if (old == a) return;
            a = old;
        }
    }
    atomicExch(err, 1);
}

__global__ void k_union(const uint8_t *mask, int *label, int n_rows, int n_cols, long long n_px, int *err)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_px;
         p += (long long)gridDim.x * blockDim.x) {
        if (!mask[p]) continue;
        const long long fpx = (long long)n_rows * n_cols;
        const int local = (int)(p % fpx);
        const int x = local % n_rows, y = local / n_rows;
        // neighbours earlier in raster order: left, and the three above
        if (x > 0 && mask[p - 1]) unite(label, (int)p, (int)(p - 1), err);
        if (y > 0) {
            const long long up = p - n_rows;
            if (x > 0 && mask[up - 1]) unite(label, (int)p, (int)(up - 1), err);
            if (mask[up]) unite(label, (int)p, (int)up, err);
            if (x + 1 < n_rows && mask[up + 1]) unite(label, (int)p, (int)(up + 1), err);
        }
    }
}

__global__ void k_flatten(const uint8_t *mask, int *label, long long n_px)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_px;
         p += (long long)gridDim.x * blockDim.x)
        if (mask[p]) label[p] = find_root(label, (int)p);
}

// roots (first pixels of components) per frame
__global__ void k_count_roots(const uint8_t *mask, const int *label, int frame_px, int *count)
{
    const int f = blockIdx.x;
    const size_t base = (size_t)f * frame_px;
    int c = 0;
    for (int i = threadIdx.x; i < frame_px; i += blockDim.x) {
        const size_t p = base + i;
        c += (mask[p] && label[p] == (int)p) ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
        count[f] = t;
    }
}

// particle ids in raster order of the roots, one block per frame
__global__ void k_assign(const uint8_t *mask, const int *label, int frame_px, const int *offset, int *pid,
                         int *pframe, int frame0)
{
    const int f = blockIdx.x;
    const size_t base = (size_t)f * frame_px;
    __shared__ int warp_tot[32];
    __shared__ int running;
    if (threadIdx.x == 0) running = offset[f];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int start = 0; start < frame_px; start += blockDim.x) {
        const int i = start + threadIdx.x;
        const size_t p = base + i;
        const bool root = i < frame_px && mask[p] && label[p] == (int)p;
        const unsigned b = __ballot_sync(0xffffffffu, root);
        if (lane == 0) warp_tot[wid] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < nw; ++w) {
            const int t = warp_tot[w];
            before += w < wid ? t : 0;
            total += t;
        }
        if (root) {
            const int id = running + before + __popc(b & ((1u << lane) - 1));
            pid[p] = id;
            pframe[id] = frame0 + f;
        }
        __syncthreads();
        if (threadIdx.x == 0) running += total;
        __syncthreads();
    }
}

__global__ void k_accumulate(const uint8_t *mask, const int *label, const int *pid, const uint16_t *frames,
                             int n_rows, int frame_px, long long n_px, unsigned long long *sx,
                             unsigned long long *sy, unsigned int *cnt, unsigned int *mx)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_px;
         p += (long long)gridDim.x * blockDim.x) {
        if (!mask[p]) continue;
        const int id = pid[label[p]];
        const int local = (int)(p % frame_px);
        atomicAdd(&sx[id], (unsigned long long)(local % n_rows));
        atomicAdd(&sy[id], (unsigned long long)(local / n_rows));
        atomicAdd(&cnt[id], 1u);
        atomicMax(&mx[id], (unsigned int)frames[p]);
    }
}

__global__ void k_emit(int n, const int *pframe, int frame0, const unsigned long long *sx,
                       const unsigned long long *sy, const unsigned int *cnt, const unsigned int *mx,
                       const unsigned long long *bg_sum, const unsigned long long *bg_cnt, loc_candidate *out,
                       long long out_base, long long max_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long o = out_base + i;
    if (o >= max_out) return;
    const int f = pframe[i];
    const double bg = __ddiv_rn((double)bg_sum[f - frame0], (double)bg_cnt[f - frame0]);
    loc_candidate c;
    c.x = __ddiv_rn((double)sx[i], (double)cnt[i]);
    c.y = __ddiv_rn((double)sy[i], (double)cnt[i]);
    c.intensity = __dsub_rn((double)mx[i], bg);
    c.background = bg;
    c.frame = f;
    c.half_width = 0;
    out[o] = c;
}

struct Buf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) cap = n;
        return e;
    }
    ~Buf()
    {
        if (p) cudaFree(p);
    }
};

long long fail(int code, const std::string &m) { return locb::record_error_fixed(code, m.c_str()); }

}  // namespace

extern "C" LOC_API long loc_find_candidates(const uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                                            double pfa, double psf_width, loc_candidate *d_cands, long max_cands,
                                            void *stream)
{
    if (!d_frames || n_frames < 0 || n_rows <= 0 || n_cols <= 0 || !(psf_width > 0) || max_cands < 0 ||
        (max_cands > 0 && !d_cands))
        return fail(LOC_E_INVALID, "bad argument");
    int ws = (int)std::ceil(4 * psf_width);
    if (ws % 2 == 0) ws += 1;
    if (ws > kMaxWin) return fail(LOC_E_UNSUPPORTED, "PSF width too large for the GPU finder (window > 33)");
    if (n_frames == 0) return 0;
    const cudaStream_t st = (cudaStream_t)stream;
    // window as the host finder computes it (Segmentation.cpp:241-430)
    const int half = ws / 2;
    const double npix = (double)ws * (double)ws;
    std::vector<double> g((size_t)ws * ws);
    double sum = 0.0;
    for (int j = -half; j <= half; ++j)
        for (int i = -half; i <= half; ++i) {
            const double v = 1.0 / (1.77245385 * psf_width) *
                             std::exp(-1.0 / (2.0 * psf_width * psf_width) * ((double)i * i + (double)j * j));
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
    cudaError_t e = cudaMemcpyToSymbolAsync(c_g, g.data(), g.size() * sizeof(double), 0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(LOC_E_CUDA, std::string("window upload: ") + cudaGetErrorString(e));

    const long long frame_px = (long long)n_rows * n_cols;
    if (frame_px > (1ll << 30)) return fail(LOC_E_UNSUPPORTED, "frame too large");
    // chunk of frames with at most 2^26 pixels (9 bytes each of working arrays)
    int chunk = (int)std::max(1ll, std::min<long long>(n_frames, (1ll << 26) / frame_px));
    static thread_local Buf b_mask, b_label, b_pid, b_bg, b_cnt, b_part, b_pframe, b_err;
    const long long cpx = (long long)chunk * frame_px;
    if ((e = b_mask.ensure(cpx)) != cudaSuccess || (e = b_label.ensure(cpx * 4)) != cudaSuccess ||
        (e = b_pid.ensure(cpx * 4)) != cudaSuccess || (e = b_bg.ensure((size_t)chunk * 16)) != cudaSuccess ||
        (e = b_cnt.ensure((size_t)chunk * 4)) != cudaSuccess || (e = b_err.ensure(4)) != cudaSuccess)
        return fail(LOC_E_NOMEM, std::string("finder scratch: ") + cudaGetErrorString(e));
    uint8_t *mask = (uint8_t *)b_mask.p;
    int *label = (int *)b_label.p, *pid = (int *)b_pid.p, *fcount = (int *)b_cnt.p, *err = (int *)b_err.p;
    unsigned long long *bg_sum = (unsigned long long *)b_bg.p, *bg_cnt = bg_sum + chunk;
    cudaMemsetAsync(err, 0, 4, st);
    std::vector<int> hcount(chunk), hoff(chunk);
    long long total = 0;
    for (int f0 = 0; f0 < n_frames; f0 += chunk) {
        const int nf = std::min(chunk, n_frames - f0);
        const long long npx = (long long)nf * frame_px;
        const uint16_t *fr = d_frames + (size_t)f0 * frame_px;
        cudaMemsetAsync(bg_sum, 0, (size_t)chunk * 16, st);
        const dim3 grid((n_rows + kTX - 1) / kTX, (n_cols + kTY - 1) / kTY, nf);
        const size_t smem = (size_t)(kTX + 2 * half) * (kTY + 2 * half) * sizeof(uint16_t);
        k_glrt<<<grid, dim3(kTX, kTY), smem, st>>>(fr, n_rows, n_cols, ws, npix, sumsq, thr, mask, label, bg_sum,
                                                  bg_cnt);
        const int eb = (int)std::min<long long>((npx + 255) / 256, 148 * 16);
        k_union<<<eb, 256, 0, st>>>(mask, label, n_rows, n_cols, npx, err);
        k_flatten<<<eb, 256, 0, st>>>(mask, label, npx);
        k_count_roots<<<nf, 512, 0, st>>>(mask, label, (int)frame_px, fcount);
        if ((e = cudaMemcpyAsync(hcount.data(), fcount, (size_t)nf * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return fail(LOC_E_CUDA, std::string("finder: ") + cudaGetErrorString(e));
        int np = 0;
        for (int i = 0; i < nf; ++i) {
            hoff[i] = np;
            np += hcount[i];
        }
        if (np > 0) {
            const size_t part_bytes = (size_t)np * (8 + 8 + 4 + 4);
            if ((e = b_part.ensure(part_bytes)) != cudaSuccess || (e = b_pframe.ensure((size_t)np * 4)) != cudaSuccess)
                return fail(LOC_E_NOMEM, std::string("finder particles: ") + cudaGetErrorString(e));
            unsigned long long *sx = (unsigned long long *)b_part.p, *sy = sx + np;
            unsigned int *cnt = (unsigned int *)(sy + np), *mx = cnt + np;
            int *pframe = (int *)b_pframe.p;
            cudaMemsetAsync(b_part.p, 0, part_bytes, st);
            cudaMemcpyAsync(fcount, hoff.data(), (size_t)nf * 4, cudaMemcpyHostToDevice, st);
            k_assign<<<nf, 1024, 0, st>>>(mask, label, (int)frame_px, fcount, pid, pframe, f0);
            k_accumulate<<<eb, 256, 0, st>>>(mask, label, pid, fr, n_rows, (int)frame_px, npx, sx, sy, cnt, mx);
            k_emit<<<(np + 255) / 256, 256, 0, st>>>(np, pframe, f0, sx, sy, cnt, mx, bg_sum, bg_cnt, d_cands, total,
                                                     max_cands);
        }
        total += np;
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(LOC_E_CUDA, std::string("finder launch: ") + cudaGetErrorString(e));
        // the host vectors are reused by the next chunk: finish this one first
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            return fail(LOC_E_CUDA, std::string("finder: ") + cudaGetErrorString(e));
    }
    int herr = 0;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    if (herr) return fail(LOC_E_CUDA, "finder: component linking did not settle");
    return (long)total;
}
