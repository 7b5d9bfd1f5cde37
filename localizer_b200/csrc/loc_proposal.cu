// Learned start proposal for the Gaussian LM fits.
//
// A small convolutional network maps the 11 x 11 pixel window around each
// candidate to a starting parameter vector for the solver (amplitude,
// width(s), position, correlation, offset in the method's own order), so that
// the Levenberg-Marquardt iteration starts near its solution instead of at
// the finder's centroid and the reference's default width. The solver's own
// cold start stays the fallback: a proposal is taken only when its residual
// over the candidate's ROI is not worse than the cold start's, and warm fits
// the fit pipeline judges unreliable are re-run cold.
//
// Network (valid 3x3 convolutions, ReLU after each):
//   window 1x11x11 -> conv1 16x9x9 -> conv2 32x7x7 -> conv3 32x5x5 -> linear(800 -> P)
// The three convolutions run on the 5th-generation tensor cores
// (tcgen05.mma, BF16 operands, FP32 accumulation in tensor memory): conv1
// (one input channel) as an im2col GEMM with its 9 taps padded to K = 16,
// conv2 and conv3 (K = 144 and 288) as implicit GEMMs; the linear head runs on
// the CUDA cores in FP32. The window pixels of a CTA's next group are loaded
// into registers while the current group is processed.
//
// Implicit GEMM without im2col: activations of R windows live in shared
// memory on a 9-wide grid, one row per grid position (81 rows per window,
// channels along K). Output position p of a valid 3x3 convolution reads input
// rows p + dy*9 + dx, so each of the nine taps is the same K-major operand
// shifted by dy*9 + dx rows, i.e. a descriptor whose start address moves by
// 16 bytes per row. Rows that fall off the valid output area of a window are
// computed and discarded (conv2: 49 of 81 rows valid, conv3: 25 of 81).
//
// Input normalisation per window: b0 = mean of the 40 border pixels,
// s0 = max(mean of the central 3x3 - b0, 10), v = (pixel - b0) / s0.
// Outputs are mapped to parameters as A = s0 exp(o), width = 1.5 exp(o),
// position = window centre + o, correlation = o (clamped to +-0.9),
// offset = b0 + s0 o. The window centre is the candidate position rounded to
// the nearest pixel.
//
// Training (hand-written kernels): the forward kernel saves its activations,
// k_prop_bwd back-propagates a weighted squared error against targets mapped
// the same way (FP32 on the CUDA cores, with the BF16-rounded weights the
// forward used), k_adam updates the FP32 master weights and k_pack re-packs
// the BF16 tensor-core operands.
#include "../../include/localizer_b200.h"
#include "loc_device.cuh"
#include "loc_proposal.cuh"
#include "loc_tc.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <math_constants.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace locb {
int record_error_fixed(int code, const char *msg);
}

namespace locb {
namespace {

constexpr int kWin = 11, kWin2 = 121;
constexpr int kR = 8;                             // windows per CTA iteration
constexpr int kRows = 81 * kR;                    // activation grid rows per iteration
constexpr int kTiles = (kRows + 127) / 128;       // M = 128 tiles
constexpr int kRowsAlloc = kTiles * 128 + 24;     // + largest tap shift (20), multiple of 8
constexpr uint32_t kLBO = kRowsAlloc * 16;        // bytes between 8-channel chunks
constexpr uint32_t kTmemCols = kTiles * 32 <= 32 ? 32 : kTiles * 32 <= 64 ? 64 : kTiles * 32 <= 128 ? 128 : 256;
static_assert(kTiles * 32 <= (int)kTmemCols, "accumulators must fit in tensor memory");
constexpr int kThreads = 256;               // 8 warps: two per TMEM lane quarter
constexpr int kCtasPerSm = 2;               // two CTAs per SM overlap tensor and CUDA-core phases
constexpr int kBwdThreads = 256;            // backward pass block (its conv1 step uses 160 threads)
constexpr float kSigmaRef = 1.5f;
constexpr int kWaitLimit = 1 << 20;

// FP32 master weight layout
constexpr int kW1 = 0;        // [16][9]       conv1 (out channel, tap)
constexpr int kB1 = 144;      // [16]
constexpr int kW2 = 160;      // [32][16][9]   conv2 (out, in, tap)
constexpr int kB2 = 4768;     // [32]
constexpr int kW3 = 4800;     // [32][32][9]   conv3
constexpr int kB3 = 14016;    // [32]
constexpr int kWH = 14048;    // [P][32][25]   head (output, channel, position)
__host__ __device__ constexpr int weight_count(int nout) { return kWH + nout * 800 + nout; }

// packed BF16 operands, K-major chunks: conv2 [tap][chunk 2][out 32][8], conv3 [tap][chunk 4][out 32][8],
// conv1 [chunk 2][out 16][8] (K = tap, taps 9..15 zero)
constexpr int kW2P = 9 * 2 * 32 * 8;
constexpr int kW3P = 9 * 4 * 32 * 8;
constexpr int kW1P = 2 * 16 * 8;
constexpr int kWP = kW2P + kW3P + kW1P;

// Raw pixels staged per window: a 15 x 15 region centred like the window,
// which holds the 11 x 11 network window at offset (2, 2) and, for ROI
// half-widths up to 6, the whole ROI the start check evaluates.
constexpr int kReg = 15, kReg2 = kReg * kReg;
constexpr int kRegOff = (kReg - kWin) / 2;

// One window's record, filled one group ahead: region origin in the frame,
// frame (or ROI index; -1: no window), the candidate's ROI half-width
// (-1: rejected before the fit) and the fields the start check needs.
struct WinRec {
    double cx, cy;
    float intensity, background;
    int x0, y0, frame, r;
};

// forward kernel shared memory (bytes)
constexpr int SO_ACT1 = 0;
constexpr int SO_ACT2 = SO_ACT1 + 2 * (int)kLBO;
constexpr int SO_WP = SO_ACT2 + 4 * (int)kLBO;
constexpr int SO_V = SO_WP + kWP * 2;
constexpr int SO_W1 = SO_V + kR * kWin2 * 4;      // w1 + b1
constexpr int SO_B23 = SO_W1 + 160 * 4;           // b2 + b3
constexpr int SO_HACC = SO_B23 + 64 * 4;          // head outputs (head weights are read through L1)
constexpr int SO_STAT = SO_HACC + kR * 8 * 4;
constexpr int SO_RAW = SO_STAT + kR * 4 * 4;       // raw pixel regions of the current group
constexpr int SO_WIN = SO_RAW + ((kR * kReg2 * 2 + 15) / 16) * 16;   // window records: [current, next][kR]
constexpr int SO_BAR = SO_WIN + 2 * kR * (int)sizeof(WinRec);
constexpr int SO_MISC = SO_BAR + 8;
constexpr int kSmemFwd = SO_MISC + 16;
static_assert(kCtasPerSm * (kSmemFwd + 1024) <= 228 * 1024, "forward CTAs per SM: shared memory");
static_assert(kCtasPerSm * (int)kTmemCols <= 512, "forward CTAs per SM: tensor memory");
static_assert(SO_ACT2 % 16 == 0 && SO_WP % 16 == 0 && SO_V % 16 == 0 && SO_WIN % 8 == 0 && SO_BAR % 8 == 0,
              "alignment");

constexpr uint32_t kIdesc = tc::idesc_bf16_f32<128, 32>();
constexpr uint32_t kIdesc1 = tc::idesc_bf16_f32<128, 16>();
constexpr int kPre = (kR * kReg2 + kThreads - 1) / kThreads;   // prefetched region pixels per thread
constexpr int kA3Stride = 808;   // floats per window of conv3 output in shared memory (800 + bank padding)
static_assert(kR * kA3Stride * 4 <= 4 * (int)kLBO, "conv3 outputs fit in the conv2 activation buffer");

// output roles: 0 amplitude, 1 width, 2 x, 3 y, 4 correlation, 5 offset
template <int NOUT> __host__ __device__ constexpr int role(int j)
{
    return NOUT == 4 ? (j == 0 ? 0 : j == 1 ? 2 : j == 2 ? 3 : 5)
         : NOUT == 5 ? (j == 0 ? 0 : j == 1 ? 1 : j == 2 ? 2 : j == 3 ? 3 : 5)
                     : (j == 0 ? 0 : j <= 2 ? 1 : j == 3 ? 2 : j == 4 ? 3 : j == 5 ? 4 : 5);
}

// raw output -> parameter, positions relative to the window centre
template <int NOUT> __device__ __forceinline__ float out_to_param(int j, float o, float b0, float s0)
{
    switch (role<NOUT>(j)) {
    case 0: return s0 * __expf(fminf(fmaxf(o, -8.f), 8.f));
    case 1: return kSigmaRef * __expf(fminf(fmaxf(o, -3.f), 3.f));
    case 2: case 3: return o;
    case 4: return fminf(fmaxf(o, -0.9f), 0.9f);
    default: return b0 + s0 * o;
    }
}

// parameter label -> training target (inverse of out_to_param inside the clamps)
template <int NOUT> __device__ __forceinline__ float param_to_target(int j, float p, float b0, float s0)
{
    switch (role<NOUT>(j)) {
    case 0: return logf(fmaxf(p, 1.0f) / s0);
    case 1: return logf(fmaxf(p, 0.05f) / kSigmaRef);
    case 2: case 3: case 4: return p;
    default: return (p - b0) / s0;
    }
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// The method's Gaussian of a parameter vector (amplitude, width(s), centre,
// correlation, offset in the method's order) as
// A exp(qa u^2 + qb u w + qc w^2) + b with u = i - x0, w = j - y0, so that
// evaluating it over a ROI takes no division per pixel
struct GaussQ {
    float A, b, qa, qb, qc, x0, y0;
};
template <int P> __device__ __forceinline__ GaussQ gauss_q(const float (&t)[7], float w0)
{
    if constexpr (P == 5) {
        const float h = -0.5f / (t[1] * t[1]);
        return GaussQ{t[0], t[4], h, 0.f, h, t[2], t[3]};
    } else if constexpr (P == 4) {
        const float h = -0.5f / (w0 * w0);
        return GaussQ{t[0], t[3], h, 0.f, h, t[1], t[2]};
    } else {
        // exponent -(u^2/sx^2 - 2 rho u w/(sx sy) + w^2/sy^2) / (2 (1 - rho^2))
        const float k = 1.f / (1.f - t[5] * t[5]);
        return GaussQ{t[0], t[6], -0.5f * k / (t[1] * t[1]), k * t[5] / (t[1] * t[2]), -0.5f * k / (t[2] * t[2]),
                      t[3], t[4]};
    }
}
__device__ __forceinline__ float gauss_at(const GaussQ &g, float i, float j)
{
    const float u = i - g.x0, w = j - g.y0;
    return g.A * __expf(fmaf(g.qa * u, u, fmaf(g.qb * u, w, g.qc * w * w))) + g.b;
}

struct FwdArgs {
    // MODE 0: ROI stack (n windows of 11 x 11, x fastest), optional gather index
    const uint16_t *rois;
    const int *index;
    // MODE 1: frames + candidates (fit pipeline)
    const uint16_t *frames;
    long long frame_px;
    int n_rows, n_cols;
    const Cand *cands;
    const int *cls;
    int n;
    const float *w;
    const void *wp;
    // MODE 0 outputs: raw head outputs, optional saved activations for training
    float *out;
    float *save_v;             // n x 121 normalised window
    float *save_stat;          // n x 2 (b0, s0)
    __nv_bfloat16 *save_a1;    // n x 81 x 16
    __nv_bfloat16 *save_a2;    // n x 81 x 32 (valid 7 x 7 positions written)
    float *save_a3;            // n x 25 x 32
    // MODE 1 outputs
    float w0;
    float *init;
    unsigned long long *n_warm;
    int *err;
};

template <int NOUT, int MODE>
__global__ void __launch_bounds__(kThreads, kCtasPerSm) k_prop_fwd(FwdArgs a)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + SO_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + SO_MISC);
    int *wcount = reinterpret_cast<int *>(sm + SO_MISC + 4);
    float *v = reinterpret_cast<float *>(sm + SO_V);
    float *w1 = reinterpret_cast<float *>(sm + SO_W1);
    float *b23 = reinterpret_cast<float *>(sm + SO_B23);
    const float *wh = a.w + kWH;
    float *hacc = reinterpret_cast<float *>(sm + SO_HACC);
    float *stat = reinterpret_cast<float *>(sm + SO_STAT);

    // weights into shared memory
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(a.wp);
        uint4 *dst = reinterpret_cast<uint4 *>(sm + SO_WP);
        for (int k = tid; k < kWP * 2 / 16; k += kThreads) dst[k] = src[k];
        for (int k = tid; k < 160; k += kThreads) w1[k] = a.w[kW1 + k];
        for (int k = tid; k < 32; k += kThreads) {
            b23[k] = a.w[kB2 + k];
            b23[32 + k] = a.w[kB3 + k];
        }
        for (int k = tid; k < kR * 8; k += kThreads) hacc[k] = 0.f;
        // padding rows past the last window: read only by discarded outputs,
        // zeroed so that they hold finite values
        const uint4 z = make_uint4(0, 0, 0, 0);
        constexpr int pad = kRowsAlloc - kRows;
        for (int k = tid; k < 6 * pad; k += kThreads) {
            const int c = k / pad, row = kRows + k % pad;
            *reinterpret_cast<uint4 *>(sm + (c < 2 ? SO_ACT1 : SO_ACT2) + (c < 2 ? c : c - 2) * kLBO + row * 16) = z;
        }
        if (tid == 0) *wcount = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(tslot, kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    uint32_t phase = 0;
    bool failed = false;
    // epilogues: a warp reads its TMEM lane quarter; with more than 4 warps,
    // the warps of one quarter split the accumulator columns between them
    constexpr int kEpiSets = kThreads / 128;
    static_assert(kEpiSets * 128 == kThreads && (kEpiSets == 1 || kEpiSets == 2), "epilogue warp sets");
    const int q = warp & 3, eset = warp >> 2;
    const uint32_t t_lane = (uint32_t)(32 * q) << 16;
    const float *bh = wh + NOUT * 800;

    const int ngroups = (a.n + kR - 1) / kR;
    // window records, kept by the first kR threads: the candidate data of
    // group g is loaded into registers (load_records) one group before
    // store_records writes it to win_next, so the loads' latency is hidden
    WinRec *win_cur = reinterpret_cast<WinRec *>(sm + SO_WIN);
    WinRec *win_next = win_cur + kR;
    uint16_t *raw = reinterpret_cast<uint16_t *>(sm + SO_RAW);
    int rec_src = -1;   // MODE 0: ROI index; MODE 1: the candidate's ROI half-width (-1: none)
    Cand rec_c{};
    auto load_records = [&](int g) {
        rec_src = -1;
        if (tid < kR) {
            const int item = g * kR + tid;
            if (g < ngroups && item < a.n) {
                if constexpr (MODE == 0) {
                    rec_src = a.index ? a.index[item] : item;
                } else {
                    rec_src = a.cls[item];
                    rec_c = a.cands[item];
                }
            }
        }
    };
    auto store_records = [&]() {
        if (tid < kR) {
            WinRec w{0.0, 0.0, 0.f, 0.f, 0, 0, -1, -1};
            if constexpr (MODE == 0) {
                w.frame = rec_src;
            } else if (rec_src >= 0) {
                w.cx = rec_c.x;
                w.cy = rec_c.y;
                w.intensity = (float)rec_c.intensity;
                w.background = (float)rec_c.background;
                w.x0 = (int)floor(rec_c.x + 0.5) - 5 - kRegOff;
                w.y0 = (int)floor(rec_c.y + 0.5) - 5 - kRegOff;
                w.frame = rec_c.frame;
                w.r = rec_src;
            }
            win_next[tid] = w;
        }
    };
    // the raw region pixels of the group whose records are in win_next, into
    // registers (consumed one group later, so the loads' latency is hidden
    // behind the current group's work); pixels outside the frame repeat its
    // edge, and a ROI-stack window (training) fills only the inner 11 x 11
    uint16_t pre[kPre];
    auto fetch_windows = [&]() {
#pragma unroll
        for (int i = 0; i < kPre; ++i) {
            const int k = tid + i * kThreads;
            uint16_t val = 0;
            if (k < kR * kReg2) {
                const int rr = k / kReg2, px = k - rr * kReg2;
                const int jy = px / kReg, ix = px - jy * kReg;
                const int fr = win_next[rr].frame;
                if (fr >= 0) {
                    if constexpr (MODE == 0) {
                        const int wx = ix - kRegOff, wy = jy - kRegOff;
                        if (wx >= 0 && wx < kWin && wy >= 0 && wy < kWin)
                            val = __ldg(a.rois + (size_t)fr * kWin2 + wx + wy * kWin);
                    } else {
                        const int xx = min(max(win_next[rr].x0 + ix, 0), a.n_rows - 1);
                        const int yy = min(max(win_next[rr].y0 + jy, 0), a.n_cols - 1);
                        val = __ldg(a.frames + (size_t)fr * (size_t)a.frame_px + xx + (size_t)yy * a.n_rows);
                    }
                }
            }
            pre[i] = val;
        }
    };
    load_records(blockIdx.x);
    store_records();
    load_records(blockIdx.x + (int)gridDim.x);
    __syncthreads();
    fetch_windows();
    __syncthreads();   // every thread has read win_next before the loop rewrites it
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int base = g * kR;
        // ---- 1. raw regions (counts) from the prefetched registers ----
#pragma unroll
        for (int i = 0; i < kPre; ++i) {
            const int k = tid + i * kThreads;
            if (k < kR * kReg2) raw[k] = pre[i];
        }
        if (tid < kR) win_cur[tid] = win_next[tid];   // this group's record, before the next one replaces it
        store_records();                            // group g + grid, loaded one group ago
        load_records(g + 2 * (int)gridDim.x);
        __syncthreads();
        // the 11 x 11 window inside a region
        auto window_px = [&](int rr, int px) -> float {
            const int jy = px / kWin, ix = px - jy * kWin;
            return (float)raw[rr * kReg2 + (jy + kRegOff) * kReg + ix + kRegOff];
        };
        // ---- 2. normalisation statistics, one warp per window ----
        for (int rr = warp; rr < kR; rr += kThreads / 32) {
            float sb = 0.f, sc = 0.f;
            for (int px = lane; px < kWin2; px += 32) {
                const int jy = px / kWin, ix = px - jy * kWin;
                const float x = window_px(rr, px);
                if (jy == 0 || jy == kWin - 1 || ix == 0 || ix == kWin - 1) sb += x;
                if (jy >= 4 && jy <= 6 && ix >= 4 && ix <= 6) sc += x;
            }
            sb = warp_sum(sb);
            sc = warp_sum(sc);
            if (lane == 0) {
                const float b0 = sb / 40.f;
                const float s0 = fmaxf(sc / 9.f - b0, 10.f);
                stat[rr * 4 + 0] = b0;
                stat[rr * 4 + 1] = s0;
                stat[rr * 4 + 2] = 1.f / s0;
            }
        }
        __syncthreads();
        fetch_windows();   // the next group's pixels, in flight during this group's work
        // normalised pixels, rounded to BF16 (conv1's tensor-core operand)
        for (int k = tid; k < kR * kWin2; k += kThreads) {
            const int rr = k / kWin2;
            const float nv =
                __bfloat162float(__float2bfloat16_rn((window_px(rr, k - rr * kWin2) - stat[rr * 4]) * stat[rr * 4 + 2]));
            v[k] = nv;
            if constexpr (MODE == 0) {
                if (a.save_v && base + rr < a.n) a.save_v[(size_t)base * kWin2 + k] = nv;
            }
        }
        if constexpr (MODE == 0) {
            if (a.save_stat && tid < kR && base + tid < a.n) {
                a.save_stat[(size_t)(base + tid) * 2 + 0] = stat[tid * 4 + 0];
                a.save_stat[(size_t)(base + tid) * 2 + 1] = stat[tid * 4 + 1];
            }
        }
        __syncthreads();
        // ---- 3. conv1 on the tensor cores: im2col rows (9 taps + 7 zeros, BF16)
        // in the conv2 activation buffer (free until the conv2 epilogue) ----
        for (int m = tid; m < kTiles * 128; m += kThreads) {
            uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0;
            if (m < kRows) {
                const int rr = m / 81, pos = m - rr * 81, iy = pos / 9, ix = pos - iy * 9;
                const float *wv = v + rr * kWin2 + iy * kWin + ix;
                c0 = make_uint4(pack_bf16x2(wv[0], wv[1]), pack_bf16x2(wv[2], wv[kWin]),
                                pack_bf16x2(wv[kWin + 1], wv[kWin + 2]), pack_bf16x2(wv[2 * kWin], wv[2 * kWin + 1]));
                c1.x = pack_bf16x2(wv[2 * kWin + 2], 0.f);
            }
            *reinterpret_cast<uint4 *>(sm + SO_ACT2 + m * 16) = c0;
            *reinterpret_cast<uint4 *>(sm + SO_ACT2 + kLBO + m * 16) = c1;
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t cb = tc::smem_addr(sm + SO_ACT2), w1 = tc::smem_addr(sm + SO_WP + (kW2P + kW3P) * 2);
            const uint64_t bd = tc::smem_desc(w1, 256, 128);
            for (int i = 0; i < kTiles; ++i)
                tc::mma_bf16(tmem + (uint32_t)i * 32u, tc::smem_desc(cb + (uint32_t)i * 128u * 16u, kLBO, 128), bd,
                             kIdesc1, 0u);
            tc::mma_commit(bar);
        }
        __syncwarp();
        if (!tc::mbar_wait(bar, phase, kWaitLimit)) failed = true;
        phase ^= 1u;
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        tc::fence_after_sync();
        // conv1 epilogue: bias, ReLU, BF16 -> act1 (K-major chunks)
        for (int i = eset; i < kTiles; i += kEpiSets) {
            float acc[16];
            tc::tmem_ld16(tmem + t_lane + (uint32_t)(i * 32), acc);
            tc::tmem_ld_wait();
            const int m = i * 128 + 32 * q + lane;
            if (m < kRows) {
                uint32_t pk[8];
#pragma unroll
                for (int c = 0; c < 16; c += 2)
                    pk[c / 2] = pack_bf16x2(fmaxf(acc[c] + w1[144 + c], 0.f), fmaxf(acc[c + 1] + w1[144 + c + 1], 0.f));
                const uint4 c0 = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                const uint4 c1 = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                *reinterpret_cast<uint4 *>(sm + SO_ACT1 + m * 16) = c0;
                *reinterpret_cast<uint4 *>(sm + SO_ACT1 + kLBO + m * 16) = c1;
                if constexpr (MODE == 0) {
                    const int rr = m / 81, pos = m - rr * 81;
                    if (a.save_a1 && base + rr < a.n) {
                        uint4 *d = reinterpret_cast<uint4 *>(a.save_a1 + ((size_t)(base + rr) * 81 + pos) * 16);
                        d[0] = c0;
                        d[1] = c1;
                    }
                }
            }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        // ---- 4. conv2 on the tensor cores: 9 shifted K = 16 blocks per tile ----
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a1 = tc::smem_addr(sm + SO_ACT1), w2 = tc::smem_addr(sm + SO_WP);
            for (int i = 0; i < kTiles; ++i)
#pragma unroll
                for (int t = 0; t < 9; ++t) {
                    const uint32_t sh = (uint32_t)((t / 3) * 9 + t % 3);
                    const uint64_t ad = tc::smem_desc(a1 + ((uint32_t)i * 128u + sh) * 16u, kLBO, 128);
                    const uint64_t bd = tc::smem_desc(w2 + (uint32_t)t * 1024u, 512, 128);
                    tc::mma_bf16(tmem + (uint32_t)i * 32u, ad, bd, kIdesc, t > 0 ? 1u : 0u);
                }
            tc::mma_commit(bar);
        }
        __syncwarp();
        if (!tc::mbar_wait(bar, phase, kWaitLimit)) failed = true;
        phase ^= 1u;
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        tc::fence_after_sync();
        // ---- 5. conv2 epilogue: bias, ReLU, BF16 -> act2 ----
        for (int i = 0; i < kTiles; ++i)
        for (int h = eset; h < 2; h += kEpiSets) {
            float acc[16];
            tc::tmem_ld16(tmem + t_lane + (uint32_t)(i * 32 + 16 * h), acc);
            tc::tmem_ld_wait();
            const int m = i * 128 + 32 * q + lane;
            if (m < kRows) {
                uint32_t pk[8];
#pragma unroll
                for (int c = 0; c < 16; c += 2)
                    pk[c / 2] = pack_bf16x2(fmaxf(acc[c] + b23[16 * h + c], 0.f),
                                            fmaxf(acc[c + 1] + b23[16 * h + c + 1], 0.f));
                const uint4 c0 = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                const uint4 c1 = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                *reinterpret_cast<uint4 *>(sm + SO_ACT2 + (2 * h) * kLBO + m * 16) = c0;
                *reinterpret_cast<uint4 *>(sm + SO_ACT2 + (2 * h + 1) * kLBO + m * 16) = c1;
                if constexpr (MODE == 0) {
                    const int rr = m / 81, pos = m - rr * 81;
                    if (a.save_a2 && base + rr < a.n && pos / 9 < 7 && pos % 9 < 7) {
                        uint4 *d =
                            reinterpret_cast<uint4 *>(a.save_a2 + ((size_t)(base + rr) * 81 + pos) * 32 + 16 * h);
                        d[0] = c0;
                        d[1] = c1;
                    }
                }
            }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        // ---- 6. conv3 on the tensor cores: 9 taps x 2 K = 16 blocks per tile ----
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a2 = tc::smem_addr(sm + SO_ACT2), w3 = tc::smem_addr(sm + SO_WP + kW2P * 2);
            for (int i = 0; i < kTiles; ++i)
#pragma unroll
                for (int t = 0; t < 9; ++t) {
                    const uint32_t sh = (uint32_t)((t / 3) * 9 + t % 3);
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const uint64_t ad =
                            tc::smem_desc(a2 + (uint32_t)kk * 2u * kLBO + ((uint32_t)i * 128u + sh) * 16u, kLBO, 128);
                        const uint64_t bd = tc::smem_desc(w3 + (uint32_t)t * 2048u + (uint32_t)kk * 1024u, 512, 128);
                        tc::mma_bf16(tmem + (uint32_t)i * 32u, ad, bd, kIdesc, (t | kk) ? 1u : 0u);
                    }
                }
            tc::mma_commit(bar);
        }
        __syncwarp();
        if (!tc::mbar_wait(bar, phase, kWaitLimit)) failed = true;
        phase ^= 1u;
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        tc::fence_after_sync();
        // ---- 7. conv3 epilogue: bias, ReLU -> a3 in shared memory (the
        // activation buffers are free once the conv3 MMAs have completed) ----
        float *a3s = reinterpret_cast<float *>(sm + SO_ACT2);   // [kR][kA3Stride], (channel, position)
        for (int i = 0; i < kTiles; ++i)
        for (int h = eset; h < 2; h += kEpiSets) {
            float acc[16];
            tc::tmem_ld16(tmem + t_lane + (uint32_t)(i * 32 + 16 * h), acc);
            tc::tmem_ld_wait();
            const int m = i * 128 + 32 * q + lane;
            const int rr = m / 81, pos = m - rr * 81, oy = pos / 9, ox = pos - oy * 9;
            if (m < kRows && oy < 5 && ox < 5) {
                const int p25 = oy * 5 + ox;
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int ch = 16 * h + c;
                    acc[c] = fmaxf(acc[c] + b23[32 + ch], 0.f);
                    a3s[rr * kA3Stride + ch * 25 + p25] = acc[c];
                }
                if constexpr (MODE == 0) {
                    if (a.save_a3 && base + rr < a.n) {
                        float4 *d =
                            reinterpret_cast<float4 *>(a.save_a3 + ((size_t)(base + rr) * 25 + p25) * 32 + 16 * h);
#pragma unroll
                        for (int c = 0; c < 16; c += 4)
                            d[c / 4] = make_float4(acc[c], acc[c + 1], acc[c + 2], acc[c + 3]);
                    }
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        // ---- head: kTPW threads per window, each over every kTPW-th feature ----
        {
            constexpr int kTPW = kThreads / kR;
            static_assert(kTPW * kR == kThreads && kTPW <= 32 && (kTPW & (kTPW - 1)) == 0, "head mapping");
            const int rr = tid / kTPW, sub = tid % kTPW;
            const float *x = a3s + rr * kA3Stride;
            float part[NOUT];
#pragma unroll
            for (int j = 0; j < NOUT; ++j) part[j] = 0.f;
            for (int f = sub; f < 800; f += kTPW) {
                const float xv = x[f];
#pragma unroll
                for (int j = 0; j < NOUT; ++j) part[j] = fmaf(wh[j * 800 + f], xv, part[j]);
            }
#pragma unroll
            for (int j = 0; j < NOUT; ++j) {
                float t = part[j];
#pragma unroll
                for (int o = kTPW / 2; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (sub == 0) hacc[rr * 8 + j] = t;
            }
        }
        __syncthreads();
        // ---- 8. outputs ----
        if constexpr (MODE == 0) {
            for (int k = tid; k < kR * NOUT; k += kThreads) {
                const int rr = k / NOUT, j = k - rr * NOUT;
                if (base + rr < a.n) a.out[(size_t)(base + rr) * NOUT + j] = hacc[rr * 8 + j] + bh[j];
            }
        } else {
            // start check: proposal vs cold start, residual over the ROI
            constexpr int P = NOUT;
            constexpr int IX = P == 5 ? 2 : P == 4 ? 1 : 3;
            for (int rr = warp; rr < kR; rr += kThreads / 32) {
                const int item = base + rr;
                if (item >= a.n) continue;
                float *dst = a.init + (size_t)item * P;
                const WinRec &c = win_cur[rr];
                const int r = c.r;
                if (r < 0) {
                    if (lane == 0) dst[0] = CUDART_NAN_F;
                    continue;
                }
                const int xo = (int)floor(c.cx - (double)r), yo = (int)floor(c.cy - (double)r);
                const int cx = (int)floor(c.cx + 0.5), cy = (int)floor(c.cy + 0.5);
                const float b0 = stat[rr * 4 + 0], s0 = stat[rr * 4 + 1];
                float tw[7] = {0, 0, 0, 0, 0, 0, 0}, tcold[7] = {0, 0, 0, 0, 0, 0, 0};
                bool ok = true;
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    float p = out_to_param<NOUT>(j, hacc[rr * 8 + j] + bh[j], b0, s0);
                    if (j == IX) p += (float)(cx - xo);
                    if (j == IX + 1) p += (float)(cy - yo);
                    tw[j] = p;
                    ok = ok && isfinite(p);
                }
                const float side = (float)(2 * r);
                ok = ok && tw[0] > 0.f && tw[IX] >= 0.f && tw[IX] <= side && tw[IX + 1] >= 0.f && tw[IX + 1] <= side;
                const float xl = (float)(c.cx - (double)xo), yl = (float)(c.cy - (double)yo);
                if constexpr (P == 5) {
                    tcold[0] = c.intensity; tcold[1] = a.w0; tcold[2] = xl; tcold[3] = yl; tcold[4] = c.background;
                } else if constexpr (P == 4) {
                    tcold[0] = c.intensity; tcold[1] = xl; tcold[2] = yl; tcold[3] = c.background;
                } else {
                    tcold[0] = c.intensity; tcold[1] = a.w0; tcold[2] = a.w0; tcold[3] = xl;
                    tcold[4] = yl; tcold[5] = 0.f; tcold[6] = c.background;
                }
                const GaussQ gw = gauss_q<P>(tw, a.w0), gc = gauss_q<P>(tcold, a.w0);
                const int s = 2 * r + 1;
                // the ROI's origin inside the staged region: inside it for
                // half-widths up to 6, else the ROI is read from the frame
                const int ox = xo - c.x0, oy = yo - c.y0;
                const bool staged = ox >= 0 && oy >= 0 && ox + s <= kReg && oy + s <= kReg;
                const uint16_t *rg = raw + rr * kReg2 + ox + oy * kReg;
                const uint16_t *fb = a.frames + (size_t)c.frame * (size_t)a.frame_px + xo + (size_t)yo * a.n_rows;
                float cw = 0.f, cc = 0.f;
                for (int k = lane; k < s * s; k += 32) {
                    const int j = k / s, i = k - j * s;
                    const float d = staged ? (float)rg[i + j * kReg] : (float)__ldg(fb + i + (size_t)j * a.n_rows);
                    const float ew = gauss_at(gw, (float)i, (float)j) - d;
                    const float ec = gauss_at(gc, (float)i, (float)j) - d;
                    cw = fmaf(ew, ew, cw);
                    cc = fmaf(ec, ec, cc);
                }
                cw = warp_sum(cw);
                cc = warp_sum(cc);
                const bool warm = ok && isfinite(cw) && !(cw > cc);
                if (lane == 0) {
                    if (warm) {
#pragma unroll
                        for (int j = 0; j < P; ++j)
                            dst[j] = tw[j] + (j == IX ? (float)xo : (j == IX + 1 ? (float)yo : 0.f));
                        atomicAdd(wcount, 1);
                    } else {
                        dst[0] = CUDART_NAN_F;
                    }
                }
            }
        }
        __syncthreads();
        for (int k = tid; k < kR * 8; k += kThreads) hacc[k] = 0.f;
    }
    // teardown: every tensor-core operation has completed (each batch waited
    // on its commit), or a wait ran out and the loop left early
    tc::fence_before_sync();
    __syncthreads();
    if (failed) {
        // give the MMAs still in flight a bounded chance to land before freeing TMEM
        tc::mbar_wait(bar, phase ^ 1u, kWaitLimit);
        if (tid == 0) atomicExch(a.err, 1);
    }
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
    if constexpr (MODE == 1) {
        if (tid == 0 && *wcount > 0 && a.n_warm) atomicAdd(a.n_warm, (unsigned long long)*wcount);
    }
}

// ---------------------------------------------------------------------------
// Backward pass (FP32, CUDA cores). One CTA walks a strided subset of the
// batch, accumulating weight gradients in shared memory, then adds them to the
// global gradient once.
// ---------------------------------------------------------------------------
struct BwdArgs {
    int n;
    const int *index;          // label gather index (same as the forward's), or NULL
    const float *labels;       // N x P parameter labels, positions relative to the window centre
    const float *lam;          // P loss weights (device)
    const float *w;            // master weights (W2/W3 rounded to BF16 as the forward used them)
    const float *out;          // n x P
    const float *save_v, *save_stat;
    const __nv_bfloat16 *save_a1, *save_a2;
    const float *save_a3;
    float *grad;               // weight_count(P), accumulated
    float *loss;               // accumulated sum over the batch of sum_j lam_j (o_j - t_j)^2
    float inv_batch;
};

template <int NOUT> struct BwdSmem {
    static constexpr int NW = weight_count(NOUT);
    static constexpr int G = 0;                  // NW gradient accumulators
    static constexpr int W2 = G + NW;            // 4608 (BF16-rounded)
    static constexpr int W3 = W2 + 4608;         // 9216
    static constexpr int V = W3 + 9216;          // 121
    static constexpr int A1 = V + 124;           // [16][81]
    static constexpr int A2 = A1 + 16 * 81;      // [32][49]
    static constexpr int Z3 = A2 + 32 * 49;      // [32][25]  a3, then dz3
    static constexpr int Z2 = Z3 + 32 * 25;      // [32][49]  dz2
    static constexpr int Z1 = Z2 + 32 * 49;      // [16][81]  dz1
    static constexpr int DO = Z1 + 16 * 81;      // [8]
    static constexpr int TOTAL = DO + 8;
};

template <int NOUT>
__global__ void __launch_bounds__(kBwdThreads, 1) k_prop_bwd(BwdArgs a)
{
    using L = BwdSmem<NOUT>;
    extern __shared__ __align__(16) float bs[];
    const int tid = threadIdx.x;
    float *g = bs + L::G;
    float *w2 = bs + L::W2, *w3 = bs + L::W3;
    float *v = bs + L::V, *a1 = bs + L::A1, *a2 = bs + L::A2, *z3 = bs + L::Z3, *z2 = bs + L::Z2, *z1 = bs + L::Z1;
    float *dO = bs + L::DO;
    for (int k = tid; k < L::NW; k += kBwdThreads) g[k] = 0.f;
    for (int k = tid; k < 4608; k += kBwdThreads) w2[k] = __bfloat162float(__float2bfloat16_rn(a.w[kW2 + k]));
    for (int k = tid; k < 9216; k += kBwdThreads) w3[k] = __bfloat162float(__float2bfloat16_rn(a.w[kW3 + k]));
    const float *wh = a.w + kWH;
    float lsum = 0.f;
    __syncthreads();
    for (int b = blockIdx.x; b < a.n; b += gridDim.x) {
        // ---- load this window's activations ----
        for (int k = tid; k < kWin2; k += kBwdThreads) v[k] = a.save_v[(size_t)b * kWin2 + k];
        for (int k = tid; k < 81 * 16; k += kBwdThreads) {
            const int p = k >> 4, c = k & 15;
            a1[c * 81 + p] = __bfloat162float(a.save_a1[(size_t)b * 81 * 16 + k]);
        }
        for (int k = tid; k < 49 * 32; k += kBwdThreads) {
            const int p49 = k >> 5, c = k & 31;
            const int pos = (p49 / 7) * 9 + p49 % 7;
            a2[c * 49 + p49] = __bfloat162float(a.save_a2[((size_t)b * 81 + pos) * 32 + c]);
        }
        for (int k = tid; k < 25 * 32; k += kBwdThreads) {
            const int p = k >> 5, c = k & 31;
            z3[c * 25 + p] = a.save_a3[(size_t)b * 800 + k];
        }
        if (tid < NOUT) {
            const int j = tid;
            const int src = a.index ? a.index[b] : b;
            const float b0 = a.save_stat[(size_t)b * 2], s0 = a.save_stat[(size_t)b * 2 + 1];
            const float t = param_to_target<NOUT>(j, a.labels[(size_t)src * NOUT + j], b0, s0);
            const float d = a.out[(size_t)b * NOUT + j] - t;
            dO[j] = 2.f * a.lam[j] * d * a.inv_batch;
            lsum += a.lam[j] * d * d;
        }
        __syncthreads();
        // ---- head ----
        for (int f = tid; f < 800; f += kBwdThreads) {
            const float act = z3[f];  // [channel][position] flattening, as the head's
            float da = 0.f;
#pragma unroll
            for (int j = 0; j < NOUT; ++j) {
                g[kWH + j * 800 + f] += dO[j] * act;
                da = fmaf(wh[j * 800 + f], dO[j], da);
            }
            z3[f] = act > 0.f ? da : 0.f;
        }
        if (tid < NOUT) g[kWH + NOUT * 800 + tid] += dO[tid];
        __syncthreads();
        // ---- conv3: weight gradients ----
        for (int k = tid; k < 1024; k += kBwdThreads) {
            const int co = k & 31, ci = k >> 5;
            float acc[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) acc[t] = 0.f;
            for (int p = 0; p < 25; ++p) {
                const float d = z3[co * 25 + p];
                const int oy = p / 5, ox = p - oy * 5;
                const float *src = a2 + ci * 49 + oy * 7 + ox;
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[t] = fmaf(d, src[(t / 3) * 7 + t % 3], acc[t]);
            }
#pragma unroll
            for (int t = 0; t < 9; ++t) g[kW3 + (co * 32 + ci) * 9 + t] += acc[t];
        }
        if (tid < 32) {
            float s = 0.f;
            for (int p = 0; p < 25; ++p) s += z3[tid * 25 + p];
            g[kB3 + tid] += s;
        }
        // ---- conv3: input gradient, ReLU mask -> dz2 ----
        for (int k = tid; k < 32 * 49; k += kBwdThreads) {
            const int ci = k / 49, qp = k - ci * 49, iy = qp / 7, ix = qp - iy * 7;
            float s = 0.f;
            if (a2[ci * 49 + qp] > 0.f) {
                for (int co = 0; co < 32; ++co) {
                    const float *wr = w3 + (co * 32 + ci) * 9;
                    const float *dz = z3 + co * 25;
#pragma unroll
                    for (int t = 0; t < 9; ++t) {
                        const int oy = iy - t / 3, ox = ix - t % 3;
                        if (oy >= 0 && oy < 5 && ox >= 0 && ox < 5) s = fmaf(wr[t], dz[oy * 5 + ox], s);
                    }
                }
            }
            z2[k] = s;
        }
        __syncthreads();
        // ---- conv2: weight gradients ----
        for (int k = tid; k < 512; k += kBwdThreads) {
            const int co = k & 31, ci = k >> 5;
            float acc[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) acc[t] = 0.f;
            for (int p = 0; p < 49; ++p) {
                const float d = z2[co * 49 + p];
                const int oy = p / 7, ox = p - oy * 7;
                const float *src = a1 + ci * 81 + oy * 9 + ox;
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[t] = fmaf(d, src[(t / 3) * 9 + t % 3], acc[t]);
            }
#pragma unroll
            for (int t = 0; t < 9; ++t) g[kW2 + (co * 16 + ci) * 9 + t] += acc[t];
        }
        if (tid < 32) {
            float s = 0.f;
            for (int p = 0; p < 49; ++p) s += z2[tid * 49 + p];
            g[kB2 + tid] += s;
        }
        // ---- conv2: input gradient, ReLU mask -> dz1 ----
        for (int k = tid; k < 16 * 81; k += kBwdThreads) {
            const int ci = k / 81, qp = k - ci * 81, iy = qp / 9, ix = qp - iy * 9;
            float s = 0.f;
            if (a1[ci * 81 + qp] > 0.f) {
                for (int co = 0; co < 32; ++co) {
                    const float *wr = w2 + (co * 16 + ci) * 9;
                    const float *dz = z2 + co * 49;
#pragma unroll
                    for (int t = 0; t < 9; ++t) {
                        const int oy = iy - t / 3, ox = ix - t % 3;
                        if (oy >= 0 && oy < 7 && ox >= 0 && ox < 7) s = fmaf(wr[t], dz[oy * 7 + ox], s);
                    }
                }
            }
            z1[k] = s;
        }
        __syncthreads();
        // ---- conv1: weight gradients ----
        static_assert(kBwdThreads >= 160, "one thread per conv1 weight and bias");
        if (tid < 144) {
            const int co = tid / 9, t = tid - co * 9, dy = t / 3, dx = t % 3;
            float s = 0.f;
            for (int p = 0; p < 81; ++p) s = fmaf(z1[co * 81 + p], v[(p / 9 + dy) * kWin + p % 9 + dx], s);
            g[kW1 + tid] += s;
        } else if (tid < 160) {
            const int co = tid - 144;
            float s = 0.f;
            for (int p = 0; p < 81; ++p) s += z1[co * 81 + p];
            g[kB1 + co] += s;
        }
        __syncthreads();
    }
    for (int k = tid; k < L::NW; k += kBwdThreads)
        if (g[k] != 0.f) atomicAdd(&a.grad[k], g[k]);
    if (tid < NOUT) atomicAdd(a.loss, lsum);
}

__global__ void k_adam(float *w, const float *grad, float *m, float *v2, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v2[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v2[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

__global__ void k_pack(const float *w, __nv_bfloat16 *wp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kW2P) {
        const int e = i & 7, co = (i >> 3) & 31, c = (i >> 8) & 1, t = i >> 9;
        wp[i] = __float2bfloat16_rn(w[kW2 + (co * 16 + c * 8 + e) * 9 + t]);
    } else if (i < kW2P + kW3P) {
        const int k = i - kW2P;
        const int e = k & 7, co = (k >> 3) & 31, c = (k >> 8) & 3, t = k >> 10;
        wp[i] = __float2bfloat16_rn(w[kW3 + (co * 32 + c * 8 + e) * 9 + t]);
    } else if (i < kWP) {
        const int k = i - kW2P - kW3P;
        const int e = k & 7, co = (k >> 3) & 15, t = (k >> 7) * 8 + e;
        wp[i] = __float2bfloat16_rn(t < 9 ? w[kW1 + co * 9 + t] : 0.f);
    }
}

// ---------------------------------------------------------------------------
// Synthetic training windows from the method's forward model: one emitter
// near the centre (offset U[-1, 1] px per axis), width U[1, 2] px per axis
// (equal axes for the symmetric models), amplitude lognormal (median 500,
// log-sd 0.6), background U[50, 200]; Poisson(0.5) further emitters anywhere
// within 3 px of the window; Poisson shot noise plus Gaussian read noise
// (sd 2), rounded and clipped to uint16. One block per window.
// ---------------------------------------------------------------------------
__global__ void k_synth_rois(uint16_t *rois, int n, int elliptic, unsigned long long seed, float *truth)
{
    __shared__ float em[4][5];
    __shared__ float bg;
    __shared__ int ne;
    const int roi = blockIdx.x;
    if (roi >= n) return;
    if (threadIdx.x == 0) {
        curandStatePhilox4_32_10_t st;
        curand_init(seed, (unsigned long long)roi, 0, &st);
        bg = 50.f + 150.f * curand_uniform(&st);
        int extra = (int)curand_poisson(&st, 0.5);
        extra = extra > 3 ? 3 : extra;
        ne = 1 + extra;
        for (int e = 0; e < ne; ++e) {
            float x, y;
            if (e == 0) {
                x = 5.f + (2.f * curand_uniform(&st) - 1.f);
                y = 5.f + (2.f * curand_uniform(&st) - 1.f);
            } else {
                x = -3.f + 16.f * curand_uniform(&st);
                y = -3.f + 16.f * curand_uniform(&st);
            }
            const float amp = 500.f * expf(0.6f * curand_normal(&st));
            const float sx = 1.f + curand_uniform(&st);
            const float sy = elliptic ? 1.f + curand_uniform(&st) : sx;
            em[e][0] = x; em[e][1] = y; em[e][2] = amp; em[e][3] = sx; em[e][4] = sy;
        }
        if (truth) {
            float *t = truth + (size_t)roi * 6;
            t[0] = em[0][0]; t[1] = em[0][1]; t[2] = em[0][2]; t[3] = em[0][3]; t[4] = em[0][4]; t[5] = bg;
        }
    }
    __syncthreads();
    const int px = threadIdx.x;
    if (px >= kWin2) return;
    const float xi = (float)(px % kWin), yj = (float)(px / kWin);
    float lam = bg;
    for (int e = 0; e < ne; ++e) {
        const float dx = xi - em[e][0], dy = yj - em[e][1];
        lam += em[e][2] * __expf(-0.5f * (dx * dx / (em[e][3] * em[e][3]) + dy * dy / (em[e][4] * em[e][4])));
    }
    curandStatePhilox4_32_10_t st;
    curand_init(seed, (unsigned long long)roi, 1 + (unsigned long long)px * 4, &st);
    float val = (float)curand_poisson(&st, (double)lam) + 2.f * curand_normal(&st);
    val = rintf(val);
    val = val < 0.f ? 0.f : (val > 65535.f ? 65535.f : val);
    rois[(size_t)roi * kWin2 + px] = (uint16_t)val;
}

template <int NOUT, int MODE> cudaError_t launch_fwd(const FwdArgs &a, int grid, cudaStream_t stream)
{
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(k_prop_fwd<NOUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFwd);
    });
    if (attr_err != cudaSuccess) return attr_err;
    k_prop_fwd<NOUT, MODE><<<grid, kThreads, kSmemFwd, stream>>>(a);
    return cudaGetLastError();
}

template <int NOUT> cudaError_t launch_bwd(const BwdArgs &a, int grid, cudaStream_t stream)
{
    constexpr int bytes = BwdSmem<NOUT>::TOTAL * 4;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(k_prop_bwd<NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    });
    if (attr_err != cudaSuccess) return attr_err;
    k_prop_bwd<NOUT><<<grid, kBwdThreads, bytes, stream>>>(a);
    return cudaGetLastError();
}

int sm_count(int device)
{
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v > 0 ? v : 148;
}

}  // namespace

int proposal_nout(int method)
{
    return method == 0 ? 5 : method == 1 ? 4 : (method == 5 || method == 7) ? 7 : 0;
}

cudaError_t enqueue_proposal(const ProposalView &net, const uint16_t *frames, long long frame_px, int n_rows,
                             int n_cols, const void *cands, const int *cls, int n, int method, float w0, float *init,
                             unsigned long long *n_warm, int *err, cudaStream_t stream, int *launches)
{
    if (n <= 0) return cudaSuccess;
    const int nout = proposal_nout(method);
    if (nout != net.nout) return cudaErrorInvalidValue;
    FwdArgs a{};
    a.frames = frames;
    a.frame_px = frame_px;
    a.n_rows = n_rows;
    a.n_cols = n_cols;
    a.cands = static_cast<const Cand *>(cands);
    a.cls = cls;
    a.n = n;
    a.w = net.w;
    a.wp = net.wp;
    a.w0 = w0;
    a.init = init;
    a.n_warm = n_warm;
    a.err = err;
    const int groups = (n + kR - 1) / kR;
    const int sms = sm_count(net.device);
    const int grid = groups < kCtasPerSm * sms ? groups : kCtasPerSm * sms;
    if (launches) ++*launches;
    switch (nout) {
    case 5: return launch_fwd<5, 1>(a, grid, stream);
    case 4: return launch_fwd<4, 1>(a, grid, stream);
    default: return launch_fwd<7, 1>(a, grid, stream);
    }
}

}  // namespace locb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct loc_proposal {
    int device = 0;
    int method = 0;
    int nout = 0;
    int nw = 0;
    float *w = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *lam = nullptr, *loss = nullptr;
    __nv_bfloat16 *wp = nullptr;
    int *err = nullptr;
    long long step = 0;
    // saved activations of the last training batch
    int cap = 0;
    float *s_v = nullptr, *s_stat = nullptr, *s_a3 = nullptr, *s_out = nullptr;
    __nv_bfloat16 *s_a1 = nullptr, *s_a2 = nullptr;
};

namespace {

int pfail(int code, const std::string &msg) { return locb::record_error_fixed(code, msg.c_str()); }

int pcuda(cudaError_t e, const char *what)
{
    return pfail(LOC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void free_saved(loc_proposal *p)
{
    cudaFree(p->s_v);
    cudaFree(p->s_stat);
    cudaFree(p->s_a1);
    cudaFree(p->s_a2);
    cudaFree(p->s_a3);
    cudaFree(p->s_out);
    p->s_v = p->s_stat = p->s_a3 = p->s_out = nullptr;
    p->s_a1 = p->s_a2 = nullptr;
    p->cap = 0;
}

cudaError_t ensure_saved(loc_proposal *p, int n)
{
    if (n <= p->cap) return cudaSuccess;
    free_saved(p);
    cudaError_t e;
    if ((e = cudaMalloc(&p->s_v, (size_t)n * 121 * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p->s_stat, (size_t)n * 2 * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p->s_a1, (size_t)n * 81 * 16 * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p->s_a2, (size_t)n * 81 * 32 * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p->s_a3, (size_t)n * 800 * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p->s_out, (size_t)n * 8 * 4)) != cudaSuccess) return e;
    // conv2 rows outside the valid 7 x 7 area are never written: keep them finite
    if ((e = cudaMemset(p->s_a2, 0, (size_t)n * 81 * 32 * 2)) != cudaSuccess) return e;
    p->cap = n;
    return cudaSuccess;
}

// deterministic He-normal initialisation (splitmix64 + Box-Muller)
void init_weights(std::vector<float> &w, int nout, unsigned long long seed)
{
    unsigned long long s = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E5ull;
    auto next = [&]() {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() {
        const double u1 = next(), u2 = next();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    w.assign(locb::weight_count(nout), 0.f);
    auto fill = [&](int off, int cnt, double sd) {
        for (int k = 0; k < cnt; ++k) w[off + k] = (float)(sd * normal());
    };
    fill(locb::kW1, 144, std::sqrt(2.0 / 9.0));
    fill(locb::kW2, 4608, std::sqrt(2.0 / 144.0));
    fill(locb::kW3, 9216, std::sqrt(2.0 / 288.0));
    fill(locb::kWH, nout * 800, 0.1 * std::sqrt(1.0 / 800.0));
}

int forward_stack(loc_proposal *p, const uint16_t *d_rois, const int *d_index, int n, float *d_out, bool save,
                  cudaStream_t st)
{
    locb::FwdArgs a{};
    a.rois = d_rois;
    a.index = d_index;
    a.n = n;
    a.w = p->w;
    a.wp = p->wp;
    a.out = d_out;
    a.err = p->err;
    if (save) {
        a.save_v = p->s_v;
        a.save_stat = p->s_stat;
        a.save_a1 = p->s_a1;
        a.save_a2 = p->s_a2;
        a.save_a3 = p->s_a3;
    }
    const int groups = (n + locb::kR - 1) / locb::kR;
    const int sms = locb::sm_count(p->device);
    const int grid = groups < locb::kCtasPerSm * sms ? groups : locb::kCtasPerSm * sms;
    cudaError_t e;
    switch (p->nout) {
    case 5: e = locb::launch_fwd<5, 0>(a, grid, st); break;
    case 4: e = locb::launch_fwd<4, 0>(a, grid, st); break;
    default: e = locb::launch_fwd<7, 0>(a, grid, st); break;
    }
    return e == cudaSuccess ? LOC_OK : pcuda(e, "proposal forward launch");
}

// Gradient of the mean weighted squared error over a batch (no update).
int gradient(loc_proposal *p, const uint16_t *d_rois, const int *d_index, int n, const float *d_labels,
             const float *lam, cudaStream_t st)
{
    cudaError_t e = ensure_saved(p, n);
    if (e != cudaSuccess) return pcuda(e, "activation buffers");
    if ((e = cudaMemcpyAsync(p->lam, lam, (size_t)p->nout * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return pcuda(e, "loss weights");
    if ((e = cudaMemsetAsync(p->grad, 0, (size_t)p->nw * 4, st)) != cudaSuccess) return pcuda(e, "grad clear");
    if ((e = cudaMemsetAsync(p->loss, 0, 4, st)) != cudaSuccess) return pcuda(e, "loss clear");
    int rc = forward_stack(p, d_rois, d_index, n, p->s_out, true, st);
    if (rc) return rc;
    locb::BwdArgs b{};
    b.n = n;
    b.index = d_index;
    b.labels = d_labels;
    b.lam = p->lam;
    b.w = p->w;
    b.out = p->s_out;
    b.save_v = p->s_v;
    b.save_stat = p->s_stat;
    b.save_a1 = p->s_a1;
    b.save_a2 = p->s_a2;
    b.save_a3 = p->s_a3;
    b.grad = p->grad;
    b.loss = p->loss;
    b.inv_batch = 1.f / (float)n;
    const int sms = locb::sm_count(p->device);
    const int grid = n < sms ? n : sms;
    switch (p->nout) {
    case 5: e = locb::launch_bwd<5>(b, grid, st); break;
    case 4: e = locb::launch_bwd<4>(b, grid, st); break;
    default: e = locb::launch_bwd<7>(b, grid, st); break;
    }
    return e == cudaSuccess ? LOC_OK : pcuda(e, "proposal backward launch");
}

}  // namespace

extern "C" {

LOC_API int loc_proposal_weight_count(int method)
{
    const int nout = locb::proposal_nout(method);
    if (!nout) return pfail(LOC_E_UNSUPPORTED, "no proposal network for this method");
    return locb::weight_count(nout);
}

LOC_API int loc_proposal_create(loc_proposal **out, int device, int method, unsigned long long seed)
{
    if (!out) return pfail(LOC_E_INVALID, "out is NULL");
    *out = nullptr;
    const int nout = locb::proposal_nout(method);
    if (!nout) return pfail(LOC_E_UNSUPPORTED, "no proposal network for this method");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return pcuda(e, "cudaSetDevice");
    loc_proposal *p = new (std::nothrow) loc_proposal();
    if (!p) return pfail(LOC_E_NOMEM, "allocation failed");
    p->device = device;
    p->method = method;
    p->nout = nout;
    p->nw = locb::weight_count(nout);
    const size_t wb = (size_t)p->nw * 4;
    if ((e = cudaMalloc(&p->w, wb)) != cudaSuccess || (e = cudaMalloc(&p->grad, wb)) != cudaSuccess ||
        (e = cudaMalloc(&p->m, wb)) != cudaSuccess || (e = cudaMalloc(&p->v, wb)) != cudaSuccess ||
        (e = cudaMalloc(&p->lam, 8 * 4)) != cudaSuccess || (e = cudaMalloc(&p->loss, 4)) != cudaSuccess ||
        (e = cudaMalloc(&p->wp, (size_t)locb::kWP * 2)) != cudaSuccess || (e = cudaMalloc(&p->err, 4)) != cudaSuccess) {
        loc_proposal_destroy(p);
        return pcuda(e, "proposal allocation");
    }
    std::vector<float> w;
    init_weights(w, nout, seed);
    cudaMemset(p->m, 0, wb);
    cudaMemset(p->v, 0, wb);
    cudaMemset(p->err, 0, 4);
    if ((e = cudaMemcpy(p->w, w.data(), wb, cudaMemcpyHostToDevice)) != cudaSuccess) {
        loc_proposal_destroy(p);
        return pcuda(e, "weight upload");
    }
    locb::k_pack<<<(locb::kWP + 255) / 256, 256>>>(p->w, p->wp);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
        loc_proposal_destroy(p);
        return pcuda(e, "weight packing");
    }
    *out = p;
    return LOC_OK;
}

LOC_API int loc_proposal_destroy(loc_proposal *p)
{
    if (!p) return LOC_OK;
    cudaSetDevice(p->device);
    free_saved(p);
    cudaFree(p->w);
    cudaFree(p->grad);
    cudaFree(p->m);
    cudaFree(p->v);
    cudaFree(p->lam);
    cudaFree(p->loss);
    cudaFree(p->wp);
    cudaFree(p->err);
    delete p;
    return LOC_OK;
}

LOC_API int loc_proposal_get_weights(loc_proposal *p, float *host, int n)
{
    if (!p || !host) return pfail(LOC_E_INVALID, "NULL argument");
    if (n != p->nw) return pfail(LOC_E_INVALID, "weight count mismatch");
    cudaSetDevice(p->device);
    cudaError_t e = cudaMemcpy(host, p->w, (size_t)n * 4, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LOC_OK : pcuda(e, "weight download");
}

LOC_API int loc_proposal_set_weights(loc_proposal *p, const float *host, int n)
{
    if (!p || !host) return pfail(LOC_E_INVALID, "NULL argument");
    if (n != p->nw) return pfail(LOC_E_INVALID, "weight count mismatch");
    cudaSetDevice(p->device);
    cudaError_t e = cudaMemcpy(p->w, host, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return pcuda(e, "weight upload");
    cudaMemset(p->m, 0, (size_t)n * 4);
    cudaMemset(p->v, 0, (size_t)n * 4);
    p->step = 0;
    locb::k_pack<<<(locb::kWP + 255) / 256, 256>>>(p->w, p->wp);
    e = cudaDeviceSynchronize();
    return e == cudaSuccess ? LOC_OK : pcuda(e, "weight packing");
}

LOC_API int loc_proposal_forward(loc_proposal *p, const uint16_t *d_rois, const int *d_index, int n, float *d_out,
                                 float *d_stat, void *stream)
{
    if (!p || !d_rois || !d_out || n < 0) return pfail(LOC_E_INVALID, "bad argument");
    if (n == 0) return LOC_OK;
    cudaSetDevice(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (d_stat) {
        cudaError_t e = ensure_saved(p, n);
        if (e != cudaSuccess) return pcuda(e, "activation buffers");
    }
    int rc = forward_stack(p, d_rois, d_index, n, d_out, d_stat != nullptr, st);
    if (rc) return rc;
    if (d_stat) {
        cudaError_t e = cudaMemcpyAsync(d_stat, p->s_stat, (size_t)n * 2 * 4, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return pcuda(e, "stat copy");
    }
    return LOC_OK;
}

LOC_API int loc_proposal_gradient(loc_proposal *p, const uint16_t *d_rois, const int *d_index, int n,
                                  const float *d_labels, const float *lam, float *d_grad, float *loss_out,
                                  void *stream)
{
    if (!p || !d_rois || !d_labels || !lam || n <= 0) return pfail(LOC_E_INVALID, "bad argument");
    cudaSetDevice(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    int rc = gradient(p, d_rois, d_index, n, d_labels, lam, st);
    if (rc) return rc;
    cudaError_t e;
    if (d_grad &&
        (e = cudaMemcpyAsync(d_grad, p->grad, (size_t)p->nw * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return pcuda(e, "grad copy");
    if (loss_out) {
        float l = 0.f;
        if ((e = cudaMemcpyAsync(&l, p->loss, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return pcuda(e, "loss");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return pcuda(e, "gradient");
        *loss_out = l / (float)n;
    }
    return LOC_OK;
}

LOC_API int loc_proposal_train_step(loc_proposal *p, const uint16_t *d_rois, const int *d_index, int n,
                                    const float *d_labels, const float *lam, float lr, float *loss_out, void *stream)
{
    if (!p || !d_rois || !d_labels || !lam || n <= 0 || !(lr > 0)) return pfail(LOC_E_INVALID, "bad argument");
    cudaSetDevice(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    int rc = gradient(p, d_rois, d_index, n, d_labels, lam, st);
    if (rc) return rc;
    p->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)p->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)p->step)));
    locb::k_adam<<<(p->nw + 255) / 256, 256, 0, st>>>(p->w, p->grad, p->m, p->v, p->nw, lr, b1, b2, 1e-8f, c1, c2);
    locb::k_pack<<<(locb::kWP + 255) / 256, 256, 0, st>>>(p->w, p->wp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return pcuda(e, "optimizer launch");
    if (loss_out) {
        float l = 0.f;
        if ((e = cudaMemcpyAsync(&l, p->loss, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return pcuda(e, "loss");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return pcuda(e, "train step");
        *loss_out = l / (float)n;
    }
    return LOC_OK;
}

LOC_API int loc_proposal_status(loc_proposal *p)
{
    if (!p) return pfail(LOC_E_INVALID, "NULL argument");
    cudaSetDevice(p->device);
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, p->err, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return pcuda(e, "status");
    return v ? pfail(LOC_E_CUDA, "tensor-core wait timed out in the proposal kernel") : LOC_OK;
}

LOC_API int loc_synth_rois(uint16_t *d_rois, int n, int elliptic, unsigned long long seed, float *d_truth,
                           void *stream)
{
    if (!d_rois || n < 0) return pfail(LOC_E_INVALID, "bad argument");
    if (n == 0) return LOC_OK;
    locb::k_synth_rois<<<n, 128, 0, (cudaStream_t)stream>>>(d_rois, n, elliptic, seed, d_truth);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LOC_OK : pcuda(e, "synth launch");
}

}  // extern "C"

// accessor for the fit pipeline
namespace locb {
bool proposal_view(const loc_proposal *p, ProposalView *v)
{
    if (!p) return false;
    v->nout = p->nout;
    v->device = p->device;
    v->w = p->w;
    v->wp = p->wp;
    v->err = p->err;
    return true;
}
}  // namespace locb
