// Frame ingest: camera buffers of any of the reference's storage types
// (LocalizerStorageType, reference source/Defines.h:82-95) in row- or
// column-major order (BufferWithFormatToImage / CopyBufferToImage,
// source/FileIO.cpp:195-234, FileIO.h:96-116) into the fit path's uint16
// frame stack (x fastest). The reference widens every pixel to double; the
// fit path works on uint16, which holds every value of 8- and 16-bit unsigned
// cameras exactly. Other values are rounded to the nearest integer and
// clamped to [0, 65535]; the call returns how many pixels that changed, so a
// caller can tell a lossless ingest (0) from a lossy one.
//
// Column-major input is a streaming conversion; row-major input is
// transposed through 64 x 64 shared-memory tiles so that both the reads and
// the writes are coalesced. HBM-bound: element size + 2 bytes per pixel.
#include "../../include/localizer_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>

namespace locb {
int record_error_fixed(int code, const char *msg);
}

namespace {

constexpr int kTile = 64;     // row-major transpose tile (64 x 64 pixels, 256 threads)

template <typename S> __device__ __forceinline__ uint16_t to_u16(S v, unsigned &lossy)
{
    if constexpr (sizeof(S) <= 2 && !std::is_signed<S>::value) {
        return (uint16_t)v;
    } else if constexpr (std::is_same<S, float>::value) {
        float r = rintf(v);
        r = r < 0.0f ? 0.0f : (r > 65535.0f ? 65535.0f : r);
        if (!(r == v)) ++lossy;   // rounded, clamped, or NaN (-> 0)
        return (uint16_t)(r == r ? r : 0.0f);
    } else {
        const double d = (double)v;
        double r = rint(d);
        r = r < 0.0 ? 0.0 : (r > 65535.0 ? 65535.0 : r);
        if (!(r == d)) ++lossy;
        return (uint16_t)(r == r ? r : 0.0);
    }
}

// V consecutive elements moved by one load or store (the host checks the
// alignment and the sizes before it picks V > 1)
template <typename T, int V> struct alignas(V * sizeof(T)) Vec {
    T v[V];
};

__device__ __forceinline__ void count_lossy(unsigned lossy, unsigned long long *counter)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lossy += __shfl_xor_sync(0xffffffffu, lossy, o);
    if ((threadIdx.x & 31) == 0 && lossy) atomicAdd(counter, (unsigned long long)lossy);
}

// column-major: the same pixel order on both sides, V pixels per thread and trip
template <typename S, int V>
__global__ void k_ingest_cm(const S *src, uint16_t *dst, long long n, unsigned long long *lossy_count)
{
    unsigned lossy = 0;
    const long long nv = n / V;
    const Vec<S, V> *sv = reinterpret_cast<const Vec<S, V> *>(src);
    Vec<uint16_t, V> *dv = reinterpret_cast<Vec<uint16_t, V> *>(dst);
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nv; p += (long long)gridDim.x * blockDim.x) {
        const Vec<S, V> x = sv[p];
        Vec<uint16_t, V> y;
#pragma unroll
        for (int k = 0; k < V; ++k) y.v[k] = to_u16<S>(x.v[k], lossy);
        dv[p] = y;
    }
    count_lossy(lossy, lossy_count);
}

// row-major: frame buffer element (i, j) at i * n_cols + j -> pixel i + j * n_rows,
// through a 64 x 64 shared-memory tile so that reads (along j) and writes
// (along i) are both coalesced. V = 2: each thread reads a pair along j and
// writes a pair along i (a warp moves a 64-pixel segment per access; needs
// even n_rows and n_cols and aligned buffers); V = 1: single pixels.
template <typename S, int V>
__global__ void __launch_bounds__(256) k_ingest_rm(const S *src, uint16_t *dst, int n_rows, int n_cols,
                                                   unsigned long long *lossy_count)
{
    __shared__ uint16_t t[kTile][kTile + 1];
    const size_t fpx = (size_t)n_rows * n_cols;
    const S *fs = src + (size_t)blockIdx.z * fpx;
    uint16_t *fd = dst + (size_t)blockIdx.z * fpx;
    const int j0 = blockIdx.x * kTile, i0 = blockIdx.y * kTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned lossy = 0;
    if constexpr (V == 2) {
        for (int di = warp; di < kTile; di += 8) {
            const int i = i0 + di, j = j0 + 2 * lane;
            if (i < n_rows && j < n_cols) {   // j even, n_cols even: j + 1 < n_cols
                const Vec<S, 2> x = *reinterpret_cast<const Vec<S, 2> *>(fs + (size_t)i * n_cols + j);
                t[di][2 * lane] = to_u16<S>(x.v[0], lossy);
                t[di][2 * lane + 1] = to_u16<S>(x.v[1], lossy);
            }
        }
        __syncthreads();
        for (int dj = warp; dj < kTile; dj += 8) {
            const int j = j0 + dj, i = i0 + 2 * lane;
            if (j < n_cols && i < n_rows) {   // i even, n_rows even: i + 1 < n_rows
                Vec<uint16_t, 2> y;
                y.v[0] = t[2 * lane][dj];
                y.v[1] = t[2 * lane + 1][dj];
                *reinterpret_cast<Vec<uint16_t, 2> *>(fd + i + (size_t)j * n_rows) = y;
            }
        }
    } else {
        for (int di = warp; di < kTile; di += 8)
            for (int dj = lane; dj < kTile; dj += 32) {
                const int i = i0 + di, j = j0 + dj;
                if (i < n_rows && j < n_cols) t[di][dj] = to_u16<S>(fs[(size_t)i * n_cols + j], lossy);
            }
        __syncthreads();
        for (int dj = warp; dj < kTile; dj += 8)
            for (int di = lane; di < kTile; di += 32) {
                const int i = i0 + di, j = j0 + dj;
                if (i < n_rows && j < n_cols) fd[i + (size_t)j * n_rows] = t[di][dj];
            }
    }
    count_lossy(lossy, lossy_count);
}

template <typename S>
cudaError_t launch(const void *src, uint16_t *dst, int n_frames, int n_rows, int n_cols, int row_major,
                   unsigned long long *cnt, cudaStream_t st)
{
    const S *s = static_cast<const S *>(src);
    const uintptr_t sa = reinterpret_cast<uintptr_t>(src), da = reinterpret_cast<uintptr_t>(dst);
    if (!row_major) {
        const long long n = (long long)n_frames * n_rows * n_cols;
        const bool v4 = n % 4 == 0 && sa % (4 * sizeof(S)) == 0 && da % 8 == 0;
        const long long units = v4 ? n / 4 : n;
        const int blocks = (int)((units + 255) / 256 < 148 * 16 ? (units + 255) / 256 : 148 * 16);
        if (v4) k_ingest_cm<S, 4><<<blocks, 256, 0, st>>>(s, dst, n, cnt);
        else k_ingest_cm<S, 1><<<blocks, 256, 0, st>>>(s, dst, n, cnt);
    } else {
        const bool v2 = n_rows % 2 == 0 && n_cols % 2 == 0 && sa % (2 * sizeof(S)) == 0 && da % 4 == 0;
        dim3 grid((n_cols + kTile - 1) / kTile, (n_rows + kTile - 1) / kTile, n_frames);
        if (v2) k_ingest_rm<S, 2><<<grid, 256, 0, st>>>(s, dst, n_rows, n_cols, cnt);
        else k_ingest_rm<S, 1><<<grid, 256, 0, st>>>(s, dst, n_rows, n_cols, cnt);
    }
    return cudaGetLastError();
}

}  // namespace

extern "C" LOC_API long long loc_ingest_frames(const void *d_src, int format, int n_frames, int n_rows, int n_cols,
                                               int row_major, uint16_t *d_dst, void *stream)
{
    if (!d_src || !d_dst || n_frames < 0 || n_rows <= 0 || n_cols <= 0)
        return locb::record_error_fixed(LOC_E_INVALID, "bad argument");
    if (n_frames > 65535 && row_major) return locb::record_error_fixed(LOC_E_UNSUPPORTED, "too many frames in one call");
    if (n_frames == 0) return 0;
    const cudaStream_t st = (cudaStream_t)stream;
    // one lossy counter per host thread and device, kept across calls (a
    // stream-ordered allocation per call would go back to the driver at every
    // synchronisation)
    struct Counter {
        unsigned long long *p = nullptr;
        int dev = -1;
        ~Counter()
        {
            if (p) cudaFree(p);
        }
    };
    static thread_local Counter counter;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && counter.dev != dev) {
        if (counter.p) cudaFree(counter.p);
        counter.p = nullptr;
        counter.dev = -1;
        e = cudaMalloc((void **)&counter.p, sizeof(unsigned long long));
        if (e == cudaSuccess) counter.dev = dev;
    }
    if (e != cudaSuccess) return locb::record_error_fixed(LOC_E_NOMEM, "ingest counter");
    unsigned long long *cnt = counter.p;
    cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st);
    switch (format) {
    case 2: e = launch<int8_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 3: e = launch<uint8_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 4: e = launch<int16_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 5: e = launch<uint16_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 6: e = launch<int32_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 7: e = launch<uint32_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 8: e = launch<int64_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 9: e = launch<uint64_t>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 10: e = launch<float>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    case 11: e = launch<double>(d_src, d_dst, n_frames, n_rows, n_cols, row_major, cnt, st); break;
    default:
        return locb::record_error_fixed(LOC_E_UNSUPPORTED, "unsupported storage format (4-bit types are not)");
    }
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, cnt, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return locb::record_error_fixed(LOC_E_CUDA, (std::string("ingest: ") + cudaGetErrorString(e)).c_str());
    return (long long)h;
}
