// Synthetic single-molecule frames on the GPU (workload generation, not part
// of the fit path). Expected photons = per-frame background + sum of
// point-sampled 2D Gaussians A exp(-(dx^2/2sx^2 + dy^2/2sy^2)); counts are
// Poisson draws plus Gaussian read noise, rounded and clipped to uint16
// (gain 1). Layout as the fit path expects: frame f, pixel (x, y) at
// f*n_rows*n_cols + x + y*n_rows.
//
// One block renders a 16 x 16 tile of one frame; the frame's emitters whose
// 5-sigma box touches the tile are filtered into shared memory first, in
// emitter order (at most 1024 per tile), so a seed gives the same frames on
// every run.
#include "../../include/localizer_b200.h"

#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstdint>

namespace {

constexpr int kTile = 16;
constexpr int kMaxLocal = 1024;

__global__ void k5_render(uint16_t *frames, int n_rows, int n_cols, const float *em, const int *frame_start,
                          const float *background, float read_noise, unsigned long long seed)
{
    __shared__ float sem_raw[kMaxLocal * 5];
    __shared__ float sem[kMaxLocal * 5];
    __shared__ int sidx[kMaxLocal];
    __shared__ int scount;
    const int f = blockIdx.z;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
    if (threadIdx.x == 0 && threadIdx.y == 0) scount = 0;
    __syncthreads();
    const int e0 = frame_start[f], e1 = frame_start[f + 1];
    const int tid = threadIdx.y * kTile + threadIdx.x;
    for (int k = e0 + tid; k < e1; k += kTile * kTile) {
        const float x = em[5 * k + 0], y = em[5 * k + 1], sx = em[5 * k + 3], sy = em[5 * k + 4];
        const float rx = 5.0f * sx + 1.0f, ry = 5.0f * sy + 1.0f;
        if (x + rx < tx0 || x - rx > tx0 + kTile - 1 || y + ry < ty0 || y - ry > ty0 + kTile - 1) continue;
        const int slot = atomicAdd(&scount, 1);
        if (slot < kMaxLocal) {
            sidx[slot] = k;
            for (int q = 0; q < 5; ++q) sem_raw[5 * slot + q] = em[5 * k + q];
        }
    }
    __syncthreads();
    const int n = scount < kMaxLocal ? scount : kMaxLocal;
    // emitters back into index order (each goes to the count of smaller
    // indices), so that the expected counts are summed in the same order on
    // every run and the frames are reproducible bit for bit
    for (int t = tid; t < n; t += kTile * kTile) {
        const int kk = sidx[t];
        int rank = 0;
        for (int j = 0; j < n; ++j) rank += sidx[j] < kk ? 1 : 0;
        for (int q = 0; q < 5; ++q) sem[5 * rank + q] = sem_raw[5 * t + q];
    }
    __syncthreads();
    const int px = tx0 + threadIdx.x, py = ty0 + threadIdx.y;
    if (px >= n_rows || py >= n_cols) return;
    float lam = background[f];
    for (int k = 0; k < n; ++k) {
        const float dx = (float)px - sem[5 * k + 0], dy = (float)py - sem[5 * k + 1];
        const float sx = sem[5 * k + 3], sy = sem[5 * k + 4];
        lam += sem[5 * k + 2] * __expf(-0.5f * (dx * dx / (sx * sx) + dy * dy / (sy * sy)));
    }
    const size_t at = (size_t)f * n_rows * n_cols + px + (size_t)py * n_rows;
    curandStatePhilox4_32_10_t st;
    curand_init(seed, at, 0, &st);
    float v = (float)curand_poisson(&st, (double)lam) + read_noise * curand_normal(&st);
    v = rintf(v);
    v = v < 0.f ? 0.f : (v > 65535.f ? 65535.f : v);
    frames[at] = (uint16_t)v;
}

}  // namespace

extern "C" LOC_API int loc_synth_frames(uint16_t *d_frames, int n_frames, int n_rows, int n_cols,
                                        const float *d_emitters, const int *d_frame_start,
                                        const float *d_background, float read_noise, unsigned long long seed,
                                        void *stream)
{
    if (!d_frames || n_frames <= 0 || n_rows <= 0 || n_cols <= 0 || !d_emitters || !d_frame_start || !d_background)
        return LOC_E_INVALID;
    dim3 grid((n_rows + kTile - 1) / kTile, (n_cols + kTile - 1) / kTile, n_frames);
    dim3 block(kTile, kTile);
    k5_render<<<grid, block, 0, (cudaStream_t)stream>>>(d_frames, n_rows, n_cols, d_emitters, d_frame_start,
                                                        d_background, read_noise, seed);
    return cudaGetLastError() == cudaSuccess ? LOC_OK : LOC_E_CUDA;
}
