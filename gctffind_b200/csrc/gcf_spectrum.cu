// gcf_spectrum.cu -- tile-spectrum stage (CGenAvgSpectrum / GCalcSpectrum)
// and the Fourier-crop rescale (CRescaleImage / GFtResize2D).
//
// Two implementations of the averaged amplitude spectrum:
//   * the batched-cuFFT variant here: one pass extracts every tile with its
//     mean removed and the GRoundEdge taper applied, one cuFFT R2C batch,
//     one pass accumulates |F| with the DC moved to (0, tile/2);
//   * the fused hand-written tile-FFT kernel in gcf_fused.cu.
#include <cuda_runtime.h>

#include "gcf_internal.h"

namespace gcf {

namespace {

__device__ __forceinline__ double block_sum_double(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    int nw = blockDim.x >> 5;
    if (threadIdx.x < 32) {
        t = threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sh[0] = t;
    }
    __syncthreads();
    t = sh[0];
    __syncthreads();
    return t;
}

// mExtractPadTile + GCalcMoment2D + GNormalize2D + GRoundEdge
// (FindCTF/CGenAvgSpectrum.cpp:105-139): tile with its mean removed and
// the taper applied, dense tile x tile.
__global__ void k_extract_tiles(const float* __restrict__ img, int pitch, int tile, int ntx,
                                int offx, int offy, int stride, int first_tile,
                                const float* __restrict__ taper, float* __restrict__ out)
{
    __shared__ double sh[32];
    int t = first_tile + blockIdx.x;
    int tx = t % ntx, ty = t / ntx;
    const float* src = img + (size_t)(offy + ty * stride) * pitch + offx + tx * stride;
    int n = tile * tile;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int y = i / tile, x = i - y * tile;
        s += (double)src[(size_t)y * pitch + x];
    }
    double mean = block_sum_double(s, sh) / (double)n;
    float m = (float)mean;
    float* dst = out + (size_t)blockIdx.x * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int y = i / tile, x = i - y * tile;
        dst[i] = (src[(size_t)y * pitch + x] - m) * taper[i];
    }
}

// GCalcSpectrum::mGCalculate + GAddImages (FindCTF/GCalcSpectrum.cu:15-31,
// Util/GAddImages.cu:10-23): accumulate |F| of `ntiles` R2C outputs into a
// double buffer with the DC moved to row tile/2.
__global__ void k_amp_accumulate(const float2* __restrict__ cmp, int tile, int ntiles,
                                 double* __restrict__ acc)
{
    int cx = tile / 2 + 1;
    int n = cx * tile;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int yd = i / cx, kx = i - yd * cx;
    int ky = yd + tile / 2;
    if (ky >= tile) ky -= tile;
    const float2* p = cmp + (size_t)ky * cx + kx;
    double s = 0.0;
    for (int b = 0; b < ntiles; ++b) {
        float2 v = p[(size_t)b * n];
        s += (double)sqrtf(v.x * v.x + v.y * v.y);
    }
    acc[i] += s;
}

__global__ void k_finalize_raw(const double* __restrict__ acc, int n, double inv, float* raw)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) raw[i] = (float)(acc[i] * inv);
}

// GFtResize2D::mGTruncate without summation (Util/GFtResize2D.cu:7-32).
// One output row per blockIdx.y (its source row computed once), columns
// over the threads of blockIdx.x.
__global__ void k_fourier_crop(const float2* __restrict__ in, int cx_in, int cy_in,
                               float2* __restrict__ out, int cx_out, int cy_out)
{
    const int y = blockIdx.y, x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= cx_out) return;
    const int ys = (y > cy_out / 2) ? y - cy_out + cy_in : y;
    out[(size_t)y * cx_out + x] = __ldg(in + (size_t)ys * cx_in + x);
}

}  // namespace

void launch_extract_tiles(const float* img, int w, int h, int pitch, int tile, int ntx,
                          int offx, int offy, int stride, int first_tile, int ntiles,
                          const float* taper, float* out, cudaStream_t st)
{
    (void)w;
    (void)h;
    if (ntiles <= 0) return;
    k_extract_tiles<<<ntiles, 256, 0, st>>>(img, pitch, tile, ntx, offx, offy, stride,
                                            first_tile, taper, out);
}

void launch_amp_accumulate(const float2* cmp, int tile, int ntiles, double* acc, cudaStream_t st)
{
    int n = (tile / 2 + 1) * tile;
    k_amp_accumulate<<<(n + 255) / 256, 256, 0, st>>>(cmp, tile, ntiles, acc);
}

void launch_finalize_raw(const double* acc, int n, double inv, float* raw, cudaStream_t st)
{
    k_finalize_raw<<<(n + 255) / 256, 256, 0, st>>>(acc, n, inv, raw);
}

void launch_fourier_crop(const float2* in, int cx_in, int cy_in, float2* out, int cx_out,
                         int cy_out, cudaStream_t st)
{
    const dim3 grid((cx_out + 255) / 256, cy_out);
    k_fourier_crop<<<grid, 256, 0, st>>>(in, cx_in, cy_in, out, cx_out, cy_out);
}

}  // namespace gcf
