// gcf_background.cu -- the 1D background of GBackground1D
// (FindCTF/GBackground1D.cu:13-169): a linear fit over the middle three
// fifths of a 1D spectrum finds the first bin where the spectrum drops to
// the line (the start), then a moving average of width start/2*2-1
// (mirrored at the far end) is the background from the start on.
// Remove1D / Remove2D subtract it from a 1D spectrum or, by radius with
// linear interpolation, from a half spectrum, zeroing inside the start.
//
// The reference fits on the host in double; here one lane of one block
// sums in the same order with round-to-nearest intrinsics, so no FMA
// contraction changes the line, and every background bin is its own float
// sum in the reference's order: start and background are bit-identical.
// Remove2D keeps the reference's expression and default contraction.
#include <cuda_runtime.h>

#include "gcf_internal.h"

namespace gcf {
namespace {

constexpr int kBgThreads = 256;

__global__ void k_background1d(const float* __restrict__ spec, int n, float* __restrict__ bg,
                               int* __restrict__ start_out)
{
    extern __shared__ float s_spec[];
    __shared__ int s_start;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_spec[i] = spec[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        // GBackground1D::mFindStart (FindCTF/GBackground1D.cu:140-169)
        int i0 = n / 5, i1 = n - i0;
        double dx = 0.0, dy = 0.0, dx2 = 0.0, dxy = 0.0;
        for (int i = i0; i < i1; ++i) {
            dx = __dadd_rn(dx, (double)i);
            dx2 = __dadd_rn(dx2, (double)(i * i));
            dy = __dadd_rn(dy, (double)s_spec[i]);
            dxy = __dadd_rn(dxy, (double)__fmul_rn((float)i, s_spec[i]));
        }
        int cnt = i1 - i0;
        dx = __ddiv_rn(dx, (double)cnt);
        dy = __ddiv_rn(dy, (double)cnt);
        dx2 = __ddiv_rn(dx2, (double)cnt);
        dxy = __ddiv_rn(dxy, (double)cnt);
        double a = __ddiv_rn(__dsub_rn(__dmul_rn(dx, dy), dxy), __dsub_rn(__dmul_rn(dx, dx), dx2));
        double b = __dsub_rn(dy, __dmul_rn(a, dx));
        int start = i0;
        for (int i = 2; i < n; ++i) {
            double y = __dadd_rn(__dmul_rn(a, (double)i), b);
            if (y < (double)s_spec[i]) continue;
            start = i;
            break;
        }
        s_start = start;
        *start_out = start;
    }
    __syncthreads();
    const int start = s_start;
    const int win = start / 2 * 2 - 1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (i < start) {
            bg[i] = 0.0f;
            continue;
        }
        float sum = 0.0f;
        for (int j = 0; j < win; ++j) {
            int k = i + j - win / 2;
            if (k >= n) k = 2 * n - 1 - k;
            sum = __fadd_rn(sum, s_spec[k]);
        }
        bg[i] = __fdiv_rn(sum, (float)win);
    }
}

// GBackground1D::Remove1D (FindCTF/GBackground1D.cu:13-30,61-72).  Bins at
// or past bg_n are left alone: the reference sends all of them to bin
// bg_n - 1 at once (a write race), which is not reproduced.
__global__ void k_remove_bg1d(float* __restrict__ spec, int n, const float* __restrict__ bg, int bg_n,
                              int start)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i < start) {
        spec[i] = 0.0f;
        return;
    }
    if (i >= bg_n) return;
    spec[i] -= bg[i];
}

// GBackground1D::Remove2D (FindCTF/GBackground1D.cu:32-59,74-93) on a
// tile x (tile/2 + 1) half spectrum with the DC at (0, tile/2).
__global__ void k_remove_bg2d(float* __restrict__ spec, int cx, int cy, const float* __restrict__ bg,
                              int bg_n, int start)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= cx) return;
    int i = y * cx + x;
    int yc = y - cy / 2;
    float r = sqrtf((float)(x * x + yc * yc));
    if (r < start) {
        spec[i] = 0.0f;
        return;
    }
    if (r >= (bg_n - 1)) {
        spec[i] -= bg[bg_n - 1];
        return;
    }
    int ir = (int)r;
    float v = bg[ir] * (ir + 1 - r) + bg[ir + 1] * (r - ir);
    spec[i] -= v;
}

}  // namespace

cudaError_t launch_background1d(const float* spec, int n, float* bg, int* start, cudaStream_t st)
{
    if (n <= 0 || n > kMaxBackgroundBins) return cudaErrorInvalidValue;
    k_background1d<<<1, kBgThreads, n * sizeof(float), st>>>(spec, n, bg, start);
    return cudaGetLastError();
}

cudaError_t launch_remove_background1d(float* spec, int n, const float* bg, int bg_n, int start,
                                       cudaStream_t st)
{
    if (n <= 0 || bg_n <= 0) return cudaErrorInvalidValue;
    k_remove_bg1d<<<(n + 255) / 256, 256, 0, st>>>(spec, n, bg, bg_n, start);
    return cudaGetLastError();
}

cudaError_t launch_remove_background2d(float* spec, int tile, const float* bg, int bg_n, int start,
                                       cudaStream_t st)
{
    if (tile <= 0 || bg_n <= 0) return cudaErrorInvalidValue;
    int cx = tile / 2 + 1;
    dim3 grid((cx + 127) / 128, tile);
    k_remove_bg2d<<<grid, 128, 0, st>>>(spec, cx, tile, bg, bg_n, start);
    return cudaGetLastError();
}

}  // namespace gcf
