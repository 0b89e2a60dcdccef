// gcf_post.cu -- spectrum post-processing on the averaged half spectrum:
// background removal (GRmBackground2D), moments and B-factor lowpass
// (CFindCtfBase::mRemoveBackground/mLowpass), radial average (GRadialAvg),
// gathering of the in-band pixels for the candidate kernels, the diagnostic
// full spectrum (CSpectrumImage, GCalcCTF2D::EmbedCtf) and the spectral-CC
// resolution (GSpectralCC2D).
//
// Compiled with -fmad=false: the float expressions that decide masks and
// bands are rounded operation by operation, like the oracle.
#include <cuda_runtime.h>
#include <math.h>

#include "gcf_internal.h"

namespace gcf {

namespace {

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh /* 32*NV */)
{
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        v[k] = warp_sum(v[k]);
        if (lane == 0) sh[k * 32 + warp] = v[k];
    }
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < nw ? sh[k * 32 + lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) sh[k * 32] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = sh[k * 32];
    __syncthreads();
}

// Value of the background plane at relative position (u, R): the Hermitian
// fold of GRmBackground2D::mGRemove (FindCTF/GRmBackground2D.cu:42-64).
__device__ __forceinline__ float bg_val(const float* row, const float* mrow, int u, int half_x,
                                        int tile)
{
    if (u >= half_x) u -= 2 * half_x;
    (void)tile;
    return (u >= 0) ? row[u] : mrow[-u];
}

// Rows per block of the horizontal box sums (powers of two, so that the
// 256 threads split evenly over the rows).
__host__ __device__ constexpr int bg_rows_per_block(int tile)
{
    return tile <= 512 ? 8 : tile <= 1024 ? 4 : tile <= 2048 ? 2 : 1;
}

// Horizontal box sums of sqrt(raw) (or raw if log_spect) for every row and
// every output column x in [0, cx).  A block holds bg_rows_per_block rows
// and their mirror rows; each thread sums the box at the first column of
// its run of consecutive columns and slides it over the rest (add the
// entering, subtract the leaving value), in FP64.
__global__ void __launch_bounds__(256) k_bg_horizontal(const float* __restrict__ raw, int tile, int log_spect,
                                                       int box, double* __restrict__ hsum)
{
    extern __shared__ float sh[];
    const int cx = tile / 2 + 1, half_x = cx - 1;
    const int RB = bg_rows_per_block(tile), tpr = blockDim.x / RB;
    const int r0 = blockIdx.x * RB, m = blockIdx.y;
    const float* src = raw + (size_t)m * cx * tile;
    for (int i = threadIdx.x; i < RB * cx; i += blockDim.x) {
        const int rr = i / cx, x = i - rr * cx, R = r0 + rr;
        if (R >= tile) continue;
        const int mr = (tile - R) % tile;   // half_y - (R - half_y) modulo tile
        float a = src[(size_t)R * cx + x], b = src[(size_t)mr * cx + x];
        sh[rr * 2 * cx + x] = log_spect ? a : sqrtf(a);
        sh[rr * 2 * cx + cx + x] = log_spect ? b : sqrtf(b);
    }
    __syncthreads();
    const int rr = threadIdx.x / tpr, t = threadIdx.x - rr * tpr, R = r0 + rr;
    if (rr >= RB || R >= tile) return;
    const float* row = sh + rr * 2 * cx;
    const float* mrow = row + cx;
    const int seg = (cx + tpr - 1) / tpr;
    const int x0 = t * seg, x1 = min(cx, x0 + seg);
    if (x0 >= x1) return;
    const int hb = box / 2;
    double* out = hsum + ((size_t)m * tile + R) * cx;
    double sum = 0.0;
    for (int j = -hb; j <= hb; ++j) sum += (double)bg_val(row, mrow, x0 + j, half_x, tile);
    out[x0] = sum;
    for (int x = x0 + 1; x < x1; ++x) {
        sum += (double)bg_val(row, mrow, x + hb, half_x, tile) - (double)bg_val(row, mrow, x - 1 - hb, half_x, tile);
        out[x] = sum;
    }
}

// Vertical box sums, DC mask (fR < 0.04) and subtraction
// (FindCTF/GRmBackground2D.cu:18-31, :67-69).  A block covers kBgSegY rows
// of every column; each thread slides the vertical box down its column (one
// column per thread up to tile 1024: the block has cx threads rounded up to
// whole warps, at most kBgVertThreads).
constexpr int kBgSegY = 16;
constexpr int kBgVertThreads = 544;
__global__ void k_bg_vertical(const float* __restrict__ raw, const double* __restrict__ hsum,
                                                     int tile, int log_spect, int box, float* __restrict__ ctf)
{
    const int cx = tile / 2 + 1, cy = tile;
    const int m = blockIdx.y;
    const int y0 = blockIdx.x * kBgSegY, y1 = min(cy, y0 + kBgSegY);
    const size_t base = (size_t)m * cx * cy;
    const int hb = box / 2;
    const double norm = (double)box * (double)box;
    for (int x = threadIdx.x; x < cx; x += blockDim.x) {
        double sum = 0.0;
        for (int k = -hb; k <= hb; ++k) {
            int yy = y0 + k;
            if (yy < 0) yy += cy;
            else if (yy >= cy) yy -= cy;
            sum += hsum[base + (size_t)yy * cx + x];
        }
        for (int y = y0; y < y1; ++y) {
            if (y > y0) {
                int yin = y + hb, yout = y - 1 - hb;
                if (yin >= cy) yin -= cy;
                if (yout < 0) yout += cy;
                sum += hsum[base + (size_t)yin * cx + x] - hsum[base + (size_t)yout * cx + x];
            }
            const int i = y * cx + x;
            const int yr = y - cy / 2;
            float fr = x * 0.5f / (cx - 1);
            fr = sqrtf(fr * fr + yr * yr / (float)(cy * cy));
            if ((double)fr < 0.04) {
                ctf[base + i] = 0.0f;
                continue;
            }
            double b = sum / norm;
            if (!log_spect) b *= b;
            ctf[base + i] = (float)((double)raw[base + i] - b);
        }
    }
}

// Mean and second moment of each half spectrum (Util/GCalcMoment2D.cu:10-58).
// One block per spectrum; each thread keeps eight loads in flight.
__global__ void __launch_bounds__(1024) k_moments(const float* __restrict__ spect, int n,
                                                  double* __restrict__ out2)
{
    __shared__ double sh[64];
    int m = blockIdx.x;
    const float* p = spect + (size_t)m * n;
    const int S = blockDim.x;
    double v[2] = {0.0, 0.0};
    int i = threadIdx.x;
    for (; i + 7 * S < n; i += 8 * S) {
        double a[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = p[i + k * S];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v[0] += a[k];
            v[1] += a[k] * a[k];
        }
    }
    for (; i < n; i += S) {
        double a = p[i];
        v[0] += a;
        v[1] += a * a;
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        out2[2 * m] = v[0] / n;
        out2[2 * m + 1] = v[1] / n;
    }
}

// Full spectrum value (DC at column tile/2) from the half spectrum
// (FindCTF/GCalcSpectrum.cu:47-69; mirror row modulo tile).
__device__ __forceinline__ float full_val(const float* half, int tile, int y, int X)
{
    int cx = tile / 2 + 1, hx = cx - 1;
    int xd = X - hx;
    if (xd >= 0) return half[(size_t)y * cx + xd];
    int ys = tile - y;
    if (ys >= tile) ys -= tile;
    return half[(size_t)ys * cx - xd];
}

// CFindCtfBase::mLowpass (FindCTF/CFindCtfBase.cpp:191-219) around a batched
// R2C / C2R pair: the full spectrum (DC at column tile/2), the B-factor
// filter exp(-B (kx^2 + ky^2) / (2 tile^2)) of GLowpass2D::DoBFactor
// (FindCTF/GLowpass2D.cu:9-23) with the 1/tile^2 of the normalised forward
// transform, and the copy of columns tile/2 .. tile back into the half
// spectrum (the last one from the periodic neighbour, column 0).
__global__ void k_lp_full(const float* __restrict__ ctf0, int tile, float* __restrict__ full)
{
    int m = blockIdx.y;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tile * tile) return;
    int y = i / tile, X = i - y * tile;
    int cx = tile / 2 + 1;
    full[(size_t)m * tile * tile + i] = full_val(ctf0 + (size_t)m * cx * tile, tile, y, X);
}

// The filter depends on the tile size and B-factor only: one table per
// context, shared by every micrograph (the same double expression per bin).
__global__ void k_lp_table(double* __restrict__ g, int tile, double bfactor)
{
    int cx = tile / 2 + 1;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cx * tile) return;
    int y = i / cx, x = i - y * cx;
    int ky = (y > tile / 2) ? y - tile : y;
    double scale = -bfactor / ((double)tile * tile + (double)tile * tile);
    g[i] = exp(scale * ((double)x * x + (double)ky * ky)) / ((double)tile * tile);
}

__global__ void k_lp_filter(float2* __restrict__ cmp, int tile, const double* __restrict__ gtab)
{
    int m = blockIdx.y;
    int cx = tile / 2 + 1;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cx * tile) return;
    double g = gtab[i];
    float2 v = cmp[(size_t)m * cx * tile + i];
    cmp[(size_t)m * cx * tile + i] = make_float2((float)(v.x * g), (float)(v.y * g));
}

// Variance gate of mRemoveBackground (FindCTF/CFindCtfBase.cpp:169-174):
// micrographs whose background-removed spectrum has variance < 1 keep it
// unfiltered.
__global__ void k_lp_extract(const float* __restrict__ ctf0, const float* __restrict__ full, int tile,
                             const double* __restrict__ mom, float* __restrict__ out,
                             int* __restrict__ lowpassed)
{
    int m = blockIdx.y;
    int cx = tile / 2 + 1, hx = cx - 1;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mean = mom[2 * m], var = mom[2 * m + 1] - mean * mean;
    bool run = !(var < 1.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) lowpassed[m] = run ? 1 : 0;
    if (i >= cx * tile) return;
    size_t base = (size_t)m * cx * tile;
    if (!run) {
        out[base + i] = ctf0[base + i];
        return;
    }
    int y = i / cx, x = i - y * cx;
    int X = x + hx;
    if (X >= tile) X -= tile;
    out[base + i] = full[(size_t)m * tile * tile + (size_t)y * tile + X];
}

// GRadialAvg (FindCTF/GRadialAvg.cu:11-33) with the nearest-pixel sample
// table precomputed on the host.
// One warp per radius: the lanes stride over the ring's samples.
__global__ void k_radial(const float* __restrict__ spect, int cmp_n, int cx,
                         const int* __restrict__ off, const int* __restrict__ pix,
                         float* __restrict__ radial)
{
    int m = blockIdx.y;
    int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= cx) return;
    const float* p = spect + (size_t)m * cmp_n;
    double s = 0.0;
    int a = off[r], b = off[r + 1];
    for (int k = a + lane; k < b; k += 32) s += p[pix[k]];
    s = warp_sum(s);
    if (lane == 0) radial[(size_t)m * cx + r] = (float)(s / (b - a));
}

// Spectrum of each job gathered in band order, and its sum of squares.
__global__ void k_band_gather(const float* __restrict__ ctf, int cmp_n,
                              const SearchJob* __restrict__ jobs, const BandDev* __restrict__ bands,
                              const int* __restrict__ spec_off, float* __restrict__ band_spec,
                              double* __restrict__ sum_ss)
{
    __shared__ double sh[32];
    int j = blockIdx.x;
    const SearchJob& jb = jobs[j];
    const BandDev& b = bands[jb.band];
    const float* src = ctf + (size_t)jb.mic * cmp_n;
    float* dst = band_spec + spec_off[j];
    double v[1] = {0.0};
    const int S = blockDim.x;
    int k = threadIdx.x;
    for (; k + 3 * S < b.n; k += 4 * S) {   // four gathers in flight per thread
        int q[4];
        float s[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = b.idx[k + u * S];
#pragma unroll
        for (int u = 0; u < 4; ++u) s[u] = src[q[u]];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            dst[k + u * S] = s[u];
            v[0] += (double)s[u] * (double)s[u];
        }
    }
    for (; k < b.n; k += S) {
        float s = src[b.idx[k]];
        dst[k] = s;
        v[0] += (double)s * (double)s;
    }
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) sum_ss[j] = v[0];
}

// Signed CTF of GCalcCTF2D (FindCTF/GCalcCTF2D.cu:15-38), double, from a
// pixel's s^2 and polar angle.
__device__ double ctf_geo(double s2, double th, const PixOptics& o, double add, double mean, double sigma,
                          double az)
{
    double df = mean + sigma * cos(2.0 * (th - az));
    double chi = add + M_PI * (double)o.wl * s2 * (df - 0.5 * s2 * (double)o.wl * o.wl * o.cs);
    return -sin(chi);
}

// The same at one pixel (x, y) of the half spectrum.
__device__ double ctf_at(int x, int y, int cx, int cy, const PixOptics& o, double add,
                         double mean, double sigma, double az)
{
    double fx = x * 0.5 / (cx - 1);
    double fy = (double)(y - cy / 2) / cy;
    double s2 = fx * fx + fy * fy;
    double th = atan(fy / (fx + 1e-30));
    return ctf_geo(s2, th, o, add, mean, sigma, az);
}

// CSpectrumImage::mGenFullSpectrum + mEmbedCTF (FindCTF/CSpectrumImage.cpp:36-71,
// FindCTF/GCalcCTF2D.cu:49-78).
__global__ void k_full_spectrum(const float* __restrict__ ctf, int tile, const int* __restrict__ mic_of,
                                const gcf_result* __restrict__ res, const PixOptics* __restrict__ op,
                                const double* __restrict__ mom, float* __restrict__ full)
{
    int k = blockIdx.y;
    int m = mic_of[k];
    int cx = tile / 2 + 1, cy = tile, hx = cx - 1;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tile * tile) return;
    int y = i / tile, X = i - y * tile;
    const float* half = ctf + (size_t)m * cx * cy;
    float v = full_val(half, tile, y, X);
    const PixOptics o = op[k];
    const gcf_result r = res[k];
    // CFindCtfBase::Setup1 resolution range (FindCTF/CFindCtfBase.cpp:64-68)
    float r0 = 25.0f * o.px, r1 = (2.0f * o.px) / 0.8f;
    if (r1 < 3.5f) r1 = 3.5f;
    float fmn = o.px / r0, fmx = o.px / r1;
    if (X < hx) {
        float fy = (y - cy * 0.5f) / cy;
        float fx = (X - (float)hx) * 0.5f / hx;
        float rr = sqrtf(fx * fx + fy * fy);
        if (!(rr < fmn || rr > fmx)) {
            double mean = mom[2 * m], var = mom[2 * m + 1] - mean * mean;
            double sd = var < 0 ? 0.0 : sqrt(var);
            // CFindCtfBase::GenFullSpectrum (FindCTF/CFindCtfBase.cpp:118-126)
            float az = r.azimuth * 0.017453f;
            float dmin = r.df_min / o.px, dmax = r.df_max / o.px;
            float ph = fmodf(r.ext_phase * 0.01745329f, 3.14159265358979f);
            float mn = 0.5f * (dmin + dmax), sg = 0.5f * (dmax - dmin);
            int ix = hx - X, iy = (cy - y) % cy;
            double c = fabs(ctf_at(ix, iy, cx, cy, o, (double)(o.amp_phase + ph), mn, sg, az));
            v = (float)((c - 0.5) * (sd * 1.5) + mean);
        }
    }
    full[(size_t)k * tile * tile + i] = v;
}

// GSpectralCC2D::mGCalc2D (FindCTF/GSpectralCC2D.cu:12-110) in two steps:
// sums over the integer-radius rings (one CTF evaluation per pixel), then
// the Pearson CC of each width-10 shell from its rings.
__global__ void k_ring_sums(const float* __restrict__ ctf, int tile, const SearchJob* __restrict__ jobs,
                            const int* __restrict__ ring_off, const int* __restrict__ ring_pix,
                            const double2* __restrict__ ring_geo, double* __restrict__ ring_sums)
{
    __shared__ double sh[5 * 32];
    int ring = blockIdx.x, j = blockIdx.y;
    const SearchJob jb = jobs[j];
    int cx = tile / 2 + 1, cy = tile;
    const PixOptics o = jb.o;
    float dmin = jb.df_mean * (1.0f - jb.ast_ratio) / o.px;
    float dmax = jb.df_mean * (1.0f + jb.ast_ratio) / o.px;
    float mn = 0.5f * (dmin + dmax), sg = 0.5f * (dmax - dmin);
    double add = (double)(o.amp_phase + jb.ext_phase * 0.01745329f);
    double az = (double)(jb.ast_angle * 0.01745329f);
    const float* sp = ctf + (size_t)jb.mic * cx * cy;
    double v[5] = {0, 0, 0, 0, 0};
    for (int k = ring_off[ring] + threadIdx.x; k < ring_off[ring + 1]; k += blockDim.x) {
        int pix = ring_pix[k];
        const double2 g = ring_geo[k];   // (s^2, polar angle) of the pixel
        double c = ctf_geo(g.x, g.y, o, add, mn, sg, az);
        double s = sp[pix];
        v[0] += c * s;
        v[1] += c;
        v[2] += s;
        v[3] += c * c;
        v[4] += s * s;
    }
    block_sum<5>(v, sh);
    if (threadIdx.x == 0) {
        double* out = ring_sums + ((size_t)j * cx + ring) * 6;
        for (int q = 0; q < 5; ++q) out[q] = v[q];
        out[5] = (double)(ring_off[ring + 1] - ring_off[ring]);
    }
}

__global__ void k_shell_cc(int tile, const double* __restrict__ ring_sums, float* __restrict__ cc_out)
{
    int j = blockIdx.x;
    int cx = tile / 2 + 1;
    const int width = 10;
    for (int b = threadIdx.x; b < cx; b += blockDim.x) {
        int lo = b - width / 2, hi = lo + width;
        if (lo < 0) {
            lo = 0;
            hi = width;
        } else if (hi > cx) {
            lo = cx - width;
            hi = cx;
        }
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int ring = lo; ring < hi; ++ring)
            for (int q = 0; q < 6; ++q) v[q] += ring_sums[((size_t)j * cx + ring) * 6 + q];
        float out = 0.0f;
        if (v[5] > 0) {
            double n = v[5];
            double cs = v[0] / n, mc = v[1] / n, ms = v[2] / n, sc = v[3] / n, ss = v[4] / n;
            sc -= mc * mc;
            ss -= ms * ms;
            if (sc > 0 && ss > 0) out = (float)((cs - mc * ms) / sqrt(sc * ss));
        }
        cc_out[(size_t)j * cx + b] = out;
    }
}

}  // namespace

void launch_bg_horizontal(const float* raw, int tile, int nmic, int log_spect, double* hsum,
                          cudaStream_t st)
{
    // box of GRmBackground2D::mGRemove (FindCTF/GRmBackground2D.cu:33-36), fMinFreq = 1/15
    float fmin = 1.0f / 15.0f;
    int box = (int)(fmin * tile);
    if (box > (0.3f * tile)) box = (int)(0.3f * tile);
    box = box / 2 * 2 + 1;
    if (box < 7) box = 7;
    int cx = tile / 2 + 1, rb = bg_rows_per_block(tile);
    dim3 grid((tile + rb - 1) / rb, nmic);
    k_bg_horizontal<<<grid, 256, 2 * rb * cx * sizeof(float), st>>>(raw, tile, log_spect, box, hsum);
}

void launch_bg_vertical(const float* raw, const double* hsum, int tile, int nmic, int log_spect,
                        float* ctf, cudaStream_t st)
{
    float fmin = 1.0f / 15.0f;
    int box = (int)(fmin * tile);
    if (box > (0.3f * tile)) box = (int)(0.3f * tile);
    box = box / 2 * 2 + 1;
    if (box < 7) box = 7;
    int cx = tile / 2 + 1;
    int th = std::min(kBgVertThreads, ((cx + 31) / 32) * 32);
    dim3 grid((tile + kBgSegY - 1) / kBgSegY, nmic);
    k_bg_vertical<<<grid, th, 0, st>>>(raw, hsum, tile, log_spect, box, ctf);
}

void launch_moments(const float* spect, int n, int nmic, double* out2, cudaStream_t st)
{
    k_moments<<<nmic, 1024, 0, st>>>(spect, n, out2);
}

void launch_lp_full(const float* ctf0, int tile, int nmic, float* full, cudaStream_t st)
{
    dim3 grid((tile * tile + 255) / 256, nmic);
    k_lp_full<<<grid, 256, 0, st>>>(ctf0, tile, full);
}

void launch_lp_table(double* g, int tile, double bfactor, cudaStream_t st)
{
    int n = (tile / 2 + 1) * tile;
    k_lp_table<<<(n + 255) / 256, 256, 0, st>>>(g, tile, bfactor);
}

void launch_lp_filter(float2* cmp, int tile, int nmic, const double* g, cudaStream_t st)
{
    int n = (tile / 2 + 1) * tile;
    dim3 grid((n + 255) / 256, nmic);
    k_lp_filter<<<grid, 256, 0, st>>>(cmp, tile, g);
}

void launch_lp_extract(const float* ctf0, const float* full, int tile, int nmic, const double* moments,
                       float* out, int* lowpassed, cudaStream_t st)
{
    int n = (tile / 2 + 1) * tile;
    dim3 grid((n + 255) / 256, nmic);
    k_lp_extract<<<grid, 256, 0, st>>>(ctf0, full, tile, moments, out, lowpassed);
}

void launch_radial(const float* spect, int tile, int nmic, const int* off, const int* pix,
                   float* radial, cudaStream_t st)
{
    int cx = tile / 2 + 1;
    dim3 grid((cx + 7) / 8, nmic);
    k_radial<<<grid, 256, 0, st>>>(spect, cx * tile, cx, off, pix, radial);
}

void launch_band_gather(const float* ctf, int cmp_n, const SearchJob* jobs, const BandDev* bands,
                        const int* spec_off, int njobs, float* band_spec, double* sum_ss,
                        cudaStream_t st)
{
    if (njobs <= 0) return;
    k_band_gather<<<njobs, 1024, 0, st>>>(ctf, cmp_n, jobs, bands, spec_off, band_spec, sum_ss);
}

void launch_full_spectrum(const float* ctf, int tile, int nmic, const int* mic_of,
                          const gcf_result* res, const PixOptics* o, const double* moments,
                          float res_lo_freq_dummy, float* full, cudaStream_t st)
{
    (void)res_lo_freq_dummy;
    if (nmic <= 0) return;
    dim3 grid((tile * tile + 255) / 256, nmic);
    k_full_spectrum<<<grid, 256, 0, st>>>(ctf, tile, mic_of, res, o, moments, full);
}

void launch_ctf_res(const float* ctf, int tile, const SearchJob* jobs, int njobs, const int* ring_off,
                    const int* ring_pix, const double2* ring_geo, double* ring_sums, float* cc,
                    cudaStream_t st)
{
    if (njobs <= 0) return;
    dim3 grid(tile / 2 + 1, njobs);
    k_ring_sums<<<grid, 128, 0, st>>>(ctf, tile, jobs, ring_off, ring_pix, ring_geo, ring_sums);
    k_shell_cc<<<njobs, 128, 0, st>>>(tile, ring_sums, cc);
}

}  // namespace gcf
