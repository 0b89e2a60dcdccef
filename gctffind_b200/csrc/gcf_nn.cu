// gcf_nn.cu -- the learned initialiser's kernels: its inputs from a
// background-removed spectrum, the synthetic training spectra, and the
// layer pieces around the tensor-core products of gcf_umma.cu (im2col,
// col2im with the ReLU derivative, weight-gradient reductions, loss, Adam).
//
// Network (activations BF16, channel-last; weights FP32 masters with BF16
// copies for the products):
//   x2 : 256 x 256 polar half spectrum (angle rows x s^2 columns), 1 channel
//   conv1 4x4 stride 4, 1 -> 16   -> 64 x 64 x 16      (ReLU)
//   conv2 3x3 stride 2 pad 1, 16 -> 32 -> 32 x 32 x 32  (ReLU)
//   conv3 3x3 stride 2 pad 1, 32 -> 32 -> 16 x 16 x 32  (ReLU)
//   conv4 3x3 stride 2 pad 1, 32 -> 32 ->  8 x  8 x 32  (ReLU)
//   x1 : 256-bin rotational profile
//   fc1 [x1, conv4] 2304 -> 256 (ReLU), fc2 256 -> 128 (ReLU), fc3 128 -> 3
//   outputs: (mean defocus - 22500) / 10000, astigmatism / 1000 * (cos 2a, sin 2a)
// Forward layers and the input gradients run as tensor-core products
// (im2col rows x weights); weight gradients are reductions over the batch's
// rows (long K, few outputs) done here on the FP32 pipe.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "gcf_internal.h"

namespace gcf {

namespace {

constexpr float kPiF = 3.14159265358979f;

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// ---------------------------------------------------------------------------
// Seeded random numbers: a 64-bit mix of (seed, stream, counter) (the
// SplitMix64 finaliser), uniform in (0, 1), normal by Box-Muller.
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ float uni(uint64_t seed, uint64_t stream, uint64_t i)
{
    const uint64_t r = mix64(seed ^ mix64(stream * 0x632BE59BD9B4E019ull + i));
    return ((float)(r >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float gauss(uint64_t seed, uint64_t stream, uint64_t i)
{
    const float u1 = uni(seed, stream, 2 * i), u2 = uni(seed, stream, 2 * i + 1);
    return sqrtf(-2.0f * logf(u1)) * cosf(2.0f * kPiF * u2);
}

}  // namespace

// ---------------------------------------------------------------------------
// Network inputs from a background-removed half spectrum (tile/2+1 columns x
// tile rows, DC at (0, tile/2)) of pixel size px: pixels inside the fixed
// band s in [1/40, 1/3.5] 1/A are averaged into 256 s^2 bins x 256 angle
// bins (x2, angle rows) and 256 s^2 bins over all angles (x1); each is then
// standardised over its non-empty cells (empty cells 0).  One CTA per job;
// the angle bins are done in two halves of 128 so the sums fit in shared
// memory.  Angle bin t = (atan2(fy, fx) + pi/2) * 256 / pi: rows above the
// DC row (fy < 0, |angle| >= atan(1/256) off the axis) fall in t < 128 and
// the others in t >= 128, so each half visits only its own rows, one warp
// per row over the row's in-band column interval.
__global__ void __launch_bounds__(1024)
k_nn_input(const float* __restrict__ ctf, int tile, const float* __restrict__ px_of, int px_stride,
           __nv_bfloat16* __restrict__ x1, __nv_bfloat16* __restrict__ x2)
{
    extern __shared__ float nsm[];
    float* sum = nsm;                                                   // [128][256]
    unsigned short* cnt = reinterpret_cast<unsigned short*>(nsm + 128 * 256);   // [128][256]
    __shared__ float s_prof[256];
    __shared__ int s_pcnt[256];
    __shared__ double s_red[4][32];
    const int j = blockIdx.x;
    const int cx = tile / 2 + 1, cy = tile;
    const float px = px_of[(size_t)j * px_stride];
    const float* S = ctf + (size_t)j * cx * cy;
    const float s2lo = 1.0f / 1600.0f, s2hi = 1.0f / 12.25f;
    const float ds2 = (s2hi - s2lo) / 256.0f;
    const float inv_px2 = 1.0f / (px * px);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        s_prof[i] = 0.0f;
        s_pcnt[i] = 0;
    }
    double m2 = 0.0, q2 = 0.0, n2 = 0.0;
    for (int half = 0; half < 2; ++half) {
        for (int i = threadIdx.x; i < 128 * 256; i += blockDim.x) {
            sum[i] = 0.0f;
            cnt[i] = 0;
        }
        __syncthreads();
        for (int yr = warp; yr < cy / 2; yr += nwarps) {
            const int y = half * (cy / 2) + yr;
            const float fy = (float)(y - cy / 2) / (float)tile;
            // columns whose s^2 can fall in [s2lo, s2hi), one column of slack on
            // each side; the exact test below decides
            const float alo = s2lo * px * px - fy * fy, ahi = s2hi * px * px - fy * fy;
            const int xlo = alo > 0.0f ? max((int)(sqrtf(alo) * (float)tile) - 1, 0) : 0;
            const int xhi = min(ahi > 0.0f ? (int)(sqrtf(ahi) * (float)tile) + 2 : 2, cx);
            for (int x = xlo + lane; x < xhi; x += 32) {
                const float fx = (float)x / (float)tile;
                const float s2 = (fx * fx + fy * fy) * inv_px2;
                if (s2 < s2lo || s2 >= s2hi) continue;
                const int k = min(max((int)((s2 - s2lo) / ds2), 0), 255);
                const int t = min(max((int)((atan2f(fy, fx) + 0.5f * kPiF) * (256.0f / kPiF)), 0), 255);
                if ((t >> 7) != half) continue;
                const float v = S[(size_t)y * cx + x];
                const int c = (t & 127) * 256 + k;
                atomicAdd(&sum[c], v);
                // counts stay below 65536: at most a few hundred pixels per cell
                atomicAdd(reinterpret_cast<unsigned int*>(&cnt[c & ~1]), (c & 1) ? 65536u : 1u);
            }
        }
        __syncthreads();
        // the profile's sums from this half's cells (every band pixel is in
        // exactly one cell of one half)
        for (int k = threadIdx.x; k < 256; k += blockDim.x) {
            float ps = 0.0f;
            int pc = 0;
            for (int t = 0; t < 128; ++t) {
                ps += sum[t * 256 + k];
                pc += cnt[t * 256 + k];
            }
            s_prof[k] += ps;
            s_pcnt[k] += pc;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < 128 * 256; i += blockDim.x) {
            const int n = cnt[i];
            const float v = n ? sum[i] / (float)n : 0.0f;
            sum[i] = v;
            if (n) {
                m2 += v;
                q2 += (double)v * v;
                n2 += 1.0;
            }
        }
        __syncthreads();
        // keep the means in the output (standardised below)
        for (int i = threadIdx.x; i < 128 * 256; i += blockDim.x)
            x2[(size_t)j * 65536 + (size_t)half * 32768 + i] = __float2bfloat16_rn(cnt[i] ? sum[i] : 0.0f);
        __syncthreads();
    }
    // standardise x2 over non-empty cells
    for (int o = 16; o > 0; o >>= 1) {
        m2 += __shfl_xor_sync(0xffffffffu, m2, o);
        q2 += __shfl_xor_sync(0xffffffffu, q2, o);
        n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    }
    if (lane == 0) {
        s_red[0][warp] = m2;
        s_red[1][warp] = q2;
        s_red[2][warp] = n2;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        double a = 0, b = 0, c = 0;
        if (threadIdx.x < (blockDim.x >> 5)) {
            a = s_red[0][threadIdx.x];
            b = s_red[1][threadIdx.x];
            c = s_red[2][threadIdx.x];
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (threadIdx.x == 0) {
            const double mean = c > 0 ? a / c : 0.0;
            const double var = c > 0 ? b / c - mean * mean : 0.0;
            s_red[3][0] = mean;
            s_red[3][1] = var > 1e-30 ? 1.0 / sqrt(var) : 0.0;
        }
    }
    __syncthreads();
    const float mean2 = (float)s_red[3][0], inv2 = (float)s_red[3][1];
    for (int i = threadIdx.x; i < 65536; i += blockDim.x) {
        __nv_bfloat16* q = x2 + (size_t)j * 65536 + i;
        const float v = bf(*q);
        *q = __float2bfloat16_rn(v != 0.0f ? (v - mean2) * inv2 : 0.0f);
    }
    // profile: mean per bin, standardised over non-empty bins
    if (threadIdx.x < 32) {
        double a = 0, b = 0, c = 0;
        for (int k = threadIdx.x; k < 256; k += 32) {
            if (!s_pcnt[k]) continue;
            const double v = s_prof[k] / s_pcnt[k];
            a += v;
            b += v * v;
            c += 1.0;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (threadIdx.x == 0) {
            const double mean = c > 0 ? a / c : 0.0;
            const double var = c > 0 ? b / c - mean * mean : 0.0;
            s_red[3][2] = mean;
            s_red[3][3] = var > 1e-30 ? 1.0 / sqrt(var) : 0.0;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 256; k += blockDim.x) {
        const float v = s_pcnt[k] ? s_prof[k] / (float)s_pcnt[k] : 0.0f;
        x1[(size_t)j * 256 + k] =
            __float2bfloat16_rn(s_pcnt[k] ? (float)((v - s_red[3][2]) * s_red[3][3]) : 0.0f);
    }
}

// ---------------------------------------------------------------------------
// Synthetic training spectra: the expected averaged amplitude spectrum of
// the micrograph model of gctffind_b200/synth.py (white object through
// CTF x exp(-B s^2 / 4), B = 100 A^2; smooth background of amplitude
// 1 / (f^2 + f0^2), f0 = 1/200 A; Poisson counts at dose D), with the
// tile-averaging noise of a Rayleigh amplitude averaged over the tiles.
// params[j]: (mean df A, astig A, angle rad, px_n A, dose, tiles, raw px A, scale)
__global__ void k_synth_params(unsigned long long seed, unsigned long long first, int n, float* __restrict__ params,
                               float* __restrict__ target)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint64_t id = first + (uint64_t)j;
    const float df = 5000.0f + 35000.0f * uni(seed, id, 0);
    const float ast = 1000.0f * uni(seed, id, 1);
    const float ang = kPiF * uni(seed, id, 2) - 0.5f * kPiF;
    const float px_raw = 0.8f + 0.7f * uni(seed, id, 3);
    const float px = fmaxf(px_raw, 1.2f);
    const float dose = 0.5f + 1.5f * uni(seed, id, 4);
    // sizes of the uneven batch (4096^2, 5760 x 4092, 3838 x 3710) after rescale, in tiles of 512
    const int sz = min((int)(3.0f * uni(seed, id, 5)), 2);
    const float W = (sz == 0 ? 4096.0f : sz == 1 ? 5760.0f : 3838.0f) * px_raw / px;
    const float H = (sz == 0 ? 4096.0f : sz == 1 ? 4092.0f : 3710.0f) * px_raw / px;
    const float tiles = floorf((W - 256.0f) / 256.0f) * floorf((H - 256.0f) / 256.0f);
    float* p = params + (size_t)j * 8;
    p[0] = df;
    p[1] = ast;
    p[2] = ang;
    p[3] = px;
    p[4] = dose;
    p[5] = tiles;
    p[6] = px_raw;
    p[7] = px_raw < px ? W * H : 1.0f;   // unnormalised inverse FFT of the Fourier crop
    target[(size_t)j * 3 + 0] = (df - 22500.0f) / 10000.0f;
    target[(size_t)j * 3 + 1] = ast / 1000.0f * cosf(2.0f * ang);
    target[(size_t)j * 3 + 2] = ast / 1000.0f * sinf(2.0f * ang);
}

__global__ void k_synth_raw(unsigned long long seed, unsigned long long first, const float* __restrict__ params,
                            int tile, PixOptics base, float* __restrict__ raw)
{
    const int j = blockIdx.y;
    const int cx = tile / 2 + 1, cy = tile;
    const float* p = params + (size_t)j * 8;
    const float df = p[0], sig = 0.5f * p[1], ang = p[2], px = p[3], dose = p[4], tiles = p[5];
    const float px_raw = p[6], scale = p[7];
    const float wl = base.wl, cs = base.cs;   // Angstrom here
    const float phi = base.amp_phase;
    // mean |h|^2 over the raw sampling's frequency square: CTF^2 averages to
    // 1/2 and the envelope factorises, exp(-50 s^2) per axis
    const float a = 0.5f / px_raw;
    const float ax = sqrtf(kPiF / 50.0f) * erff(a * sqrtf(50.0f)) / (2.0f * a);
    const float h2 = 0.5f * ax * ax;
    const float f0 = 1.0f / 200.0f;
    const float b2 = kPiF / (f0 * f0 * 4.0f * a * a);   // mean 1 / (f^2 + f0^2)^2 over the square
    const float dp = dose * px_raw * px_raw;
    const float sig_c = dp * 0.5f, bg_c = dp * 0.3f;
    const float n_eff = fmaxf(0.5f * tiles, 1.0f);
    const uint64_t id = first + (uint64_t)j;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cx * cy; q += gridDim.x * blockDim.x) {
        const int y = q / cx, x = q - y * cx;
        const float fx = (float)x / (float)tile / px, fy = (float)(y - cy / 2) / (float)tile / px;
        const float s2 = fx * fx + fy * fy;
        const float th = atan2f(fy, fx);
        const float z = df + sig * cosf(2.0f * (th - ang));
        const float chi = kPiF * wl * s2 * (z - 0.5f * wl * wl * s2 * cs) + phi;
        const float env = expf(-25.0f * s2);
        const float h = sinf(chi) * env;
        const float bgf = 1.0f / (s2 + f0 * f0);
        const float P = dp + sig_c * sig_c * h * h / h2 + bg_c * bg_c * bgf * bgf / b2;
        const float mean = 0.5f * sqrtf(kPiF * P);
        const float sd = sqrtf((1.0f - 0.25f * kPiF) * P / n_eff);
        const float v = fmaxf(mean + sd * gauss(seed ^ 0x5A5A5A5Aull, id, (uint64_t)q), 0.0f);
        raw[(size_t)j * cx * cy + q] = v * scale;
    }
}

// ---------------------------------------------------------------------------
// im2col of the 4 x 4 stride-4 first layer on the 256 x 256 x 1 input:
// row (b, oy, ox) = the 16 pixels of patch (oy, ox), (ky, kx) order.  One
// thread per (row, ky): 4 contiguous BF16 (8 bytes) in and out.
__global__ void k_im2col_p4(const __nv_bfloat16* __restrict__ x, int B, __nv_bfloat16* __restrict__ cols)
{
    const long long n = (long long)B * 4096 * 4;
    const uint2* __restrict__ xv = reinterpret_cast<const uint2*>(x);
    uint2* __restrict__ cv = reinterpret_cast<uint2*>(cols);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ky = (int)(i & 3);
        const long long r = i >> 2;
        const int ox = (int)(r & 63), oy = (int)((r >> 6) & 63);
        const long long b = r >> 12;
        // x row (oy * 4 + ky), columns ox * 4 .. ox * 4 + 3: uint2 index / 4 pixels
        cv[i] = xv[(size_t)b * 16384 + (oy * 4 + ky) * 64 + ox];
    }
}

// The first layer directly (no im2col rows): output row (b, oy, ox) is
// ReLU(bias + W x) for the 16 pixels x of patch (oy, ox) in (ky, kx) order,
// as the tensor-core product of those rows computes it (FP32 sums of the
// BF16 products, rounded to BF16); W is [16 out][16 in] BF16.  One thread
// per output row: four 8-byte patch-row loads, 256 FMAs, two 16-byte
// stores.
__global__ void __launch_bounds__(256) k_conv1_direct(const __nv_bfloat16* __restrict__ x, int B,
                                                      const __nv_bfloat16* __restrict__ w,
                                                      const float* __restrict__ bias,
                                                      __nv_bfloat16* __restrict__ y)
{
    __shared__ float sw[16][17];
    __shared__ float sb[16];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sw[i >> 4][i & 15] = __bfloat162float(w[i]);
    if (threadIdx.x < 16) sb[threadIdx.x] = bias[threadIdx.x];
    __syncthreads();
    const long long n = (long long)B * 4096;
    const uint2* __restrict__ xv = reinterpret_cast<const uint2*>(x);
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        const int ox = (int)(r & 63), oy = (int)((r >> 6) & 63);
        const long long b = r >> 12;
        float in[16];
#pragma unroll
        for (int ky = 0; ky < 4; ++ky) {
            const uint2 q = xv[(size_t)b * 16384 + (oy * 4 + ky) * 64 + ox];
            const __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162*>(&q.x);
            const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162*>(&q.y);
            in[4 * ky + 0] = __low2float(lo);
            in[4 * ky + 1] = __high2float(lo);
            in[4 * ky + 2] = __low2float(hi);
            in[4 * ky + 3] = __high2float(hi);
        }
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll 2
        for (int c = 0; c < 16; ++c) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 16; ++k) acc = fmaf(sw[c][k], in[k], acc);
            o[c] = __float2bfloat16_rn(fmaxf(acc + sb[c], 0.0f));
        }
        uint4* yv = reinterpret_cast<uint4*>(y + (size_t)r * 16);
        yv[0] = *reinterpret_cast<const uint4*>(&o[0]);
        yv[1] = *reinterpret_cast<const uint4*>(&o[8]);
    }
}

// im2col of a 3 x 3 stride-2 pad-1 layer on channel-last [B][H][W][C]:
// row (b, oy, ox), column (ky * 3 + kx) * C + c.  One thread per (row, tap,
// 8 channels): 16 bytes in and out (C a multiple of 8).
__global__ void k_im2col_3s2(const __nv_bfloat16* __restrict__ x, int B, int H, int W, int C,
                             __nv_bfloat16* __restrict__ cols)
{
    const int OH = H / 2, OW = W / 2, C8 = C / 8, K8 = 9 * C8;
    const long long n = (long long)B * OH * OW * K8;
    const uint4* __restrict__ xv = reinterpret_cast<const uint4*>(x);
    uint4* __restrict__ cv = reinterpret_cast<uint4*>(cols);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / K8;
        const int col8 = (int)(i - r * K8);
        const int kk = col8 / C8, c8 = col8 - kk * C8;
        const int ky = kk / 3, kx = kk - 3 * ky;
        const int ox = (int)(r % OW);
        const long long r2 = r / OW;
        const int oy = (int)(r2 % OH);
        const long long b = r2 / OH;
        const int yy = 2 * oy - 1 + ky, xx = 2 * ox - 1 + kx;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);   // BF16 zero is all-zero bits
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = xv[((b * H + yy) * W + xx) * C8 + c8];
        cv[i] = v;
    }
}

// Gradient of a 3 x 3 stride-2 pad-1 layer's input from its im2col
// gradient dcols (FP32, [B*OH*OW][9C]), times the ReLU derivative of the
// input activation y (> 0), as BF16 [B][H][W][C].
__global__ void k_col2im_3s2_relu(const float* __restrict__ dcols, const __nv_bfloat16* __restrict__ y, int B,
                                  int H, int W, int C, __nv_bfloat16* __restrict__ dz)
{
    const int OH = H / 2, OW = W / 2, K = 9 * C;
    const long long n = (long long)B * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long r = i / C;
        const int xx = (int)(r % W), yy = (int)((r / W) % H), b = (int)(r / ((long long)W * H));
        float s = 0.0f;
        if (bf(y[i]) > 0.0f) {
            // output rows oy with 2 oy - 1 + ky = yy, ky in 0..2
            for (int ky = 0; ky < 3; ++ky) {
                const int t = yy + 1 - ky;
                if (t < 0 || (t & 1)) continue;
                const int oy = t >> 1;
                if (oy >= OH) continue;
                for (int kx = 0; kx < 3; ++kx) {
                    const int u = xx + 1 - kx;
                    if (u < 0 || (u & 1)) continue;
                    const int ox = u >> 1;
                    if (ox >= OW) continue;
                    s += dcols[(((size_t)b * OH + oy) * OW + ox) * K + (ky * 3 + kx) * C + c];
                }
            }
        }
        dz[i] = __float2bfloat16_rn(s);
    }
}

// dz = dy * (y > 0) (FP32 in, BF16 out), rows of n columns with pitches.
__global__ void k_relu_bwd(const float* __restrict__ dy, long long ldy, const __nv_bfloat16* __restrict__ y,
                           long long ldyy, int rows, int n, __nv_bfloat16* __restrict__ dz, long long ldz)
{
    const long long tot = (long long)rows * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / n), c = (int)(i % n);
        const float v = bf(y[(size_t)r * ldyy + c]) > 0.0f ? dy[(size_t)r * ldy + c] : 0.0f;
        dz[(size_t)r * ldz + c] = __float2bfloat16_rn(v);
    }
}

// fc1 input: [profile (256) | conv4 output (2048)] per sample.
__global__ void k_concat(const __nv_bfloat16* __restrict__ x1, const __nv_bfloat16* __restrict__ y4, int B,
                         __nv_bfloat16* __restrict__ h0)
{
    const long long n = (long long)B * 2304;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / 2304), c = (int)(i % 2304);
        h0[i] = c < 256 ? x1[(size_t)b * 256 + c] : y4[(size_t)b * 2048 + (c - 256)];
    }
}

// Weight and bias gradients dW[o][k] += sum_r dz[r][o] x[r][k],
// db[o] += sum_r dz[r][o]: 32 x 32 output tiles, each CTA a slice of rows
// staged through shared memory, FP32 sums, atomics into dW.
__global__ void __launch_bounds__(256)
k_wgrad(const __nv_bfloat16* __restrict__ dz, long long ldz, const __nv_bfloat16* __restrict__ x, long long ldx,
        int rows, int nout, int nin, int rows_per_cta, float* __restrict__ dw, float* __restrict__ db)
{
    __shared__ float sz[32][33], sx[32][33];
    const int o0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    const int r0 = blockIdx.z * rows_per_cta, r1 = min(rows, r0 + rows_per_cta);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 8 row groups
    float acc[4] = {0, 0, 0, 0}, bacc = 0.0f;
    for (int rb = r0; rb < r1; rb += 32) {
        for (int q = ty; q < 32; q += 8) {
            const int r = rb + q;
            sz[q][tx] = (r < r1 && o0 + tx < nout) ? bf(dz[(size_t)r * ldz + o0 + tx]) : 0.0f;
            sx[q][tx] = (r < r1 && k0 + tx < nin) ? bf(x[(size_t)r * ldx + k0 + tx]) : 0.0f;
        }
        __syncthreads();
        // thread (ty, tx): outputs o = o0 + ty + 8 i, k = k0 + tx
        for (int q = 0; q < 32; ++q) {
            const float xv = sx[q][tx];
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[i] = fmaf(sz[q][ty + 8 * i], xv, acc[i]);
            if (blockIdx.x == 0 && ty == 0) bacc += sz[q][tx];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int o = o0 + ty + 8 * i, k = k0 + tx;
        if (o < nout && k < nin) atomicAdd(dw + (size_t)o * nin + k, acc[i]);
    }
    if (blockIdx.x == 0 && ty == 0 && o0 + tx < nout && db) atomicAdd(db + o0 + tx, bacc);
}

// Mean squared error over the 3 outputs: loss (atomic) and
// dpred = 2 (pred - target) / (3 B) as BF16 rows of pitch 8 (zero padded).
__global__ void k_mse(const float* __restrict__ pred, long long ldp, const float* __restrict__ target, int B,
                      float* __restrict__ loss, __nv_bfloat16* __restrict__ dpred)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    float l = 0.0f;
    for (int c = 0; c < 8; ++c) {
        float g = 0.0f;
        if (c < 3) {
            const float d = pred[(size_t)b * ldp + c] - target[(size_t)b * 3 + c];
            l += d * d;
            g = 2.0f * d / (3.0f * B);
        }
        dpred[(size_t)b * 8 + c] = __float2bfloat16_rn(g);
    }
    atomicAdd(loss, l / (3.0f * B));
}

// Adam on FP32 masters; writes the BF16 copies W [out][in] (pitch in) and
// W^T [in][out] (pitch ldt).  The bias follows the weights in the masters.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                       int nout, int nin, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wt,
                       long long ldt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (i < nout * nin) {
            const int o = i / nin, k = i - o * nin;
            const __nv_bfloat16 q = __float2bfloat16_rn(wi);
            wb[i] = q;
            wt[(size_t)k * ldt + o] = q;
        }
    }
}

// BF16 copies of a layer's weights without an update.
__global__ void k_copy_weights(const float* __restrict__ w, int nout, int nin, __nv_bfloat16* __restrict__ wb,
                               __nv_bfloat16* __restrict__ wt, long long ldt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nout * nin; i += gridDim.x * blockDim.x) {
        const int o = i / nin, k = i - o * nin;
        const __nv_bfloat16 q = __float2bfloat16_rn(w[i]);
        wb[i] = q;
        wt[(size_t)k * ldt + o] = q;
    }
}

// Predictions -> search prior (mean A, astigmatism ratio, angle degrees,
// window scale 1).
__global__ void k_prior(const float* __restrict__ pred, long long ldp, int n, float4* __restrict__ prior)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const float* p = pred + (size_t)j * ldp;
    const float mu = fminf(fmaxf(22500.0f + 10000.0f * p[0], 1000.0f), 200000.0f);
    const float a = 1000.0f * sqrtf(p[1] * p[1] + p[2] * p[2]);
    const float ang = 0.5f * atan2f(p[2], p[1]) * (180.0f / kPiF);
    prior[j] = make_float4(mu, 0.5f * a / mu, ang, 1.0f);
}

// ---------------------------------------------------------------------------
// Launchers
static inline int grid_for(long long n, int threads) { return (int)std::min<long long>((n + threads - 1) / threads, 148LL * 16); }

cudaError_t launch_nn_input(const float* ctf, int tile, const float* px, int px_stride, int n, __nv_bfloat16* x1,
                            __nv_bfloat16* x2, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const size_t sm = 128 * 256 * (sizeof(float) + sizeof(unsigned short));
    cudaError_t e = cudaFuncSetAttribute(k_nn_input, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_nn_input<<<n, 1024, sm, st>>>(ctf, tile, px, px_stride, x1, x2);
    return cudaGetLastError();
}

void launch_synth_params(unsigned long long seed, unsigned long long first, int n, float* params, float* target,
                         cudaStream_t st)
{
    if (n <= 0) return;
    k_synth_params<<<(n + 127) / 128, 128, 0, st>>>(seed, first, n, params, target);
}

void launch_synth_raw(unsigned long long seed, unsigned long long first, const float* params, int n, int tile,
                      const PixOptics& base, float* raw, cudaStream_t st)
{
    if (n <= 0) return;
    k_synth_raw<<<dim3(32, n), 256, 0, st>>>(seed, first, params, tile, base, raw);
}

void launch_im2col_p4(const __nv_bfloat16* x, int B, __nv_bfloat16* cols, cudaStream_t st)
{
    k_im2col_p4<<<grid_for((long long)B * 4096 * 4, 256), 256, 0, st>>>(x, B, cols);
}

void launch_conv1_direct(const __nv_bfloat16* x, int B, const __nv_bfloat16* w, const float* bias,
                         __nv_bfloat16* y, cudaStream_t st)
{
    k_conv1_direct<<<grid_for((long long)B * 4096, 256), 256, 0, st>>>(x, B, w, bias, y);
}

void launch_im2col_3s2(const __nv_bfloat16* x, int B, int H, int W, int C, __nv_bfloat16* cols, cudaStream_t st)
{
    // C is 16 or 32 here: 16-byte channel groups, buffers 256-byte aligned
    k_im2col_3s2<<<grid_for((long long)B * (H / 2) * (W / 2) * 9 * (C / 8), 256), 256, 0, st>>>(x, B, H, W, C, cols);
}

void launch_col2im_3s2_relu(const float* dcols, const __nv_bfloat16* y, int B, int H, int W, int C,
                            __nv_bfloat16* dz, cudaStream_t st)
{
    k_col2im_3s2_relu<<<grid_for((long long)B * H * W * C, 256), 256, 0, st>>>(dcols, y, B, H, W, C, dz);
}

void launch_relu_bwd(const float* dy, long long ldy, const __nv_bfloat16* y, long long ldyy, int rows, int n,
                     __nv_bfloat16* dz, long long ldz, cudaStream_t st)
{
    k_relu_bwd<<<grid_for((long long)rows * n, 256), 256, 0, st>>>(dy, ldy, y, ldyy, rows, n, dz, ldz);
}

void launch_concat(const __nv_bfloat16* x1, const __nv_bfloat16* y4, int B, __nv_bfloat16* h0, cudaStream_t st)
{
    k_concat<<<grid_for((long long)B * 2304, 256), 256, 0, st>>>(x1, y4, B, h0);
}

void launch_wgrad(const __nv_bfloat16* dz, long long ldz, const __nv_bfloat16* x, long long ldx, int rows, int nout,
                  int nin, float* dw, float* db, cudaStream_t st)
{
    const int gx = (nin + 31) / 32, gy = (nout + 31) / 32;
    // enough row slices to give every SM a few CTAs
    int slices = std::max(1, std::min((rows + 255) / 256, (148 * 4 + gx * gy - 1) / (gx * gy)));
    const int per = ((rows + slices - 1) / slices + 31) / 32 * 32;
    slices = (rows + per - 1) / per;
    k_wgrad<<<dim3(gx, gy, slices), 256, 0, st>>>(dz, ldz, x, ldx, rows, nout, nin, per, dw, db);
}

void launch_mse(const float* pred, long long ldp, const float* target, int B, float* loss, __nv_bfloat16* dpred,
                cudaStream_t st)
{
    k_mse<<<(B + 127) / 128, 128, 0, st>>>(pred, ldp, target, B, loss, dpred);
}

void launch_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                 float c1, float c2, int nout, int nin, __nv_bfloat16* wb, __nv_bfloat16* wt, long long ldt,
                 cudaStream_t st)
{
    k_adam<<<grid_for(n, 256), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, nout, nin, wb, wt, ldt);
}

void launch_copy_weights(const float* w, int nout, int nin, __nv_bfloat16* wb, __nv_bfloat16* wt, long long ldt,
                         cudaStream_t st)
{
    k_copy_weights<<<grid_for((long long)nout * nin, 256), 256, 0, st>>>(w, nout, nin, wb, wt, ldt);
}

void launch_prior(const float* pred, long long ldp, int n, float4* prior, cudaStream_t st)
{
    if (n <= 0) return;
    k_prior<<<(n + 127) / 128, 128, 0, st>>>(pred, ldp, n, prior);
}

}  // namespace gcf
