// gcf_rsgemm.cu -- the Fourier-crop rescale of CRescaleImage::DoIt
// (FindCTF/CRescaleImage.cpp:76-99, Util/GFtResize2D.cu:124-143) as two
// BF16 tensor-core products.
//
// The rescale (R2C of the raw w x h frame, crop to (nw/2 + 1) x nh, C2R of
// nw x nh, all unnormalised) is linear and nearly separable.  With
//   Rw[x][j] = sum_k c_k cos(2 pi k (x/nw - j/w)),  k = 0 .. nw/2
//              (c_0 = c_{nw/2} = 1, else 2: the C2R's Hermitian weights),
//   Rh[y][i] = the real part of the column map (forward DFT of length h,
//              keep frequencies -(nh/2 - 1) .. nh/2, inverse DFT of nh),
// the output is
//   out = Rh img Rw^T - a v^T,   a[y] = (-1)^y,
// where the rank-one term comes from the kept +nh/2 column frequency (its
// -nh/2 partner is dropped, so the column map is complex there):
//   v = Iw u,  u[j] = sum_i b[i] img[i][j],  b[i] = -sin(pi i nh / h),
//   Iw[x][j] = sum_k c_k sin(2 pi k (x/nw - j/w)).
// Both real maps have the closed form (t = r/n_out - c/n_in)
//   M[r][c] = -(-1)^r sin(pi c n_out / n_in) cot(pi t)   (n_out at t = 0),
// and Iw[x][j] = (1 - (-1)^x cos(pi j nw / w)) cot(pi t)  (0 at t = 0).
//
// A constant image c maps to c w h, so the BF16 copy holds img - c (c: the
// mean of 256 pixels of the middle row), and the second product adds c w h
// back in FP32 as a per-column bias: the BF16 rounding then scales with the
// image's fluctuations, not with its mean.
//
// So: img -> BF16 (with the column sums u), the two maps in BF16, then
//   T^T = (img Rw^T)^T    (nw x h, BF16; the product's transposed output),
//   out = Rh' T'^T + c w h (FP32), Rh' = [Rh | -a], T' = [T^T | v]:
// the rank-one term rides in one extra K column of the second product.
// The maps cost O(n_out n_in) to write, far less than the products.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "gcf_internal.h"

namespace gcf {

namespace {

constexpr int kRsgChunks = 64;        // row chunks of the conversion (partial column sums)
constexpr int kRsgRowsPerBlock = 32;  // map rows per block
constexpr int kRsgVx = 4;             // x values per block of the rank-one kernel

// pi p / q as the argument of sinpif / cospif, reduced exactly to (-1, 1]
// (p >= 0; p and 2q below 2^31: sides <= 16384)
__device__ __forceinline__ float ratio_arg(int p, int q)
{
    int r = p % (2 * q);
    if (r > q) r -= 2 * q;
    return (float)r / (float)q;
}

// cot(pi t), t = num / den with |num| < den, from the angles' sines and
// cosines (t = alpha - beta, alpha = r / n_out, beta = c / n_in).  Near
// t = 0 the difference formula loses precision, so |t| < 1/64 takes the
// direct sincos of the exactly formed ratio.
__device__ __forceinline__ float cot_pi_diff(int num, float inv_den, float sa, float ca, float sb, float cb,
                                             bool near)
{
    if (near) {
        float s, c;
        sincospif((float)num * inv_den, &s, &c);
        return __fdividef(c, s);
    }
    return __fdividef(fmaf(ca, cb, sa * sb), fmaf(sa, cb, -ca * sb));
}

// The centring constant c: the mean of the first min(w, 256) pixels of the
// middle row, summed in a fixed order, so every block that calls it gets the
// same value.  All 256 threads call it; red: 8 floats of shared memory.
__device__ float block_centre(const float* __restrict__ img, long long ip, int w, int h, float* red)
{
    const int n = min(w, 256);
    float s = threadIdx.x < n ? __ldg(img + (size_t)(h / 2) * ip + threadIdx.x) : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += red[k];
    __syncthreads();
    return t / (float)n;
}

struct PrepArgs {
    const float* img;
    long long ip;
    int w, h, nw, nh;
    __nv_bfloat16 *X, *Wm, *Km;
    long long ldw, ldk;
    float* part;
    int n_conv, n_wmap;     // blocks of the conversion and of the row map; the column map's follow
    int cb, kcb;            // column blocks of the conversion / row map and of the column map
};

// img - c (FP32, pitch ip) -> X (BF16, pitch ldx), rows of chunk `chunk`;
// part[chunk][j] = sum over the chunk's rows of b[i] (img[i][j] - c),
// b[i] = -sin(pi i nh / h).
__device__ void prep_convert(const PrepArgs& a, int colblk, int chunk, float* sh)
{
    const float c = block_centre(a.img, a.ip, a.w, a.h, sh + 256);
    const int rows = (a.h + kRsgChunks - 1) / kRsgChunks;   // <= 256 for h <= 16384
    const int i0 = chunk * rows, i1 = min(i0 + rows, a.h);
    for (int k = threadIdx.x; k < i1 - i0; k += 256) sh[k] = -sinpif(ratio_arg((i0 + k) * a.nh, a.h));
    __syncthreads();
    const int j = colblk * 256 + threadIdx.x;
    if (j >= a.w) return;
    float acc = 0.0f;
#pragma unroll 4
    for (int i = i0; i < i1; ++i) {
        const float v = __ldg(a.img + (size_t)i * a.ip + j) - c;
        a.X[(size_t)i * a.ldw + j] = __float2bfloat16_rn(v);
        acc = fmaf(sh[i - i0], v, acc);
    }
    a.part[(size_t)chunk * a.w + j] = acc;
}

// Rows rowblk * kRsgRowsPerBlock .. of the crop map M (n_out x n_in, BF16,
// row pitch ld); extra: one more column n_in holding -(-1)^r (the rank-one
// term's left factor).
__device__ void prep_map(__nv_bfloat16* M, long long ld, int n_out, int n_in, int extra, int colblk, int rowblk,
                         float* sh)
{
    float2* rsc = reinterpret_cast<float2*>(sh);
    const int r0 = rowblk * kRsgRowsPerBlock;
    const int r1 = min(r0 + kRsgRowsPerBlock, n_out);
    if (threadIdx.x < r1 - r0) {
        float s, c;
        sincospif(ratio_arg(r0 + threadIdx.x, n_out), &s, &c);
        rsc[threadIdx.x] = make_float2(s, c);
    }
    __syncthreads();
    const int c = colblk * 256 + threadIdx.x;
    if (c < n_in) {
        const float S = sinpif(ratio_arg(c * n_out, n_in));
        float sb, cb;
        sincospif(ratio_arg(c, n_in), &sb, &cb);
        const float inv_den = 1.0f / ((float)n_out * (float)n_in);
        const int near_lim = (n_out * n_in) >> 6;
        int num = r0 * n_in - c * n_out;
        for (int r = r0; r < r1; ++r, num += n_in) {
            float v;
            if (num == 0) {
                v = (float)n_out;
            } else {
                const float2 q = rsc[r - r0];
                const float ct = cot_pi_diff(num, inv_den, q.x, q.y, sb, cb, abs(num) < near_lim);
                v = ((r & 1) ? S : -S) * ct;
            }
            M[(size_t)r * ld + c] = __float2bfloat16_rn(v);
        }
    } else if (extra && c == n_in) {
        for (int r = r0; r < r1; ++r) M[(size_t)r * ld + c] = __float2bfloat16_rn((r & 1) ? 1.0f : -1.0f);
    }
}

// One launch for the three inputs of the products: the conversion (bound by
// HBM) and the two maps (bound by arithmetic) share the SMs.
__global__ void __launch_bounds__(256) k_rsg_prep(PrepArgs a)
{
    __shared__ float sh[264];
    int b = blockIdx.x;
    if (b < a.n_conv) {
        prep_convert(a, b % a.cb, b / a.cb, sh);
        return;
    }
    b -= a.n_conv;
    if (b < a.n_wmap) {
        prep_map(a.Wm, a.ldw, a.nw, a.w, 0, b % a.cb, b / a.cb, sh);
        return;
    }
    b -= a.n_wmap;
    prep_map(a.Km, a.ldk, a.nh, a.h, 1, b % a.kcb, b / a.kcb, sh);
}

// uc[j] = (u[j], cos(pi j nw / w), sin(pi j / w), cos(pi j / w)); bias[x] =
// c w h for x < nw
__global__ void __launch_bounds__(256) k_rsg_u(const float* __restrict__ img, long long ip,
                                               const float* __restrict__ part, int w, int h, int nw,
                                               float4* __restrict__ uc, float* __restrict__ bias)
{
    __shared__ float red[8];
    const float c = block_centre(img, ip, w, h, red);
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= w) return;
    if (j < nw) bias[j] = c * (float)w * (float)h;
    float s = 0.0f;
    for (int r = 0; r < kRsgChunks; ++r) s += part[(size_t)r * w + j];
    float sb, cb;
    sincospif(ratio_arg(j, w), &sb, &cb);
    uc[j] = make_float4(s, cospif(ratio_arg(j * nw, w)), sb, cb);
}

// v[x] = sum_j Iw[x][j] u[j] into column h of T (BF16), kRsgVx values of x
// per block (each u[j] read once for all of them).
__global__ void __launch_bounds__(256) k_rsg_v(const float4* __restrict__ uc, int w, int nw,
                                               __nv_bfloat16* __restrict__ T, long long ldt, int h)
{
    __shared__ float red[kRsgVx][8];
    const int x0 = blockIdx.x * kRsgVx;
    const float inv_den = 1.0f / ((float)nw * (float)w);
    const int near_lim = (nw * w) >> 6;
    float sa[kRsgVx], ca[kRsgVx], par[kRsgVx], acc[kRsgVx];
#pragma unroll
    for (int v = 0; v < kRsgVx; ++v) {
        const int x = min(x0 + v, nw - 1);
        sincospif(ratio_arg(x, nw), &sa[v], &ca[v]);
        par[v] = (x & 1) ? -1.0f : 1.0f;
        acc[v] = 0.0f;
    }
    for (int j = threadIdx.x; j < w; j += 256) {
        const float4 q = uc[j];
#pragma unroll
        for (int v = 0; v < kRsgVx; ++v) {
            const int num = (x0 + v) * w - j * nw;
            if (num == 0) continue;
            const float ct = cot_pi_diff(num, inv_den, sa[v], ca[v], q.z, q.w, abs(num) < near_lim);
            acc[v] = fmaf((1.0f - par[v] * q.y) * ct, q.x, acc[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < kRsgVx; ++v) {
        float s = acc[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x < kRsgVx && x0 + threadIdx.x < nw) {
        float s = 0.0f;
        for (int k = 0; k < 8; ++k) s += red[threadIdx.x][k];
        T[(size_t)(x0 + threadIdx.x) * ldt + h] = __float2bfloat16_rn(s);
    }
}

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

}  // namespace

bool rescale_gemm_supported(int w, int h, int nw, int nh)
{
    return w >= 2 && h >= 2 && w <= kRescaleGemmMax && h <= kRescaleGemmMax && nw >= 2 && nh >= 2 && nw <= w &&
           nh <= h;
}

RescaleGemmLayout rescale_gemm_layout(int w, int h, int nw, int nh)
{
    RescaleGemmLayout L;
    L.ldw = round_up(w, 64);
    L.ldk = round_up(h + 1, 64);
    // BF16 areas, each starting on a 256-byte boundary
    L.off_x = 0;
    L.off_w = L.off_x + round_up((long long)h * L.ldw, 128);
    L.off_k = L.off_w + round_up((long long)nw * L.ldw, 128);
    L.off_t = L.off_k + round_up((long long)nh * L.ldk, 128);
    L.bf16_elems = L.off_t + round_up((long long)nw * L.ldk, 128);
    // FP32 area: kRsgChunks x w partial sums, w float4, nw biases
    L.off_uc = round_up((long long)kRsgChunks * w, 64);
    L.off_bias = L.off_uc + 4 * (long long)w;
    L.f32_elems = L.off_bias + round_up(nw, 64);
    return L;
}

cudaError_t launch_rescale_gemm(const float* img, long long pitch, int w, int h, int nw, int nh,
                                __nv_bfloat16* bf, float* f32, int* err, float* out, cudaStream_t st)
{
    if (!rescale_gemm_supported(w, h, nw, nh) || !img || !bf || !f32 || !err || !out || pitch < w)
        return cudaErrorInvalidValue;
    const RescaleGemmLayout L = rescale_gemm_layout(w, h, nw, nh);
    __nv_bfloat16* X = bf + L.off_x;
    __nv_bfloat16* Wm = bf + L.off_w;
    __nv_bfloat16* Km = bf + L.off_k;
    __nv_bfloat16* Tt = bf + L.off_t;
    float* part = f32;
    float4* uc = reinterpret_cast<float4*>(f32 + L.off_uc);
    float* bias = f32 + L.off_bias;
    PrepArgs a;
    a.img = img;
    a.ip = pitch;
    a.w = w;
    a.h = h;
    a.nw = nw;
    a.nh = nh;
    a.X = X;
    a.Wm = Wm;
    a.Km = Km;
    a.ldw = L.ldw;
    a.ldk = L.ldk;
    a.part = part;
    a.cb = (w + 255) / 256;
    a.kcb = (h + 1 + 255) / 256;
    a.n_conv = a.cb * kRsgChunks;
    a.n_wmap = a.cb * ((nw + kRsgRowsPerBlock - 1) / kRsgRowsPerBlock);
    const int n_kmap = a.kcb * ((nh + kRsgRowsPerBlock - 1) / kRsgRowsPerBlock);
    k_rsg_prep<<<a.n_conv + a.n_wmap + n_kmap, 256, 0, st>>>(a);
    k_rsg_u<<<a.cb, 256, 0, st>>>(img, pitch, part, w, h, nw, uc, bias);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // T^T = (X Rw^T)^T: the product's transposed BF16 output, columns 0 .. h-1
    GemmArgs g1;
    g1.M = h;
    g1.N = nw;
    g1.K = w;
    g1.Dt = Tt;
    g1.ldt = L.ldk;
    g1.err = err;
    if ((e = launch_umma_gemm_persistent(X, L.ldw, Wm, L.ldw, g1, 256, 4, 0, st)) != cudaSuccess) return e;
    // column h of T^T: the rank-one term's right factor
    k_rsg_v<<<(nw + kRsgVx - 1) / kRsgVx, 256, 0, st>>>(uc, w, nw, Tt, L.ldk, h);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // out = [Rh | -a] [T^T | v]^T + c w h
    GemmArgs g2;
    g2.M = nh;
    g2.N = nw;
    g2.K = h + 1;
    g2.D = out;
    g2.ldd = nw;
    g2.bias = bias;
    g2.err = err;
    return launch_umma_gemm_persistent(Km, L.ldk, Tt, L.ldk, g2, 256, 4, 0, st);
}

}  // namespace gcf
