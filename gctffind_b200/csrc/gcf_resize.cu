// gcf_resize.cu -- the Fourier-crop rescale of CRescaleImage::DoIt
// (FindCTF/CRescaleImage.cpp:76-99, Util/GFtResize2D.cu:124-143) without a
// 2D FFT library: the R2C of the raw w x h frame, the crop to
// (nw/2 + 1) x nh and the C2R of nw x nh, as three passes of one-dimensional
// line transforms in shared memory.
//
//   pass A (rows)    : each raw row (real, length w) -> its first nw/2 + 1
//                      frequencies, through a complex transform of length
//                      w/2 on the packed (even, odd) samples;
//   pass B (columns) : groups of 4 adjacent frequency columns; per column the
//                      forward transform of length h, the crop to the nh
//                      kept frequencies (0 .. nh/2 and h - nh/2 + 1 .. h - 1,
//                      GFtResize2D's mGTruncate order) and the inverse
//                      transform of length nh;
//   pass C (rows)    : each row of nw/2 + 1 frequencies -> nw real samples,
//                      through a complex inverse transform of length nw/2.
//
// A line of length n is transformed by one CTA: directly when n is a power
// of two, otherwise by Bluestein's chirp-z convolution (the DFT as a
// circular convolution with the chirp exp(-i pi j^2 / n), evaluated by two
// power-of-two FFTs of length M >= 2n - 1).  The power-of-two FFTs are
// Stockham passes (one of radix 2, 4 or 8, then radix 16) over a padded
// shared-memory line, each thread holding its butterfly groups in registers.
// Twiddles, chirps and the chirp filter's spectrum are tables computed in
// double precision on the host, once per length.
//
// Conventions of the library transforms this replaces: all transforms are
// unnormalised (the output is nw * nh times the mean-preserving resample),
// and the C2R of a row uses only the real parts of its DC and Nyquist terms
// (which the crop leaves complex).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "gcf_internal.h"

namespace gcf {

namespace {

// Threads of a line CTA: 256 (two CTAs per SM) when the kernel's FFTs are
// at most 4096 long, 512 (one per SM) with 8192-point FFTs, so an in-place
// pass holds 16 values per thread (256 threads at 8192 points, 32 values
// each, measured slower).
template <int MMAX>
struct LineThreads {
    static constexpr int T = MMAX > 4096 ? 512 : 256;
};
constexpr int kColGroup = 1; // frequency columns per pass-B CTA
// Twiddles of every FFT length M <= 8192 from two small tables in shared
// memory: exp(-2 pi i q / 8192) = hi[q >> 7] * lo[q & 127], lo[t] =
// exp(-2 pi i t / 8192) (t < 128), hi[u] = exp(-2 pi i u / 64) (u < 64);
// an index q of length M is q * (8192 / M) of length 8192.
constexpr int kTwLo = 128, kTwHi = 64, kTwN = kTwLo + kTwHi;

// exp(-2 pi i k / 32), k < 16: the twiddles of the in-register DFTs
__constant__ float2 c_rs_w32[16];

__device__ __forceinline__ int lpad(int p) { return p + (p >> 4); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 addf2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 subf2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// In-register forward DFT of R points, natural order in and out (radix-2
// decimation in time, recursively).
template <int R>
__device__ __forceinline__ void dft_reg(float2 (&v)[R])
{
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = addf2(a, b);
        v[1] = subf2(a, b);
    } else {
        float2 e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i) {
            e[i] = v[2 * i];
            o[i] = v[2 * i + 1];
        }
        dft_reg<R / 2>(e);
        dft_reg<R / 2>(o);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            const float2 t = k == 0 ? o[0] : cmulf(o[k], c_rs_w32[k * (32 / R)]);
            v[k] = addf2(e[k], t);
            v[k + R / 2] = subf2(e[k], t);
        }
    }
}

// One Stockham pass of radix R over the padded line buf of length M (a
// power of two), Ns = product of the earlier passes' radices.  Butterfly
// group j reads elements j + r M/R, applies the twiddles
// exp(-2 pi i r (j mod Ns) / (Ns R)), transforms, and writes to
// (j - j mod Ns) R + j mod Ns + r Ns.  Thread t takes groups t + g T,
// g < G (all of them read before any is written: the pass is in place).
template <int T, int R, int G, bool TW>
__device__ __forceinline__ void stockham_pass(float2* buf, int M, int Ns, const float2* stw, int sh)
{
    const int groups = M / R;
    float2 v[G][R];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int j = threadIdx.x + g * T;
        if (j < groups) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[g][r] = buf[lpad(j + r * groups)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int j = threadIdx.x + g * T;
        if (j < groups) {
            const int k = j & (Ns - 1);
            if constexpr (TW) {
                // w_r = exp(-2 pi i r q / 8192), q = k * step: w_1, w_2, w_4 and
                // w_8 from the tables, every other w_r the product of at most
                // four of them (a few float roundings, like the table pair)
                static_assert(R == 16, "twiddled passes are radix 16");
                const int q = k * ((M / (Ns * R)) << sh);   // in units of 2 pi / 8192
                float2 wr[16];
#pragma unroll
                for (int b = 1; b < 16; b <<= 1) {
                    const int qb = b * q;
                    wr[b] = cmulf(stw[kTwLo + (qb >> 7)], stw[qb & (kTwLo - 1)]);
                }
                wr[3] = cmulf(wr[2], wr[1]);
                wr[5] = cmulf(wr[4], wr[1]);
                wr[6] = cmulf(wr[4], wr[2]);
                wr[7] = cmulf(wr[6], wr[1]);
                wr[9] = cmulf(wr[8], wr[1]);
                wr[10] = cmulf(wr[8], wr[2]);
                wr[11] = cmulf(wr[10], wr[1]);
                wr[12] = cmulf(wr[8], wr[4]);
                wr[13] = cmulf(wr[12], wr[1]);
                wr[14] = cmulf(wr[12], wr[2]);
                wr[15] = cmulf(wr[14], wr[1]);
#pragma unroll
                for (int r = 1; r < R; ++r) v[g][r] = cmulf(v[g][r], wr[r]);
            }
            dft_reg<R>(v[g]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[lpad(base + r * Ns)] = v[g][r];
        }
    }
    __syncthreads();
}

// Groups per thread of a first pass of radix r: its largest length is the
// largest r 16^k <= mmax (2 x 16^3 = 8192 gives 4096 groups, 8 per thread
// of 512).
__host__ __device__ constexpr int first_pass_groups(int r, int mmax, int t)
{
    int m = r;
    while (m * 16 <= mmax) m *= 16;
    return (m / r + t - 1) / t;
}

// Forward FFT of the padded line buf (length M, a power of two, 1..MMAX)
// in place; stw: the twiddle tables in shared memory, sh = log2(8192 / M).
// Entered and left synchronised.  Radix plan: the radix left over by the
// 16s (2, 4 or 8) first, where Ns = 1 and no twiddles apply, then radix-16
// passes of at most T groups.  Not inlined: each kernel calls it up to
// four times, and inlined copies spill.
template <int MMAX>
__device__ __noinline__ void line_fft(float2* buf, int M, const float2* stw)
{
    constexpr int T = LineThreads<MMAX>::T, G16 = (MMAX / 16 + T - 1) / T;
    int left = M, sh = 0;
    while (left % 16 == 0) left /= 16;
    while ((M << sh) < 8192) ++sh;
    int Ns = left;
    if (left == 8) stockham_pass<T, 8, first_pass_groups(8, MMAX, T), false>(buf, M, 1, stw, sh);
    else if (left == 4) stockham_pass<T, 4, first_pass_groups(4, MMAX, T), false>(buf, M, 1, stw, sh);
    else if (left == 2) stockham_pass<T, 2, first_pass_groups(2, MMAX, T), false>(buf, M, 1, stw, sh);
    for (; Ns < M; Ns *= 16) stockham_pass<T, 16, G16, true>(buf, M, Ns, stw, sh);
}

// The twiddle tables into shared memory (at kernel start).
template <int T>
__device__ __forceinline__ void load_twiddles(float2* stw, const float2* __restrict__ tw2)
{
    for (int i = threadIdx.x; i < kTwN; i += T) stw[i] = tw2[i];
    __syncthreads();
}

// The forward DFT of length L.n of load(i), i < L.n, into buf; read the
// result with line_out.  Entered with buf free, left synchronised.
template <int MMAX, class Load>
__device__ __forceinline__ void line_dft(float2* buf, const ResizeLine& L, const float2* stw, Load load)
{
    if (L.chirp) {
#pragma unroll 4
        for (int i = threadIdx.x; i < L.M; i += LineThreads<MMAX>::T)
            buf[lpad(i)] = i < L.n ? cmulf(load(i), __ldg(L.chirp + i)) : make_float2(0.0f, 0.0f);
        __syncthreads();
        line_fft<MMAX>(buf, L.M, stw);
#pragma unroll 4
        for (int i = threadIdx.x; i < L.M; i += LineThreads<MMAX>::T) buf[lpad(i)] = conjf2(cmulf(buf[lpad(i)], __ldg(L.bf + i)));
        __syncthreads();
        line_fft<MMAX>(buf, L.M, stw);
    } else {
#pragma unroll 4
        for (int i = threadIdx.x; i < L.M; i += LineThreads<MMAX>::T) buf[lpad(i)] = load(i);
        __syncthreads();
        line_fft<MMAX>(buf, L.M, stw);
    }
}

// Output k (< L.n) of the last line_dft.
__device__ __forceinline__ float2 line_out(const float2* buf, const ResizeLine& L, int k)
{
    return L.chirp ? cmulf(conjf2(buf[lpad(k)]), __ldg(L.chirp + k)) : buf[lpad(k)];
}

// A line that may be split (L.split): the DFT of its even samples into ebuf
// (n/2 values), then that of its odd samples into buf; line_out_s combines.
template <int MMAX, class Load>
__device__ __forceinline__ void line_dft_s(float2* buf, float2* ebuf, const ResizeLine& L, const float2* stw,
                                           Load load)
{
    if (!L.split) {
        line_dft<MMAX>(buf, L, stw, load);
        return;
    }
    ResizeLine H = L;
    H.n = L.n / 2;
    line_dft<MMAX>(buf, H, stw, [&](int i) { return load(2 * i); });
    for (int k = threadIdx.x; k < H.n; k += LineThreads<MMAX>::T) ebuf[k] = line_out(buf, H, k);
    __syncthreads();
    line_dft<MMAX>(buf, H, stw, [&](int i) { return load(2 * i + 1); });
}

// Output k (< L.n) of the last line_dft_s: X_k = E_k + t_k O_k and
// X_{k + n/2} = E_k - t_k O_k, t_k = exp(-2 pi i k / n).
__device__ __forceinline__ float2 line_out_s(const float2* buf, const float2* ebuf, const ResizeLine& L, int k)
{
    if (!L.split) return line_out(buf, L, k);
    ResizeLine H = L;
    H.n = L.n / 2;
    const int kk = k < H.n ? k : k - H.n;
    const float2 e = ebuf[kk], o = cmulf(line_out(buf, H, kk), __ldg(L.ts + kk));
    return k < H.n ? addf2(e, o) : subf2(e, o);
}

// Pass A: raw rows (w even) -> T1[y][k], k < K = nw/2 + 1.
template <int MMAX>
__global__ void __launch_bounds__(LineThreads<MMAX>::T, 512 / LineThreads<MMAX>::T) k_resize_rows_fwd(const float* __restrict__ img, int w, int h, int vec,
                                                         ResizeLine La, const float2* __restrict__ tA, int K,
                                                         const float2* __restrict__ tw2, float2* __restrict__ T1)
{
    extern __shared__ float2 rbuf[];
    __shared__ float2 stw[kTwN];
    load_twiddles<LineThreads<MMAX>::T>(stw, tw2);
    float2* ebuf = rbuf + La.M + La.M / 16;   // even-sample DFT of a split line
    const int N = w / 2;
    for (int y = blockIdx.x; y < h; y += gridDim.x) {
        const float* row = img + (size_t)y * w;
        if (vec) {
            const float2* r2 = reinterpret_cast<const float2*>(row);
            line_dft_s<MMAX>(rbuf, ebuf, La, stw, [&](int i) { return __ldg(r2 + i); });
        } else {
            line_dft_s<MMAX>(rbuf, ebuf, La, stw,
                             [&](int i) { return make_float2(__ldg(row + 2 * i), __ldg(row + 2 * i + 1)); });
        }
        // X_k = ((Z_k + conj Z_{N-k}) - i t_k (Z_k - conj Z_{N-k})) / 2, t_k = exp(-2 pi i k / w)
        for (int k = threadIdx.x; k < K; k += LineThreads<MMAX>::T) {
            const float2 zk = line_out_s(rbuf, ebuf, La, k < N ? k : k - N);
            const float2 zn = conjf2(line_out_s(rbuf, ebuf, La, k == 0 ? 0 : N - k));
            const float2 s = addf2(zk, zn), t = cmulf(__ldg(tA + k), subf2(zk, zn));
            T1[(size_t)y * K + k] = make_float2(0.5f * (s.x + t.y), 0.5f * (s.y - t.x));
        }
        __syncthreads();
    }
}

// Pass B: columns of T1 (h rows) -> T2 (nh rows), kColGroup columns per CTA.
template <int MMAX>
__global__ void __launch_bounds__(LineThreads<MMAX>::T, 512 / LineThreads<MMAX>::T) k_resize_cols(const float2* __restrict__ T1, int K, int h, int nh, int hs,
                                                     ResizeLine Lf, ResizeLine Li, const float2* __restrict__ tw2,
                                                     float2* __restrict__ T2)
{
    extern __shared__ float2 cbuf[];
    __shared__ float2 stw[kTwN];
    load_twiddles<LineThreads<MMAX>::T>(stw, tw2);
    float2* stash = cbuf;                          // [kColGroup][hs]
    float2* buf = cbuf + (size_t)kColGroup * hs;   // the line
    const int mb = max(Lf.M, Li.M);
    float2* ebuf = buf + mb + mb / 16;             // even-sample DFT of a split line
    for (int k0 = blockIdx.x * kColGroup; k0 < K; k0 += gridDim.x * kColGroup) {
        const int cb = min(kColGroup, K - k0);
#pragma unroll 8
        for (int i = threadIdx.x; i < h * kColGroup; i += LineThreads<MMAX>::T) {
            const int y = i / kColGroup, c = i - y * kColGroup;
            if (c < cb) stash[c * hs + y] = T1[(size_t)y * K + k0 + c];
        }
        __syncthreads();
        for (int c = 0; c < cb; ++c) {
            float2* col = stash + c * hs;
            line_dft_s<MMAX>(buf, ebuf, Lf, stw, [&](int i) { return col[i]; });
            // the kept frequencies, conjugated for the inverse transform
            for (int m = threadIdx.x; m < nh; m += LineThreads<MMAX>::T)
                col[m] = conjf2(line_out_s(buf, ebuf, Lf, m <= nh / 2 ? m : m - nh + h));
            __syncthreads();
            line_dft_s<MMAX>(buf, ebuf, Li, stw, [&](int i) { return col[i]; });
            for (int m = threadIdx.x; m < nh; m += LineThreads<MMAX>::T)
                col[m] = conjf2(line_out_s(buf, ebuf, Li, m));
            __syncthreads();
        }
        for (int i = threadIdx.x; i < nh * kColGroup; i += LineThreads<MMAX>::T) {
            const int y = i / kColGroup, c = i - y * kColGroup;
            if (c < cb) T2[(size_t)y * K + k0 + c] = stash[c * hs + y];
        }
        __syncthreads();
    }
}

// Pass C: rows of T2 (K = nw/2 + 1 frequencies) -> nw real samples.
// z = inverse DFT of Z_k = (Y_k + conj Y_{Nn-k}) + i t_k (Y_k - conj Y_{Nn-k}),
// t_k = exp(2 pi i k / nw); out[2m] = Re z_m, out[2m + 1] = Im z_m.  The
// crop leaves the DC and Nyquist terms of a row complex (the kept columns
// and rows are not Hermitian-symmetric at the new edges); like the library
// C2R of the reference, only their real parts are used.
template <int MMAX>
__global__ void __launch_bounds__(LineThreads<MMAX>::T, 512 / LineThreads<MMAX>::T) k_resize_rows_inv(const float2* __restrict__ T2, int K, int nh, int nw,
                                                         ResizeLine Lc, const float2* __restrict__ tC,
                                                         const float2* __restrict__ tw2, float* __restrict__ out)
{
    extern __shared__ float2 rbuf[];
    __shared__ float2 stw[kTwN];
    load_twiddles<LineThreads<MMAX>::T>(stw, tw2);
    const int Nn = nw / 2;
    float2* ebuf = rbuf + Lc.M + Lc.M / 16;   // even-sample DFT of a split line
    for (int y = blockIdx.x; y < nh; y += gridDim.x) {
        const float2* Y = T2 + (size_t)y * K;
        line_dft_s<MMAX>(rbuf, ebuf, Lc, stw, [&](int k) {
            float2 a = Y[k], b = Y[Nn - k];
            if (k == 0) {   // Y_0 and Y_Nn: real parts only
                a.y = 0.0f;
                b.y = 0.0f;
            }
            const float2 bc = conjf2(b);
            const float2 s = addf2(a, bc), t = cmulf(__ldg(tC + k), subf2(a, bc));
            return make_float2(s.x - t.y, -(s.y + t.x));   // conjugated: the inverse through the forward DFT
        });
        float2* o2 = reinterpret_cast<float2*>(out + (size_t)y * nw);
        for (int m = threadIdx.x; m < Nn; m += LineThreads<MMAX>::T) o2[m] = conjf2(line_out_s(rbuf, ebuf, Lc, m));
        __syncthreads();
    }
}

cudaError_t init_resize_constants()
{
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return cudaSuccess;
    float2 w[16];
    for (int k = 0; k < 16; ++k) {
        const double a = -2.0 * M_PI * k / 32.0;
        double c = std::cos(a), s = std::sin(a);
        if (std::fabs(c) < 1e-15) c = 0.0;
        w[k] = make_float2((float)c, (float)s);
    }
    e = cudaMemcpyToSymbol(c_rs_w32, w, sizeof(w));
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

size_t line_smem(int M) { return (size_t)(M + M / 16) * sizeof(float2); }

// One line kernel over `lines` lines: at most as many CTAs as can be
// resident at once (each loops over its lines).
template <int T, class K, class... Args>
cudaError_t launch_line(K kernel, int lines, size_t smem, int sms, cudaStream_t st, Args... args)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, T, smem)) != cudaSuccess) return e;
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    const int grid = std::max(1, std::min(lines, sms * per_sm));
    kernel<<<grid, T, smem, st>>>(args...);
    return cudaGetLastError();
}

// ---- tables (host, double precision), cached per device and length ----
// The twiddles of the FFT of length M, the chirp of a line of length n and
// its filter spectrum stay allocated for the life of the process (a graph
// captured with them keeps their addresses): about 100 KB per line length,
// at most kResizeMaxLine lengths.
// Forward FFT in place of n = 2^k complex values held as interleaved
// (re, im) doubles (explicit arithmetic: std::complex products check for
// NaN and run several times slower).
void fft_host(std::vector<double>& a)
{
    const size_t n = a.size() / 2;
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(a[2 * i], a[2 * j]);
            std::swap(a[2 * i + 1], a[2 * j + 1]);
        }
    }
    std::vector<double> wr(n / 2), wi(n / 2);   // exp(-2 pi i k / n)
    for (size_t k = 0; k < n / 2; ++k) {
        wr[k] = std::cos(-2.0 * M_PI * (double)k / (double)n);
        wi[k] = std::sin(-2.0 * M_PI * (double)k / (double)n);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2, stride = n / len;
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < half; ++k) {
                double* u = &a[2 * (i + k)];
                double* x = &a[2 * (i + k + half)];
                const double tr = wr[k * stride], ti = wi[k * stride];
                const double vr = x[0] * tr - x[1] * ti, vi = x[0] * ti + x[1] * tr;
                x[0] = u[0] - vr;
                x[1] = u[1] - vi;
                u[0] += vr;
                u[1] += vi;
            }
    }
}

struct TabCache {
    std::mutex mu;
    std::map<std::pair<int, int>, ResizeLine> lines;    // (device, n)
    std::map<std::tuple<int, int, int, int>, float2*> tw;   // (device, length, sign, count)
};
TabCache& tabs()
{
    static TabCache c;
    return c;
}

cudaError_t upload(const std::vector<float2>& h, float2** d)
{
    cudaError_t e = cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(float2));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(*d, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(*d);
        *d = nullptr;
    }
    return e;
}

// exp(sign 2 pi i k / len), k < count (held in the cache's lock)
cudaError_t twiddles_locked(TabCache& c, int dev, int len, int sign, int count, float2** out)
{
    auto key = std::make_tuple(dev, len, sign, count);
    auto it = c.tw.find(key);
    if (it != c.tw.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    std::vector<float2> h(count);
    for (int k = 0; k < count; ++k) {
        const double a = sign * 2.0 * M_PI * (double)k / (double)len;
        h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    float2* d = nullptr;
    cudaError_t e = upload(h, &d);
    if (e != cudaSuccess) return e;
    c.tw[key] = d;
    *out = d;
    return cudaSuccess;
}

}  // namespace

bool resize_line_ok(int n) { return n >= 1 && n <= kResizeMaxLine; }

namespace {
// The tables of a line of length n transformed whole (held in the lock).
cudaError_t whole_line_locked(TabCache& c, int dev, int n, ResizeLine* out)
{
    auto it = c.lines.find({dev, n});
    if (it != c.lines.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaError_t e = cudaSuccess;
    ResizeLine L{};
    L.n = n;
    const bool pow2 = (n & (n - 1)) == 0;
    L.M = pow2 ? n : 1;
    if (!pow2)
        while (L.M < 2 * n - 1) L.M <<= 1;
    if (!pow2) {
        // chirp c_j = exp(-i pi j^2 / n) (j^2 reduced mod 2n exactly), and
        // the spectrum of b (b_j = conj c_j for |j| < n, circular) over M
        std::vector<double> cr(n), ci(n), b(2 * (size_t)L.M, 0.0);
        for (int j = 0; j < n; ++j) {
            const long long q = ((long long)j * j) % (2LL * n);
            const double a = -M_PI * (double)q / (double)n;
            cr[j] = std::cos(a);
            ci[j] = std::sin(a);
        }
        b[0] = cr[0];
        b[1] = -ci[0];
        for (int j = 1; j < n; ++j) {
            b[2 * j] = b[2 * (L.M - j)] = cr[j];
            b[2 * j + 1] = b[2 * (L.M - j) + 1] = -ci[j];
        }
        fft_host(b);
        std::vector<float2> hc(n), hb(L.M);
        for (int j = 0; j < n; ++j) hc[j] = make_float2((float)cr[j], (float)ci[j]);
        for (int k = 0; k < L.M; ++k) hb[k] = make_float2((float)(b[2 * k] / L.M), (float)(b[2 * k + 1] / L.M));
        float2 *dc = nullptr, *db = nullptr;
        if ((e = upload(hc, &dc)) != cudaSuccess) return e;
        if ((e = upload(hb, &db)) != cudaSuccess) {
            cudaFree(dc);
            return e;
        }
        L.chirp = dc;
        L.bf = db;
    }
    c.lines[{dev, n}] = L;
    *out = L;
    return cudaSuccess;
}
}  // namespace

// An even length above 2048 that is not a power of two (whose Bluestein
// FFT would be 8192 long) is split: the DFTs of its even and odd samples
// (length n/2, FFTs of at most 4096) and one radix-2 step with the twiddles
// exp(-2 pi i k / n), k < n/2.
cudaError_t resize_line(int n, ResizeLine* out)
{
    if (!resize_line_ok(n)) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    TabCache& c = tabs();
    std::lock_guard<std::mutex> lock(c.mu);
    const bool pow2 = (n & (n - 1)) == 0;
    if (n % 2 == 0 && n > 2048 && !pow2) {
        ResizeLine H{};
        if ((e = whole_line_locked(c, dev, n / 2, &H)) != cudaSuccess) return e;
        float2* ts = nullptr;
        if ((e = twiddles_locked(c, dev, n, -1, n / 2, &ts)) != cudaSuccess) return e;
        H.n = n;
        H.split = 1;
        H.ts = ts;
        *out = H;
        return cudaSuccess;
    }
    return whole_line_locked(c, dev, n, out);
}

// lo[t] = exp(-2 pi i t / 8192), t < 128, then hi[u] = exp(-2 pi i u / 64), u < 64
cudaError_t resize_fft_twiddles(const float2** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    TabCache& c = tabs();
    std::lock_guard<std::mutex> lock(c.mu);
    auto key = std::make_tuple(dev, 8192, 0, kTwN);
    auto it = c.tw.find(key);
    if (it != c.tw.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    std::vector<float2> h(kTwN);
    for (int t = 0; t < kTwLo; ++t) {
        const double a = -2.0 * M_PI * t / 8192.0;
        h[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    for (int u = 0; u < kTwHi; ++u) {
        const double a = -2.0 * M_PI * u / 64.0;
        double cr = std::cos(a), si = std::sin(a);
        if (std::fabs(cr) < 1e-15) cr = 0.0;
        if (std::fabs(si) < 1e-15) si = 0.0;
        h[kTwLo + u] = make_float2((float)cr, (float)si);
    }
    float2* d = nullptr;
    if ((e = upload(h, &d)) != cudaSuccess) return e;
    c.tw[key] = d;
    *out = d;
    return cudaSuccess;
}

cudaError_t resize_twiddles(int len, int sign, int count, const float2** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    TabCache& c = tabs();
    std::lock_guard<std::mutex> lock(c.mu);
    float2* p = nullptr;
    e = twiddles_locked(c, dev, len, sign, count, &p);
    *out = p;
    return e;
}

size_t resize_cols_smem(int h, int m_max, int e_max)
{
    const int hs = h + ((h & 1) ? 0 : 1);
    return (size_t)kColGroup * hs * sizeof(float2) + line_smem(m_max) + (size_t)e_max * sizeof(float2);
}

cudaError_t launch_resize(const float* img, int w, int h, int nw, int nh, const ResizeLine& rowA,
                          const float2* tA, const ResizeLine& colF, const ResizeLine& colI, const ResizeLine& rowC,
                          const float2* tC, float2* T1, float2* T2, float* out, cudaStream_t st)
{
    cudaError_t e = init_resize_constants();
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int K = nw / 2 + 1;
    const int vec = ((reinterpret_cast<uintptr_t>(img) & 7) == 0) ? 1 : 0;
    auto ehalf = [](const ResizeLine& L) { return L.split ? L.n / 2 : 0; };
    const size_t sa = line_smem(rowA.M) + ehalf(rowA) * sizeof(float2);
    const size_t sc = line_smem(rowC.M) + ehalf(rowC) * sizeof(float2);
    const size_t sb = resize_cols_smem(h, std::max(colF.M, colI.M), std::max(ehalf(colF), ehalf(colI)));
    const int hs = h + ((h & 1) ? 0 : 1);
    const float2* tw2 = nullptr;
    if ((e = resize_fft_twiddles(&tw2)) != cudaSuccess) return e;
    const int ngroups = (K + kColGroup - 1) / kColGroup;
    if (rowA.M <= 4096) e = launch_line<256>(k_resize_rows_fwd<4096>, h, sa, sms, st, img, w, h, vec, rowA, tA, K, tw2, T1);
    else e = launch_line<512>(k_resize_rows_fwd<8192>, h, sa, sms, st, img, w, h, vec, rowA, tA, K, tw2, T1);
    if (e != cudaSuccess) return e;
    if (std::max(colF.M, colI.M) <= 4096)
        e = launch_line<256>(k_resize_cols<4096>, ngroups, sb, sms, st, T1, K, h, nh, hs, colF, colI, tw2, T2);
    else e = launch_line<512>(k_resize_cols<8192>, ngroups, sb, sms, st, T1, K, h, nh, hs, colF, colI, tw2, T2);
    if (e != cudaSuccess) return e;
    if (rowC.M <= 4096) e = launch_line<256>(k_resize_rows_inv<4096>, nh, sc, sms, st, T2, K, nh, nw, rowC, tC, tw2, out);
    else e = launch_line<512>(k_resize_rows_inv<8192>, nh, sc, sms, st, T2, K, nh, nw, rowC, tC, tw2, out);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace gcf
