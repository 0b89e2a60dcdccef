// gcf_fused.cu -- fused tile-spectrum kernel for 512 x 512 tiles
// (CGenAvgSpectrum::DoIt + GCalcMoment2D + GNormalize2D + GRoundEdge +
//  GCalcSpectrum::DoPad + GAddImages, FindCTF/CGenAvgSpectrum.cpp:77-139).
//
// One thread-block cluster of 8 CTAs owns one tile at a time; the tile never
// leaves the chip:
//   load    CTA r reads tile rows [64r, 64r+64) (coalesced float4 when the
//           tile start is 16-byte aligned) into its shared memory and sums
//           them; the 8 partial sums are combined over distributed shared
//           memory (DSMEM), so every CTA holds the same tile mean;
//   rows    each warp transforms two rows at once ((x - mean) * taper as the
//           real and imaginary parts of one 512-point complex FFT held in
//           registers, 16 values per lane, radix-16 x radix-32 with one
//           shared-memory transpose) and splits the result into the two
//           257-bin half spectra, written back in place;
//   columns each warp gathers one frequency column (512 rows) straight from
//           the 8 CTAs' shared memory over DSMEM and transforms it; the
//           real kx = 0 and kx = 256 columns share one complex FFT;
//   |F|     amplitudes (DC moved to row 256) accumulate in registers across
//           all tiles of a work item and are written once.
// Work items are (image, tile range) pairs; their partial spectra are summed
// in item order by k_item_reduce, so the result is deterministic.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "gcf_internal.h"

namespace cg = cooperative_groups;

namespace gcf {

namespace {

constexpr int FT = 512;          // tile edge
constexpr int FCX = FT / 2 + 1;  // 257 half-spectrum columns
constexpr int FCL = 8;           // CTAs per cluster
constexpr int FROWS = FT / FCL;  // 64 rows per CTA
constexpr int FTHR = 256;        // threads per CTA
constexpr int FWARPS = FTHR / 32;
constexpr int FNR = 32 / FWARPS;  // column rounds per tile (32 columns per CTA)
constexpr int FRS = FCX;         // row stride of the row buffer, float2 units
constexpr int FSCR = 16 * 33;    // per-warp scratch, float2 units

constexpr size_t kRowBytes = (size_t)FROWS * FRS * sizeof(float2);     // 131584
constexpr size_t kScrBytes = (size_t)FWARPS * FSCR * sizeof(float2);   // 67584
constexpr size_t kTwBytes = (size_t)FT * sizeof(float2);               // 4096
constexpr size_t kAccNBytes = (size_t)FT * sizeof(float);              // 2048
constexpr size_t kPartBytes = 32 * sizeof(double);   // 16 warp sums + CTA sum
constexpr size_t kFusedSmem = kRowBytes + kScrBytes + kTwBytes + kAccNBytes + kPartBytes;

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Forward 4-point DFT in place (W4 = -i).
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3)
{
    float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = make_float2(d02.x + d13.y, d02.y - d13.x);   // d02 - i d13
    a3 = make_float2(d02.x - d13.y, d02.y + d13.x);   // d02 + i d13
}

// exp(-2 pi i m / 16) for the compile-time products m = n2 * k1 <= 9
__device__ __forceinline__ float2 w16(int m)
{
    constexpr float C1 = 0.92387953251128674f, C2 = 0.70710678118654752f, C3 = 0.38268343236508977f;
    switch (m) {
    case 0: return make_float2(1.0f, 0.0f);
    case 1: return make_float2(C1, -C3);
    case 2: return make_float2(C2, -C2);
    case 3: return make_float2(C3, -C1);
    case 4: return make_float2(0.0f, -1.0f);
    case 6: return make_float2(-C2, -C2);
    default: return make_float2(-C1, C3);   // m = 9
    }
}

// Position of output k of dft16 in its register array.
__host__ __device__ constexpr int P16(int k) { return (k & 3) * 4 + (k >> 2); }

// Forward 16-point DFT in registers, natural-order input, output k in
// v[P16(k)] (radix-4 x radix-4: n = 4 n1 + n2, k = k1 + 4 k2).
__device__ __forceinline__ void dft16(float2 (&v)[16])
{
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    // v[4 k1 + n2] now holds stage-A output (k1, n2); twiddle W16^(n2 k1)
#pragma unroll
    for (int k1 = 1; k1 < 4; ++k1)
#pragma unroll
        for (int n2 = 1; n2 < 4; ++n2) v[4 * k1 + n2] = cmul(v[4 * k1 + n2], w16(n2 * k1));
    // stage C: DFT over n2 for each k1 -> X[k1 + 4 k2]
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4(v[4 * k1 + 0], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // X[k] now sits in v[P16(k)]: the digit reversal is left to the caller's
    // compile-time indexing instead of register moves.
}

// 512-point forward FFT held by one warp.  In: lane l holds x[32 j + l] in
// v[j].  Out: lane 2m+p holds X[m + 16 k + 256 p] in v[P16(k)].  scr: 528 float2
// of warp-private shared memory; tw: exp(-2 pi i t / 512), t < 512.
__device__ __forceinline__ void fft512_warp(float2 (&v)[16], float2* scr, const float2* tw, int lane)
{
    dft16(v);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) v[P16(k1)] = cmul(v[P16(k1)], tw[(lane * k1) & (FT - 1)]);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) scr[k1 * 33 + lane] = v[P16(k1)];
    __syncwarp();
    const int m = lane >> 1, p = lane & 1;
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = scr[m * 33 + 2 * q + p];
    dft16(v);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float2 mine = v[P16(k)];
        float2 o;
        o.x = __shfl_xor_sync(0xffffffffu, mine.x, 1);
        o.y = __shfl_xor_sync(0xffffffffu, mine.y, 1);
        float2 e0 = p ? o : mine;
        float2 e1 = p ? mine : o;
        float2 t = cmul(tw[16 * k], e1);
        v[P16(k)] = p ? csub(e0, t) : cadd(e0, t);
    }
    __syncwarp();
}

struct FusedTab {
    const float* img;
    int pitch;
    int ntx;
    int offx, offy, stride;
    int vec4;   // 1 when every tile row start is 16-byte aligned
};

__global__ void __cluster_dims__(FCL, 1, 1) __launch_bounds__(FTHR, 1)
k_fused_spectrum(const FusedTab* __restrict__ imgs, const int4* __restrict__ items, int nitems,
                 const float* __restrict__ taper, const float2* __restrict__ twg,
                 float* __restrict__ partial)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float2* rowbuf = reinterpret_cast<float2*>(smem);
    float2* scr_all = reinterpret_cast<float2*>(smem + kRowBytes);
    float2* tw = reinterpret_cast<float2*>(smem + kRowBytes + kScrBytes);
    float* accN = reinterpret_cast<float*>(smem + kRowBytes + kScrBytes + kTwBytes);
    double* part = reinterpret_cast<double*>(smem + kRowBytes + kScrBytes + kTwBytes + kAccNBytes);

    cg::cluster_group cluster = cg::this_cluster();
    const int r = (int)cluster.block_rank();
    const int cid = blockIdx.x / FCL;
    const int ncl = gridDim.x / FCL;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = lane >> 1, p = lane & 1;
    float2* scr = scr_all + warp * FSCR;
    float* rowf = reinterpret_cast<float*>(rowbuf);

    for (int i = tid; i < FT; i += FTHR) tw[i] = twg[i];
    __syncthreads();

    for (int it = cid; it < nitems; it += ncl) {
        const int4 item = items[it];   // (image, first tile, end tile, item index)
        const FusedTab im = imgs[item.x];
        float acc[FNR][16];
#pragma unroll
        for (int a = 0; a < FNR; ++a)
#pragma unroll
            for (int k = 0; k < 16; ++k) acc[a][k] = 0.0f;
        for (int i = tid; i < FT; i += FTHR) accN[i] = 0.0f;

        for (int t = item.y; t < item.z; ++t) {
            const int tx = t % im.ntx, ty = t / im.ntx;
            const float* src = im.img + (size_t)(im.offy + ty * im.stride + r * FROWS) * im.pitch +
                               im.offx + tx * im.stride;
            cluster.sync();   // peers are done with this CTA's row buffer
            // ---- load 64 rows, partial sum -------------------------------------
            double s = 0.0;
            if (im.vec4) {
#pragma unroll 4
                for (int i = 0; i < FROWS * FT / 4 / FTHR; ++i) {
                    int q = tid + i * FTHR;
                    int row = q >> 7, c4 = (q & 127) * 4;
                    float4 x = __ldg(reinterpret_cast<const float4*>(src + (size_t)row * im.pitch + c4));
                    float* d = rowf + row * (2 * FRS) + c4;
                    reinterpret_cast<float2*>(d)[0] = make_float2(x.x, x.y);
                    reinterpret_cast<float2*>(d)[1] = make_float2(x.z, x.w);
                    s += (double)x.x + (double)x.y + (double)x.z + (double)x.w;
                }
            } else {
                for (int i = 0; i < FROWS * FT / FTHR; ++i) {
                    int q = tid + i * FTHR;
                    int row = q >> 9, c = q & (FT - 1);
                    float x = __ldg(src + (size_t)row * im.pitch + c);
                    rowf[row * (2 * FRS) + c] = x;
                    s += (double)x;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) part[warp] = s;
            __syncthreads();
            if (tid == 0) {
                double b = 0.0;
                for (int w = 0; w < FWARPS; ++w) b += part[w];
                part[FWARPS] = b;   // CTA sum
            }
            cluster.sync();   // CTA sums visible cluster-wide
            double tot = 0.0;
#pragma unroll
            for (int q = 0; q < FCL; ++q) tot += *cluster.map_shared_rank(part + FWARPS, q);
            const float mean = (float)(tot / ((double)FT * FT));

            // ---- row transforms: two rows per FFT -------------------------------
#pragma unroll 1
            for (int pp = warp; pp < FROWS / 2; pp += FWARPS) {
                const int y0 = 2 * pp, Y0 = r * FROWS + y0;
                float2 v[16];
                const float* ta = taper + (size_t)Y0 * FT;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    int X = 32 * j + lane;
                    float a = (rowf[y0 * (2 * FRS) + X] - mean) * __ldg(ta + X);
                    float b = (rowf[(y0 + 1) * (2 * FRS) + X] - mean) * __ldg(ta + FT + X);
                    v[j] = make_float2(a, b);
                }
                fft512_warp(v, scr, tw, lane);
#pragma unroll
                for (int k = 0; k < 16; ++k) scr[m + 16 * k + 256 * p] = v[P16(k)];
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 9; ++i) {
                    int K = lane + 32 * i;
                    if (K <= FT / 2) {
                        float2 zk = scr[K], zn = scr[(FT - K) & (FT - 1)];
                        float2 A = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
                        float2 B = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
                        rowbuf[y0 * FRS + K] = A;
                        rowbuf[(y0 + 1) * FRS + K] = B;
                    }
                }
                __syncwarp();
            }
            cluster.sync();   // every row buffer of the cluster is complete

            // ---- column transforms over DSMEM -----------------------------------
#pragma unroll
            for (int rho = 0; rho < FNR; ++rho) {
                const int c = 32 * r + FWARPS * rho + warp;   // 0 = packed (kx 0, kx 256)
                float2 v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    // rows 32 j + lane live in CTA j / 2 at local row 32 (j & 1) + lane
                    const float2* peer = cluster.map_shared_rank(rowbuf, j >> 1);
                    int lr = 32 * (j & 1) + lane;
                    if (c == 0) {
                        v[j] = make_float2(peer[lr * FRS].x, peer[lr * FRS + FT / 2].x);
                    } else {
                        v[j] = peer[lr * FRS + c];
                    }
                }
                fft512_warp(v, scr, tw, lane);
                if (c != 0) {
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        float2 z = v[P16(k)];
                        acc[rho][k] += sqrtf(z.x * z.x + z.y * z.y);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 16; ++k) scr[m + 16 * k + 256 * p] = v[P16(k)];
                    __syncwarp();
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        int K = m + 16 * k + 256 * p;
                        float2 zk = v[P16(k)], zn = scr[(FT - K) & (FT - 1)];
                        float ax = 0.5f * (zk.x + zn.x), ay = 0.5f * (zk.y - zn.y);
                        float bx = 0.5f * (zk.y + zn.y), by = -0.5f * (zk.x - zn.x);
                        acc[rho][k] += sqrtf(ax * ax + ay * ay);
                        accN[K] += sqrtf(bx * bx + by * by);
                    }
                    __syncwarp();
                }
            }
        }
        // ---- write this item's partial spectrum (DC moved to row 256) -----------
        float* out = partial + (size_t)item.w * FCX * FT;
#pragma unroll
        for (int rho = 0; rho < FNR; ++rho) {
            const int kx = 32 * r + FWARPS * rho + warp;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                int ky = m + 16 * k + 256 * p;
                int yd = (ky + FT / 2) & (FT - 1);
                out[(size_t)yd * FCX + kx] = acc[rho][k];
            }
        }
        __syncthreads();
        if (r == 0 && warp == 0) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                int K = m + 16 * k + 256 * p;
                int yd = (K + FT / 2) & (FT - 1);
                out[(size_t)yd * FCX + FT / 2] = accN[K];
            }
        }
    }
    cluster.sync();   // keep shared memory alive until every peer is done
}

// raw[img] = sum of the img's item partials (in item order) / ntiles.
__global__ void k_item_reduce(const float* __restrict__ partial, const int* __restrict__ first,
                              const float* __restrict__ inv, float* __restrict__ raw)
{
    const int n = FCX * FT;
    int img = blockIdx.y;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = first[img]; k < first[img + 1]; ++k) s += partial[(size_t)k * n + i];
    raw[(size_t)img * n + i] = (float)(s * (double)inv[img]);
}

}  // namespace

int fused_tile_supported(int tile) { return tile == FT ? 1 : 0; }

size_t fused_smem_bytes() { return kFusedSmem; }

// Host launcher.  descs/items/first/inv are device arrays prepared by the caller.
cudaError_t launch_fused(const void* descs, const int4* items, int nitems, const int* first,
                         const float* inv, int nimg, const float* taper, const float2* tw,
                         float* partial, float* raw, int nclusters, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_fused_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFusedSmem);
    if (e != cudaSuccess) return e;
    if (nclusters < 1) nclusters = 1;
    k_fused_spectrum<<<nclusters * FCL, FTHR, kFusedSmem, st>>>(
        reinterpret_cast<const FusedTab*>(descs), items, nitems, taper, tw, partial);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 g((FCX * FT + 255) / 256, nimg);
    k_item_reduce<<<g, 256, 0, st>>>(partial, first, inv, raw);
    return cudaGetLastError();
}

cudaError_t fused_max_clusters(int* n)
{
    cudaError_t e = cudaFuncSetAttribute(k_fused_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFusedSmem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(FCL * 64, 1, 1);
    cfg.blockDim = dim3(FTHR, 1, 1);
    cfg.dynamicSmemBytes = kFusedSmem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = FCL;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(n, (void*)k_fused_spectrum, &cfg);
}

}  // namespace gcf

// ===========================================================================
// Allocation-free spectrum entry point.
//
// Some callers cannot call cudaMalloc: a host application whose framework
// owns every device allocation (a fixed arena or a pool with a hard budget),
// or an acquisition loop that must not allocate because cudaMalloc can
// synchronise the device.  gcf_avg_spectrum_noalloc computes the same
// averaged amplitude spectrum as the fused path above with the same kernel,
// but every byte of device storage it needs beyond the caller's input and
// output lives in the file-scope array below.
// ===========================================================================
namespace gcf {
namespace {

constexpr int kNaMaxItems = 16;                 // partial spectra in the scratch
constexpr int kNaMaxTilesPerItem = 256;         // => at most 4096 tiles per image
constexpr size_t kNaPartialBytes = (size_t)kNaMaxItems * FCX * FT * sizeof(float);   // 8.4 MB
constexpr size_t kNaTaperOff = kNaPartialBytes;                                        // 1 MB taper
constexpr size_t kNaTwOff = kNaTaperOff + (size_t)FT * FT * sizeof(float);            // 4 KB twiddles
constexpr size_t kNaMetaOff = kNaTwOff + (size_t)FT * sizeof(float2);                 // descriptors
struct NaMeta {
    FusedTab desc;
    int4 items[kNaMaxItems];
    int first[2];
    float inv[1];
};
constexpr size_t kNaBytes = kNaMetaOff + ((sizeof(NaMeta) + 255) / 256) * 256;

// The scratch.  In host code this name is only a stand-in; its device
// address comes from cudaGetSymbolAddress at set-up (na_setup).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
unsigned char* g_na_base[kNaMaxDevices] = {};
int g_na_clusters[kNaMaxDevices] = {};

// Once per device, with that device current: find the scratch address and
// fill the constant taper / twiddle tables inside it.
gcf_status na_setup(int dev, unsigned char** base, int* clusters)
{
    std::lock_guard<std::mutex> lk(g_na_mutex);
    if (g_na_base[dev]) {
        *base = g_na_base[dev];
        *clusters = g_na_clusters[dev];
        return GCF_OK;
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GCF_ERR_CUDA;
    std::vector<float> taper((size_t)FT * FT);
    const double c = FT * 0.5, s = FT;
    for (int y = 0; y < FT; ++y)
        for (int x = 0; x < FT; ++x) {   // GRoundEdge (FindCTF/GRoundEdge.cu:7-25)
            double fx = 2.0 * std::fabs(x - c) / s, fy = 2.0 * std::fabs(y - c) / s;
            double r = std::sqrt(fx * fx + fy * fy), v = 0.0;
            if (r < 1.0) {
                double q = 0.5 * (1.0 - std::cos(M_PI * r));
                v = 1.0 - q * q * q;
            }
            taper[(size_t)y * FT + x] = (float)v;
        }
    std::vector<float2> tw(FT);
    for (int t = 0; t < FT; ++t) {
        double a = -2.0 * M_PI * (double)t / FT;
        tw[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    unsigned char* b = static_cast<unsigned char*>(p);
    if (cudaMemcpy(b + kNaTaperOff, taper.data(), taper.size() * sizeof(float), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(b + kNaTwOff, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess)
        return GCF_ERR_CUDA;
    int n = 0;
    if (fused_max_clusters(&n) != cudaSuccess || n <= 0) return GCF_ERR_CUDA;
    g_na_base[dev] = b;
    g_na_clusters[dev] = n;
    *base = b;
    *clusters = n;
    return GCF_OK;
}

}  // namespace
}  // namespace gcf

extern "C" gcf_status gcf_avg_spectrum_noalloc(const float* dev_img, int width, int height, int pitch,
                                               float* dev_raw_out, void* cuda_stream)
{
    using namespace gcf;
    if (!dev_img || !dev_raw_out || width < FT || height < FT || pitch < width)
        return GCF_ERR_INVALID_ARG;
    // tile layout of CGenAvgSpectrum::SetSizes (FindCTF/CGenAvgSpectrum.cpp:40-75)
    int ov = (int)(FT * 0.50f) / 2 * 2, stride = FT - ov;
    int ntx = (width - ov) / stride, nty = (height - ov) / stride;
    int nt = ntx * nty;
    if (ntx <= 0 || nty <= 0) return GCF_ERR_IMAGE_TOO_SMALL;
    if (nt > kNaMaxItems * kNaMaxTilesPerItem) return GCF_ERR_INVALID_ARG;   // > 4096 tiles
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) return GCF_ERR_CUDA;
    unsigned char* base = nullptr;
    int clusters = 0;
    gcf_status s = na_setup(dev, &base, &clusters);
    if (s != GCF_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    NaMeta meta;
    std::memset(&meta, 0, sizeof(meta));
    meta.desc.img = dev_img;
    meta.desc.pitch = pitch;
    meta.desc.ntx = ntx;
    meta.desc.offx = (width - ntx * FT + (ntx - 1) * ov) / 2;
    meta.desc.offy = (height - nty * FT + (nty - 1) * ov) / 2;
    meta.desc.stride = stride;
    meta.desc.vec4 = ((meta.desc.offx % 4) == 0 && (stride % 4) == 0 && (pitch % 4) == 0 &&
                      ((uintptr_t)dev_img % 16) == 0) ? 1 : 0;
    int nitems = nt < kNaMaxItems ? nt : kNaMaxItems;
    int chunk = (nt + nitems - 1) / nitems;
    nitems = 0;
    for (int t0 = 0; t0 < nt; t0 += chunk, ++nitems)
        meta.items[nitems] = make_int4(0, t0, t0 + chunk < nt ? t0 + chunk : nt, nitems);
    meta.first[0] = 0;
    meta.first[1] = nitems;
    meta.inv[0] = 1.0f / nt;
    // Every partial element is written by the kernel before it is read, so
    // nothing in the scratch has to start at zero; the descriptors below are
    // rewritten on every call.
    NaMeta* dmeta = reinterpret_cast<NaMeta*>(base + kNaMetaOff);
    if (cudaMemcpyAsync(dmeta, &meta, sizeof(meta), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return GCF_ERR_CUDA;
    int ncl = clusters < nitems ? clusters : nitems;
    cudaError_t e = launch_fused(&dmeta->desc, dmeta->items, nitems, dmeta->first, dmeta->inv, 1,
                                 reinterpret_cast<const float*>(base + kNaTaperOff),
                                 reinterpret_cast<const float2*>(base + kNaTwOff),
                                 reinterpret_cast<float*>(base), dev_raw_out, ncl, st);
    if (e != cudaSuccess) return GCF_ERR_CUDA;
    // a copy from pageable memory has consumed `meta` when cudaMemcpyAsync returns
    return GCF_OK;
}
