// gcf_fused.cu -- fused tile-spectrum kernel for 512 x 512 tiles
// (CGenAvgSpectrum::DoIt + GCalcMoment2D + GNormalize2D + GRoundEdge +
//  GCalcSpectrum::DoPad + GAddImages, FindCTF/CGenAvgSpectrum.cpp:77-139).
//
// A thread-block cluster of CL CTAs (16, or 8 where 16-CTA clusters do not
// fit) owns one tile at a time; the tile never leaves the chip:
//   mean    every tile mean comes from one pass of k_block_sums over the
//           images (a 512 tile is 2 x 2 blocks of 256 x 256);
//   rows    each warp reads two tile rows straight from global memory,
//           forms (x - mean) * taper as the real and imaginary parts of one
//           512-point complex FFT held in registers (16 values per lane,
//           radix-16 x radix-32 with one shared-memory transpose), splits
//           the result into the two rows' 257-bin half spectra and pushes
//           each bin into the shared memory of the CTA that owns its
//           frequency column (16-byte DSMEM stores, [column][row]);
//   columns each warp transforms one frequency column (512 rows) read from
//           its own CTA's shared memory; the real kx = 0 and kx = 256
//           columns share one complex FFT;
//   |F|     amplitudes (DC moved to row 256) accumulate in registers across
//           all tiles of a work item and are written once.
// With CL = 16 the column buffer is double-buffered, so one cluster barrier
// per tile separates writers from readers.  Beside the cluster launch,
// k_fused_spectrum_solo runs one CTA on each SM that the clusters leave free
// (8-CTA clusters fit twice per GPC) and takes items from the back of the
// same queue.  Work items are (image, tile
// range) pairs, handed out in order through a counter; their partial
// spectra are summed in item order by k_item_reduce, so the result does not
// depend on which cluster took which item.
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

// exp(-2 pi i k / 32), k < 16, rounded to float from double like the host
// twiddle tables; written once per device before the first launch.
__constant__ float2 c_tw32[16];
constexpr int FCX = FT / 2 + 1;  // 257 half-spectrum columns
constexpr int FSCR = 16 * 34;    // per-warp scratch, float2 units
constexpr int FROW = 34;         // transpose row stride: 64-bit accesses of either side hit distinct banks

// Complex product, scalar.  The per-lane twiddles (read from shared
// memory) use it: a packed form with the twiddle stored pre-arranged
// (wx, wx, -wy, wy) measured slower, with twice the shared-memory reads.
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Complex product by a compile-time or constant-bank twiddle w as two packed
// operations: a * w = (a.x, a.y) (wx, wx) + (a.y, a.x) (-wy, wy).  (The form
// with a's halves broadcast, (a.x, a.x) w + (a.y, a.y) (-wy, wx), measured
// slower.)
__device__ __forceinline__ float2 cmul_k(float2 a, float2 w)
{
    return __ffma2_rn(make_float2(a.y, a.x), make_float2(-w.y, w.y), __fmul2_rn(a, make_float2(w.x, w.x)));
}
// Complex additions as packed two-float operations (one f32x2 instruction
// each; exact IEEE round-to-nearest like the scalar pair): halves the issue
// slots of the butterflies.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

// Forward 4-point DFT in place (W4 = -i).
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3)
{
    float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    const float2 sw = make_float2(d13.y, d13.x);
    a1 = __ffma2_rn(sw, make_float2(1.0f, -1.0f), d02);   // d02 - i d13
    a3 = __ffma2_rn(sw, make_float2(-1.0f, 1.0f), d02);   // d02 + i d13
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

// Slot of spectrum bin K (0..511) in the warp scratch when a whole FFT
// output is staged: bins 256..511 are shifted by 8 slots, so the 16-lane
// halves of the (m + 16 k + 256 p) stores hit distinct banks.
__device__ __forceinline__ int sslot(int K) { return K + ((K >> 8) << 3); }

// |z| with the fast square root (relative error within 2^-22): the
// amplitudes only enter averages compared at 1e-4.
__device__ __forceinline__ float amp(float x, float y)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x * x + y * y));
    return r;
}

// Position of output k of dft16 in its register array.
__host__ __device__ constexpr int P16(int k) { return (k & 3) * 4 + (k >> 2); }

// Forward 16-point DFT in registers, natural-order input, output k in
// v[P16(k)] (radix-4 x radix-4: n = 4 n1 + n2, k = k1 + 4 k2).
__device__ __forceinline__ void dft16(float2 (&v)[16])
{
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
#pragma unroll
    for (int k1 = 1; k1 < 4; ++k1)
#pragma unroll
        for (int n2 = 1; n2 < 4; ++n2) {
            if (n2 * k1 == 4) v[4 * k1 + n2] = make_float2(v[4 * k1 + n2].y, -v[4 * k1 + n2].x);   // * (-i)
            else v[4 * k1 + n2] = cmul_k(v[4 * k1 + n2], w16(n2 * k1));
        }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4(v[4 * k1 + 0], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
}

// 512-point forward FFT held by one warp.  In: lane l holds x[32 j + l] in
// v[j].  Out: lane 2m+p holds X[m + 16 k + 256 p] in v[P16(k)].
// scr: FSCR float2 of warp-private shared memory; twl[k1 * 32 + l] =
// exp(-2 pi i l k1 / 512); the 32-point twiddles are c_tw32.
__device__ __forceinline__ void fft512_warp(float2 (&v)[16], float2* scr, const float2* twl, int lane)
{
    dft16(v);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) v[P16(k1)] = cmul(v[P16(k1)], twl[k1 * 32 + lane]);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) scr[k1 * FROW + lane] = v[P16(k1)];
    __syncwarp();
    const int m = lane >> 1, p = lane & 1;
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = scr[m * FROW + 2 * q + p];
    dft16(v);
    // radix-2 across the lane pair: lane p = 1 multiplies its odd half by
    // the twiddle before the exchange, then lane 0 forms E0 + W E1 and
    // lane 1 forms E0 - W E1
    const float sg = p ? -1.0f : 1.0f;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float2 u = cmul_k(v[P16(k)], c_tw32[k]);
        if (!p) u = v[P16(k)];
        float2 o;
        o.x = __shfl_xor_sync(0xffffffffu, u.x, 1);
        o.y = __shfl_xor_sync(0xffffffffu, u.y, 1);
        v[P16(k)] = __ffma2_rn(make_float2(sg, sg), u, o);
    }
    __syncwarp();
}

struct FusedTab {
    const float* img;
    const double* bsum;   // sums of the stride x stride blocks, [nty + 1][ntx + 1]
    int pitch;
    int ntx, nty;
    int offx, offy, stride;
    int vec;              // 2: 8-byte aligned tile rows, 1: 4-byte
    int nbx;              // ntx + 1
};

// Sums of the stride x stride blocks that tile every image (tile = 2 stride,
// so a tile is 2 x 2 blocks): one pass over the images gives every tile mean
// of GCalcMoment2D (Util/GCalcMoment2D.cu:10-58) without a second read.
// Each warp sums whole block rows with 16-byte loads when the rows are
// 16-byte aligned (4 independent FP64 partial sums per lane keep several
// loads in flight); otherwise it falls back to 4-byte loads.
__global__ void __launch_bounds__(256) k_block_sums(const FusedTab* __restrict__ imgs,
                                                    double* const* __restrict__ out)
{
    __shared__ double sh[32];
    const FusedTab im = imgs[blockIdx.y];
    const int nby = im.nty + 1;
    const int b = blockIdx.x;
    if (b >= im.nbx * nby) return;
    const int bx = b % im.nbx, by = b / im.nbx, S = im.stride;
    const float* src = im.img + (size_t)(im.offy + by * S) * im.pitch + im.offx + bx * S;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool v4 = ((reinterpret_cast<uintptr_t>(src) & 15) == 0) && (im.pitch % 4 == 0) && (S % 4 == 0);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    if (v4) {
        const int q = S / 4;   // float4 per block row
        // unrolled so that several 16-byte loads per thread are in flight
        // (the additions keep their order): 2.75 GB in 0.42 ms, the measured
        // copy bandwidth, against 0.53 ms with one load in flight
#pragma unroll 4
        for (int y = warp; y < S; y += nw) {
            const float4* row = reinterpret_cast<const float4*>(src + (size_t)y * im.pitch);
#pragma unroll 2
            for (int x = lane; x < q; x += 32) {
                float4 v = __ldg(row + x);
                s0 += (double)v.x;
                s1 += (double)v.y;
                s2 += (double)v.z;
                s3 += (double)v.w;
            }
        }
    } else {
        for (int y = warp; y < S; y += nw) {
            const float* row = src + (size_t)y * im.pitch;
            for (int x = lane; x < S; x += 32) s0 += (double)__ldg(row + x);
        }
    }
    double s = (s0 + s1) + (s2 + s3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) sh[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += sh[w];
        out[blockIdx.y][b] = t;
    }
}

// The work-item queue of one launch: a 64-bit counter whose low half counts
// items taken from the front (by clusters) and whose high half counts items
// taken from the back (by the cluster-less CTAs).  An index >= nitems means
// the queue is empty.
__device__ __forceinline__ int take_front(unsigned long long* q, int nitems)
{
    const unsigned long long old = atomicAdd(q, 1ull);
    const unsigned front = (unsigned)old, back = (unsigned)(old >> 32);
    return front + back < (unsigned)nitems ? (int)front : nitems;
}
// From the back, while more than `reserve` items remain: a cluster-less CTA
// takes about eight times as long per item as a cluster, so it must not
// take one of the last items, or it would end the launch late.
__device__ __forceinline__ int take_back(unsigned long long* q, int nitems, int reserve)
{
    const unsigned long long cur = atomicAdd(q, 0ull);
    if ((long long)nitems - (long long)((unsigned)cur + (unsigned)(cur >> 32)) <= (long long)reserve) return nitems;
    const unsigned long long old = atomicAdd(q, 1ull << 32);
    const unsigned front = (unsigned)old, back = (unsigned)(old >> 32);
    return front + back < (unsigned)nitems ? nitems - 1 - (int)back : nitems;
}

// Compile-time shape of one cluster configuration.
template <int CL_, int NW_, bool DB_, bool PF_ = true, int MINB_ = 1>
struct FusedShape {
    static constexpr int CL = CL_;                   // CTAs per cluster
    static constexpr int NW = NW_;                   // warps per CTA
    static constexpr bool DB = DB_;                  // double-buffered column buffer
    static constexpr bool PF = PF_;                  // register prefetch of the next row pair
    static constexpr int MINB = MINB_;               // CTAs per SM the registers are sized for
    static constexpr int THR = NW * 32;
    static constexpr int R = FT / CL;                // tile rows per CTA
    static constexpr int C = FT / 2 / CL;            // frequency columns per CTA
    static constexpr int PW = R / 2 / NW;            // row pairs per warp
    static constexpr int NR = C / NW;                // column rounds per warp
    static constexpr int YS = FT + 2;                // column stride of the buffer (16-byte rows, pad)
    static constexpr size_t BUF = (size_t)C * YS * sizeof(float2);   // this CTA's C columns x 512 rows
    static constexpr size_t SCR = (size_t)NW * FSCR * sizeof(float2);
    static constexpr size_t TWL = 16 * 32 * sizeof(float2);
    static constexpr size_t ACCN = FT * sizeof(float);
    static constexpr size_t SMEM = (DB ? 2 : 1) * BUF + SCR + TWL + ACCN;
    static_assert(R % 32 == 0 && PW >= 1 && NR >= 1 && R / 2 == PW * NW && C == NR * NW && C <= 32, "shape");
};
using Shape16 = FusedShape<16, 16, true>;         // 16-CTA clusters, 512 threads
using Shape8 = FusedShape<8, 8, false>;           // 8-CTA clusters, 256 threads
using Shape8W16 = FusedShape<8, 16, false, false>;  // 8-CTA clusters, 512 threads, 128 registers
// 16-CTA clusters of 256 threads at <= 128 registers and 107 KB of shared
// memory: two CTAs (of different clusters, or of one) per SM, so one CTA's
// cluster barrier or DSMEM exchange overlaps the other's FFTs
using Shape16x2 = FusedShape<16, 8, false, false, 2>;
// 16-CTA clusters of 8 warps with the column buffer double-buffered (one
// cluster barrier per tile) and half the per-warp accumulators of Shape8
using Shape16W8 = FusedShape<16, 8, true>;

template <class S>
__global__ void __launch_bounds__(S::THR, S::MINB)
k_fused_spectrum(const FusedTab* __restrict__ imgs, const int4* __restrict__ items, int nitems,
                 const float* __restrict__ taper, const float2* __restrict__ twg,
                 float* __restrict__ partial, unsigned long long* __restrict__ next_item)
{
    constexpr int CL = S::CL, NW = S::NW, R = S::R, C = S::C, PW = S::PW, NR = S::NR, YS = S::YS;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* colbuf0 = reinterpret_cast<float2*>(smem);
    float2* scr_all = reinterpret_cast<float2*>(smem + (S::DB ? 2 : 1) * S::BUF);
    float2* twl = reinterpret_cast<float2*>(smem + (S::DB ? 2 : 1) * S::BUF + S::SCR);
    float* accN = reinterpret_cast<float*>(twl + 16 * 32);

    __shared__ int s_item[2];   // the item rank 0 fetched, by item parity
    cg::cluster_group cluster = cg::this_cluster();
    const int r = (int)cluster.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = lane >> 1, p = lane & 1;
    float2* scr = scr_all + warp * FSCR;

    // per-lane twiddles exp(-2 pi i l k1 / 512)
    for (int i = tid; i < 16 * 32; i += S::THR) twl[i] = twg[((i & 31) * (i >> 5)) & (FT - 1)];
    __syncthreads();

    int par = 0;    // column-buffer parity (double buffering)
    int ipar = 0;   // s_item parity
    for (;;) {
        // Items are taken in order from one counter, so clusters that become
        // resident late (SMs held by concurrent kernels) simply take fewer.
        // Each s_item slot is rewritten two items later, after a cluster
        // barrier that every peer reaches only once it has read the slot.
        if (r == 0 && tid == 0) s_item[ipar] = take_front(next_item, nitems);
        cluster.sync();
        const int it = *cluster.map_shared_rank(&s_item[ipar], 0);
        ipar ^= 1;
        if (it >= nitems) break;
        const int4 item = items[it];   // (image, first tile, end tile, item index)
        const FusedTab im = imgs[item.x];
        float acc[NR][16];
#pragma unroll
        for (int a = 0; a < NR; ++a)
#pragma unroll
            for (int k = 0; k < 16; ++k) acc[a][k] = 0.0f;
        for (int i = tid; i < FT; i += S::THR) accN[i] = 0.0f;

        for (int t = item.y; t < item.z; ++t) {
            const int tx = t % im.ntx, ty = t / im.ntx;
            const float* src = im.img + (size_t)(im.offy + ty * im.stride + r * R) * im.pitch +
                               im.offx + tx * im.stride;
            // tile mean = four block sums / tile area
            const double* bs = im.bsum + (size_t)ty * im.nbx + tx;
            const float mean = (float)((bs[0] + bs[1] + bs[im.nbx] + bs[im.nbx + 1]) / ((double)FT * FT));
            float2* colbuf = colbuf0 + (S::DB ? (size_t)par * (S::BUF / sizeof(float2)) : 0);
            // peers are done reading this CTA's column buffer: an execution
            // barrier only (the values those reads returned were consumed by
            // the column transforms before the arrive), so the arrive is
            // relaxed and carries no memory fence
            if (!S::DB) {
                asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
                asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
            }

            // ---- row transforms: two rows per FFT, rows read straight from global ----
            // S::PF: the next row pair is loaded into registers while this one
            // is transformed (for 8-warp CTAs, whose 255 registers allow it)
            float na[S::PF ? 16 : 1], nb[S::PF ? 16 : 1];
            if constexpr (S::PF) {
                const float* ga = src + (size_t)(2 * warp) * im.pitch;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    na[j] = __ldg(ga + 32 * j + lane);
                    nb[j] = __ldg(ga + im.pitch + 32 * j + lane);
                }
            }
#pragma unroll
            for (int q4 = 0; q4 < PW; ++q4) {
                const int pp = warp + q4 * NW;
                const int y0 = 2 * pp, Y0 = r * R + y0;
                float ca[16], cb[16];
                if constexpr (S::PF) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        ca[j] = na[j];
                        cb[j] = nb[j];
                    }
                    if (q4 + 1 < PW) {   // prefetch the next row pair
                        const float* ga = src + (size_t)(2 * (pp + NW)) * im.pitch;
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            na[j] = __ldg(ga + 32 * j + lane);
                            nb[j] = __ldg(ga + im.pitch + 32 * j + lane);
                        }
                    }
                } else {
                    const float* ga = src + (size_t)y0 * im.pitch;
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        ca[j] = __ldg(ga + 32 * j + lane);
                        cb[j] = __ldg(ga + im.pitch + 32 * j + lane);
                    }
                }
                float2 v[16];
                const float* ta = taper + (size_t)Y0 * FT;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    int X = 32 * j + lane;
                    v[j] = make_float2((ca[j] - mean) * __ldg(ta + X), (cb[j] - mean) * __ldg(ta + FT + X));
                }
                fft512_warp(v, scr, twl, lane);
#pragma unroll
                for (int k = 0; k < 16; ++k) scr[sslot(m + 16 * k + 256 * p)] = v[P16(k)];
                __syncwarp();
                // split into the two rows' half spectra and push bin K of both rows
                // into the shared memory of CTA K / C (column K % C, rows Y0, Y0 + 1)
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int K = lane + 32 * i;
                    float2 zk = scr[sslot(K)], zn = scr[sslot((FT - K) & (FT - 1))];
                    // twice the two rows' bins (the 1/2 of the split is applied
                    // once, exactly, to the averaged spectrum in k_item_reduce)
                    float4 AB = make_float4(zk.x + zn.x, zk.y - zn.y, zk.y + zn.y, zn.x - zk.x);
                    if (K == 0) {   // pack the real DC and Nyquist bins of both rows
                        float2 zh = scr[sslot(FT / 2)];
                        AB = make_float4(2.0f * zk.x, 2.0f * zh.x, 2.0f * zk.y, 2.0f * zh.y);
                    }
                    float2* dst = cluster.map_shared_rank(colbuf, K / C) + (size_t)(K % C) * YS + Y0;
                    *reinterpret_cast<float4*>(dst) = AB;
                }
                __syncwarp();
            }
            // every column buffer of the cluster is complete (with double
            // buffering this also tells writers of the other buffer that its
            // previous readers are done)
            cluster.sync();

            // ---- column transforms from local shared memory ---------------------
            if (t + 1 < item.z) {   // next tile's rows into L2 while the columns run
                const int t1 = t + 1, tx1 = t1 % im.ntx, ty1 = t1 / im.ntx;
                const float* src1 = im.img + (size_t)(im.offy + ty1 * im.stride + r * R) * im.pitch +
                                    im.offx + tx1 * im.stride;
                for (int q = tid; q < R * 16; q += S::THR) {   // 128-byte lines
                    const float* g = src1 + (size_t)(q >> 4) * im.pitch + (q & 15) * 32;
                    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(g));
                }
            }
#pragma unroll
            for (int rho = 0; rho < NR; ++rho) {
                const int cl = NW * rho + warp;   // local column
                const int K = C * r + cl;         // frequency bin; 0 = packed (0, 256)
                float2 v[16];
                const float2* col = colbuf + (size_t)cl * YS;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = col[32 * j + lane];
                fft512_warp(v, scr, twl, lane);
                if (K != 0) {
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        float2 z = v[P16(k)];
                        acc[rho][k] += amp(z.x, z.y);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 16; ++k) scr[sslot(m + 16 * k + 256 * p)] = v[P16(k)];
                    __syncwarp();
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        int Kk = m + 16 * k + 256 * p;
                        float2 zk = v[P16(k)], zn = scr[sslot((FT - Kk) & (FT - 1))];
                        float ax = 0.5f * (zk.x + zn.x), ay = 0.5f * (zk.y - zn.y);
                        float bx = 0.5f * (zk.y + zn.y), by = -0.5f * (zk.x - zn.x);
                        acc[rho][k] += amp(ax, ay);
                        accN[Kk] += amp(bx, by);
                    }
                    __syncwarp();
                }
            }
            par ^= 1;
        }
        // ---- write this item's partial spectrum (DC moved to row 256) -----------
        float* out = partial + (size_t)item.w * FCX * FT;
#pragma unroll
        for (int rho = 0; rho < NR; ++rho) {
            const int kx = C * r + NW * rho + warp;
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
                int Kk = m + 16 * k + 256 * p;
                int yd = (Kk + FT / 2) & (FT - 1);
                out[(size_t)yd * FCX + FT / 2] = accN[Kk];
            }
        }
        __syncthreads();
    }
    cluster.sync();   // keep shared memory alive until every peer is done
}

// ---- tiles on the SMs that the clusters leave free --------------------------
// 8-CTA clusters fit twice per GPC, so some SMs stay idle beside the cluster
// kernel.  One CTA of this kernel runs on each of them, takes work items
// from the same counter and transforms whole tiles alone: the row spectra go
// to the CTA's column buffer in global memory (L2-resident scratch), the
// column transforms read them back, and the item's |F| sums live in a second
// global buffer ([column][row]) until the item ends, when they are written
// to the item's partial spectrum in the cluster kernel's layout.  The
// transforms, the split and the order of every addition are those of
// k_fused_spectrum, so an item's partial spectrum does not depend on which
// kernel took it.
constexpr int kSoloThreads = 256;
constexpr int kSoloWarps = kSoloThreads / 32;
constexpr int kSoloYS = FT + 2;                                      // column stride, float2
constexpr size_t kSoloColFloat2 = (size_t)(FT / 2) * kSoloYS;        // columns 0..255 of one tile
constexpr size_t kSoloAccFloats = (size_t)(FT / 2) * FT;             // |F| sums, [column][row]
constexpr size_t kSoloSmem = (size_t)kSoloWarps * FSCR * sizeof(float2) + 16 * 32 * sizeof(float2) +
                             FT * sizeof(float);

__global__ void __launch_bounds__(kSoloThreads, 1)
k_fused_spectrum_solo(const FusedTab* __restrict__ imgs, const int4* __restrict__ items, int nitems,
                      const float* __restrict__ taper, const float2* __restrict__ twg,
                      float* __restrict__ partial, unsigned long long* __restrict__ next_item, int reserve,
                      float2* __restrict__ colg_all, float* __restrict__ accg_all)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float2* scr_all = reinterpret_cast<float2*>(smem);
    float2* twl = scr_all + kSoloWarps * FSCR;
    float* accN = reinterpret_cast<float*>(twl + 16 * 32);
    __shared__ int s_item;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = lane >> 1, p = lane & 1;
    float2* scr = scr_all + warp * FSCR;
    float2* colg = colg_all + (size_t)blockIdx.x * kSoloColFloat2;
    float* accg = accg_all + (size_t)blockIdx.x * kSoloAccFloats;
    for (int i = tid; i < 16 * 32; i += kSoloThreads) twl[i] = twg[((i & 31) * (i >> 5)) & (FT - 1)];
    for (;;) {
        __syncthreads();   // the previous item is written; every thread has read s_item
        if (tid == 0) s_item = take_back(next_item, nitems, reserve);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int4 item = items[it];   // (image, first tile, end tile, item index)
        const FusedTab im = imgs[item.x];
        for (int i = tid; i < FT; i += kSoloThreads) accN[i] = 0.0f;   // read after the row phase's barrier
        for (int t = item.y; t < item.z; ++t) {
            const bool first = t == item.y;
            const int tx = t % im.ntx, ty = t / im.ntx;
            const float* src = im.img + (size_t)(im.offy + ty * im.stride) * im.pitch + im.offx + tx * im.stride;
            const double* bs = im.bsum + (size_t)ty * im.nbx + tx;
            const float mean = (float)((bs[0] + bs[1] + bs[im.nbx] + bs[im.nbx + 1]) / ((double)FT * FT));

            // ---- row transforms: 256 row pairs, the next pair prefetched --------
            float na[16], nb[16];
            {
                const float* ga = src + (size_t)(2 * warp) * im.pitch;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    na[j] = __ldg(ga + 32 * j + lane);
                    nb[j] = __ldg(ga + im.pitch + 32 * j + lane);
                }
            }
            for (int q = 0; q < FT / 2 / kSoloWarps; ++q) {
                const int Y0 = 2 * (warp + kSoloWarps * q);
                float ca[16], cb[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    ca[j] = na[j];
                    cb[j] = nb[j];
                }
                if (q + 1 < FT / 2 / kSoloWarps) {
                    const float* ga = src + (size_t)(Y0 + 2 * kSoloWarps) * im.pitch;
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        na[j] = __ldg(ga + 32 * j + lane);
                        nb[j] = __ldg(ga + im.pitch + 32 * j + lane);
                    }
                }
                float2 v[16];
                const float* ta = taper + (size_t)Y0 * FT;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    int X = 32 * j + lane;
                    v[j] = make_float2((ca[j] - mean) * __ldg(ta + X), (cb[j] - mean) * __ldg(ta + FT + X));
                }
                fft512_warp(v, scr, twl, lane);
#pragma unroll
                for (int k = 0; k < 16; ++k) scr[sslot(m + 16 * k + 256 * p)] = v[P16(k)];
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int K = lane + 32 * i;
                    float2 zk = scr[sslot(K)], zn = scr[sslot((FT - K) & (FT - 1))];
                    float4 AB = make_float4(zk.x + zn.x, zk.y - zn.y, zk.y + zn.y, zn.x - zk.x);
                    if (K == 0) {
                        float2 zh = scr[sslot(FT / 2)];
                        AB = make_float4(2.0f * zk.x, 2.0f * zh.x, 2.0f * zk.y, 2.0f * zh.y);
                    }
                    *reinterpret_cast<float4*>(colg + (size_t)K * kSoloYS + Y0) = AB;
                }
                __syncwarp();
            }
            __syncthreads();   // the tile's column buffer is complete

            // ---- column transforms from the global column buffer ----------------
            for (int cc = 0; cc < FT / 2 / kSoloWarps; ++cc) {
                const int K = warp + kSoloWarps * cc;   // 0 = packed (0, 256)
                float2 v[16];
                const float2* col = colg + (size_t)K * kSoloYS;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = col[32 * j + lane];
                float* a = accg + (size_t)K * FT;
                float av[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) av[k] = first ? 0.0f : a[m + 16 * k + 256 * p];
                fft512_warp(v, scr, twl, lane);
                if (K != 0) {
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        float2 z = v[P16(k)];
                        a[m + 16 * k + 256 * p] = av[k] + amp(z.x, z.y);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 16; ++k) scr[sslot(m + 16 * k + 256 * p)] = v[P16(k)];
                    __syncwarp();
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        int Kk = m + 16 * k + 256 * p;
                        float2 zk = v[P16(k)], zn = scr[sslot((FT - Kk) & (FT - 1))];
                        float ax = 0.5f * (zk.x + zn.x), ay = 0.5f * (zk.y - zn.y);
                        float bx = 0.5f * (zk.y + zn.y), by = -0.5f * (zk.x - zn.x);
                        a[Kk] = av[k] + amp(ax, ay);
                        accN[Kk] += amp(bx, by);
                    }
                    __syncwarp();
                }
            }
            __syncthreads();   // the column buffer is free again; the sums are complete
        }
        // ---- the item's partial spectrum (DC moved to row 256) ------------------
        float* out = partial + (size_t)item.w * FCX * FT;
        for (int i = tid; i < (FT / 2) * FT; i += kSoloThreads) {
            const int kx = i / FT, ky = i - kx * FT;
            out[(size_t)((ky + FT / 2) & (FT - 1)) * FCX + kx] = accg[i];
        }
        for (int ky = tid; ky < FT; ky += kSoloThreads)
            out[(size_t)((ky + FT / 2) & (FT - 1)) * FCX + FT / 2] = accN[ky];
    }
}

// raw[img] = sum of the img's item partials (in item order) / ntiles / 2.
__global__ void k_item_reduce(const float* __restrict__ partial, const int* __restrict__ first,
                              const float* __restrict__ inv, float* __restrict__ raw)
{
    const int n = FCX * FT;
    int img = blockIdx.y;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = first[img]; k < first[img + 1]; ++k) s += partial[(size_t)k * n + i];
    raw[(size_t)img * n + i] = (float)(s * (double)inv[img] * 0.5);   // rows were split without the 1/2
}

template <class S>
cudaLaunchConfig_t fused_cfg(int nclusters, cudaStream_t st, cudaLaunchAttribute* attr)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nclusters * S::CL, 1, 1);
    cfg.blockDim = dim3(S::THR, 1, 1);
    cfg.dynamicSmemBytes = S::SMEM;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = S::CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// c_tw32 of the current device, once.
cudaError_t init_constants()
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
        double a = -2.0 * M_PI * (double)(16 * k) / FT;
        w[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    e = cudaMemcpyToSymbol(c_tw32, w, sizeof(w));
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

template <class S>
cudaError_t prepare_kernel()
{
    cudaError_t ec = init_constants();
    if (ec != cudaSuccess) return ec;
    cudaError_t e = cudaFuncSetAttribute(k_fused_spectrum<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)S::SMEM);
    if (e != cudaSuccess) return e;
    if (S::CL > 8) e = cudaFuncSetAttribute(k_fused_spectrum<S>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}

template <class S>
cudaError_t max_clusters(int* n)
{
    *n = 0;
    cudaError_t e = prepare_kernel<S>();
    if (e != cudaSuccess) return e;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = fused_cfg<S>(64, nullptr, attr);
    return cudaOccupancyMaxActiveClusters(n, (void*)k_fused_spectrum<S>, &cfg);
}

// ---- B-factor lowpass of 512 x 512 spectra with the warp FFT ----------------
// CFindCtfBase::mLowpass (FindCTF/CFindCtfBase.cpp:191-219) filters the full
// spectrum F (512 x 512 real, DC at column 256) by a forward R2C, the
// factor exp(-B (kx^2 + ky^2) / (2 N^2)) / N^2 (GLowpass2D::DoBFactor,
// FindCTF/GLowpass2D.cu:9-23) and a C2R.  The factor is a product of one
// real, even function per axis, so the filter is separable: rows first,
// then columns, each  r' = IDFT(g DFT(r)) / N  with g(k) = exp(-B k^2 / (2 N^2))
// (k wrapped to -N/2 .. N/2).  Because g is real and even it keeps real
// signals real, so two rows (columns) a, b go through one complex FFT as
// a + i b and come back as a' + i b' with no split; the inverse is the
// forward FFT of the conjugate.
constexpr int kLpWarps = 8;

// Filter values g(K) / N for the output layout of fft512_warp: lane 2m+p
// holds bin K = m + 16k + 256p in v[P16(k)].
__device__ __forceinline__ void lp_filter_pass(float2 (&v)[16], float2* scr, const float2* twl, const float* gk,
                                               int lane)
{
    const int m = lane >> 1, p = lane & 1;
    fft512_warp(v, scr, twl, lane);
    // multiply, conjugate and put the spectrum back into natural order
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int K = m + 16 * k + 256 * p;
        const float g = gk[K];
        scr[sslot(K)] = make_float2(v[P16(k)].x * g, -v[P16(k)].y * g);
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = scr[sslot(32 * j + lane)];
    __syncwarp();
    fft512_warp(v, scr, twl, lane);   // conj(result) = the filtered pair, bin order
}

__device__ __forceinline__ void lp_setup(float2* twl, float* gk, const float2* twg, double bfactor)
{
    for (int i = threadIdx.x; i < 16 * 32; i += blockDim.x) twl[i] = twg[((i & 31) * (i >> 5)) & (FT - 1)];
    const double scale = -bfactor / (2.0 * (double)FT * FT);
    for (int k = threadIdx.x; k < FT; k += blockDim.x) {
        const int kw = k <= FT / 2 ? k : k - FT;
        gk[k] = (float)(exp(scale * (double)kw * kw) / (double)FT);
    }
    __syncthreads();
}

// Rows: one warp per row pair of the full spectrum built from the half
// spectrum (GCalcSpectrum::GenFullSpect's mirror, DC at column 256);
// filtered rows to rowf [m][512][512].
__global__ void __launch_bounds__(kLpWarps * 32)
k_lowpass_rows(const float* __restrict__ ctf0, const float2* __restrict__ twg, double bfactor,
               float* __restrict__ rowf)
{
    __shared__ float2 s_twl[16 * 32];
    __shared__ float s_g[FT];
    __shared__ float2 s_scr[kLpWarps][FSCR];
    lp_setup(s_twl, s_g, twg, bfactor);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = blockIdx.y, y0 = 2 * (blockIdx.x * kLpWarps + warp);
    const float* half = ctf0 + (size_t)m * FCX * FT;
    float2 v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int X = 32 * j + lane, xd = X - (FCX - 1);
        float a, b;
        if (xd >= 0) {
            a = half[(size_t)y0 * FCX + xd];
            b = half[(size_t)(y0 + 1) * FCX + xd];
        } else {
            const int ya = (FT - y0) & (FT - 1), yb = (FT - y0 - 1) & (FT - 1);
            a = half[(size_t)ya * FCX - xd];
            b = half[(size_t)yb * FCX - xd];
        }
        v[j] = make_float2(a, b);
    }
    float2* scr = s_scr[warp];
    lp_filter_pass(v, scr, s_twl, s_g, lane);
    // the pair leaves through the scratch in bin order: coalesced rows
    const int mm = lane >> 1, p = lane & 1;
#pragma unroll
    for (int k = 0; k < 16; ++k) scr[sslot(mm + 16 * k + 256 * p)] = v[P16(k)];
    __syncwarp();
    float* ra = rowf + ((size_t)m * FT + y0) * FT;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const float2 z = scr[sslot(32 * j + lane)];
        ra[32 * j + lane] = z.x;          // conjugate: a' = Re, b' = -Im
        ra[FT + 32 * j + lane] = -z.y;
    }
}

// Columns: a CTA takes 32 adjacent columns of the row-filtered spectrum
// (a 512 x 32 block through shared memory, 128-byte rows), each warp two
// column pairs; only the columns of the half spectrum are kept: out[y][x] =
// filtered[y][x + 256] (x < 256) and out[y][256] = filtered[y][0]
// (CFindCtfBase.cpp:212-218).  Spectra whose background-removed variance is
// below 1 keep ctf0 (the variance gate of mRemoveBackground,
// FindCTF/CFindCtfBase.cpp:169-174).
__global__ void __launch_bounds__(kLpWarps * 32)
k_lowpass_cols(const float* __restrict__ rowf, const float* __restrict__ ctf0, const float2* __restrict__ twg,
               double bfactor, const double* __restrict__ mom, float* __restrict__ out, int* __restrict__ lowpassed)
{
    extern __shared__ float s_blk[];   // [512][33]
    __shared__ float2 s_twl[16 * 32];
    __shared__ float s_g[FT];
    __shared__ float2 s_scr[kLpWarps][FSCR];
    const int m = blockIdx.y;
    // blocks 0..7: columns 256 + 32 b ..; block 8: columns 0 .. 31 (column 0 kept)
    const int c0 = blockIdx.x < 8 ? FT / 2 + 32 * blockIdx.x : 0;
    const double mean = mom[2 * m], var = mom[2 * m + 1] - mean * mean;
    const bool run = !(var < 1.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) lowpassed[m] = run ? 1 : 0;
    float* o = out + (size_t)m * FCX * FT;
    const float* h0 = ctf0 + (size_t)m * FCX * FT;
    if (!run) {
        for (int i = threadIdx.x; i < FT * 32; i += blockDim.x) {
            const int y = i >> 5, X = c0 + (i & 31);
            const int x = X >= FT / 2 ? X - FT / 2 : (X == 0 ? FT / 2 : -1);
            if (x >= 0) o[(size_t)y * FCX + x] = h0[(size_t)y * FCX + x];
        }
        return;
    }
    lp_setup(s_twl, s_g, twg, bfactor);
    const float* src = rowf + (size_t)m * FT * FT + c0;
    for (int i = threadIdx.x; i < FT * 32; i += blockDim.x) {
        const int y = i >> 5, c = i & 31;
        s_blk[y * 33 + c] = src[(size_t)y * FT + c];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float2* scr = s_scr[warp];
    const int npairs = c0 == 0 ? 1 : 2;   // block 8 needs columns 0 and 1 only
    for (int q = 0; q < npairs; ++q) {
        const int cl = 2 * (2 * warp + q);   // local column of a; b = cl + 1
        if (c0 == 0 && warp != 0) break;
        float2 v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int y = 32 * j + lane;
            v[j] = make_float2(s_blk[y * 33 + cl], s_blk[y * 33 + cl + 1]);
        }
        lp_filter_pass(v, scr, s_twl, s_g, lane);
        const int mm = lane >> 1, p = lane & 1;
        const int Xa = c0 + cl;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int y = mm + 16 * k + 256 * p;
            const float2 z = v[P16(k)];
            if (Xa >= FT / 2) {
                o[(size_t)y * FCX + (Xa - FT / 2)] = z.x;
                o[(size_t)y * FCX + (Xa + 1 - FT / 2)] = -z.y;
            } else {   // Xa == 0: column 0 becomes the last half-spectrum column
                o[(size_t)y * FCX + FT / 2] = z.x;
            }
        }
    }
}

}  // namespace

int fused_tile_supported(int tile) { return tile == FT ? 1 : 0; }

cudaError_t launch_lowpass512(const float* ctf0, const float2* tw, double bfactor, int nmic, const double* moments,
                              float* rowf, float* out, int* lowpassed, cudaStream_t st)
{
    if (nmic <= 0) return cudaSuccess;
    cudaError_t e = init_constants();
    if (e != cudaSuccess) return e;
    k_lowpass_rows<<<dim3(FT / 2 / kLpWarps, nmic), kLpWarps * 32, 0, st>>>(ctf0, tw, bfactor, rowf);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t sm = (size_t)FT * 33 * sizeof(float);
    if ((e = cudaFuncSetAttribute(k_lowpass_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) !=
        cudaSuccess)
        return e;
    k_lowpass_cols<<<dim3(9, nmic), kLpWarps * 32, sm, st>>>(rowf, ctf0, tw, bfactor, moments, out, lowpassed);
    return cudaGetLastError();
}

// Picks the cluster shape that covers the most SMs: 16-CTA clusters (double
// buffered) when the device can co-schedule them, else 8-CTA clusters.
cudaError_t fused_max_clusters(int* n, int* shape)
{
    int n16 = 0, n8 = 0;
    if (max_clusters<Shape16>(&n16) != cudaSuccess) {
        cudaGetLastError();
        n16 = 0;
    }
    cudaError_t e = max_clusters<Shape8>(&n8);
    if (e != cudaSuccess && n16 == 0) return e;
    if (n16 * 16 >= n8 * 8 && n16 > 0) {
        *n = n16;
        *shape = 16;
    } else {
        *n = n8;
        *shape = 8;
    }
    return cudaSuccess;
}

// Co-resident clusters of one shape: 8 (8 CTAs x 8 warps), 816 (8 CTAs x 16
// warps, 128 registers), 16 (16 CTAs x 16 warps, double buffered), 162 (16
// CTAs x 8 warps, two CTAs per SM), 168 (16 CTAs x 8 warps, double buffered).
cudaError_t fused_clusters_of(int shape, int* n)
{
    *n = 0;
    switch (shape) {
    case 8: return max_clusters<Shape8>(n);
    case 816: return max_clusters<Shape8W16>(n);
    case 16: return max_clusters<Shape16>(n);
    case 162: return max_clusters<Shape16x2>(n);
    case 168: return max_clusters<Shape16W8>(n);
    default: return cudaErrorInvalidValue;
    }
}

// Host launcher.  descs/items/first/inv are device arrays prepared by the caller.
size_t solo_scratch_float2(int nsolo) { return (size_t)nsolo * kSoloColFloat2; }
size_t solo_scratch_floats(int nsolo) { return (size_t)nsolo * kSoloAccFloats; }

cudaError_t launch_fused(const void* descs, double* const* bsum_out, int max_blocks, const int4* items,
                         int nitems, const int* first, const float* inv, int img0, int nimg,
                         const float* taper, const float2* tw, float* partial, float* raw,
                         unsigned long long* next_item, int nclusters, int shape, cudaStream_t st, cudaEvent_t ev0,
                         cudaEvent_t ev1, const SoloLaunch* solo)
{
    if (nclusters < 1) nclusters = 1;
    k_block_sums<<<dim3(max_blocks, nimg), 256, 0, st>>>(reinterpret_cast<const FusedTab*>(descs) + img0,
                                                          bsum_out + img0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(next_item, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
    if (ev0 && (e = record_timing(ev0, st)) != cudaSuccess) return e;
    const bool use_solo = solo && solo->n > 0 && nitems > nclusters;
    if (use_solo) {
        if ((e = cudaEventRecord(solo->fork, st)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(solo->st, solo->fork, 0)) != cudaSuccess) return e;
    }
    cudaLaunchAttribute attr[1];
    if (shape == 16) {
        if ((e = prepare_kernel<Shape16>()) != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = fused_cfg<Shape16>(nclusters, st, attr);
        e = cudaLaunchKernelEx(&cfg, k_fused_spectrum<Shape16>, reinterpret_cast<const FusedTab*>(descs), items,
                               nitems, taper, tw, partial, next_item);
    } else if (shape == 168) {
        if ((e = prepare_kernel<Shape16W8>()) != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = fused_cfg<Shape16W8>(nclusters, st, attr);
        e = cudaLaunchKernelEx(&cfg, k_fused_spectrum<Shape16W8>, reinterpret_cast<const FusedTab*>(descs),
                               items, nitems, taper, tw, partial, next_item);
    } else if (shape == 162) {
        if ((e = prepare_kernel<Shape16x2>()) != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = fused_cfg<Shape16x2>(nclusters, st, attr);
        e = cudaLaunchKernelEx(&cfg, k_fused_spectrum<Shape16x2>, reinterpret_cast<const FusedTab*>(descs),
                               items, nitems, taper, tw, partial, next_item);
    } else if (shape == 816) {
        if ((e = prepare_kernel<Shape8W16>()) != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = fused_cfg<Shape8W16>(nclusters, st, attr);
        e = cudaLaunchKernelEx(&cfg, k_fused_spectrum<Shape8W16>, reinterpret_cast<const FusedTab*>(descs),
                               items, nitems, taper, tw, partial, next_item);
    } else {
        if ((e = prepare_kernel<Shape8>()) != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = fused_cfg<Shape8>(nclusters, st, attr);
        e = cudaLaunchKernelEx(&cfg, k_fused_spectrum<Shape8>, reinterpret_cast<const FusedTab*>(descs), items,
                               nitems, taper, tw, partial, next_item);
    }
    if (e != cudaSuccess) return e;
    if (use_solo) {
        // after the cluster launch, so that its clusters are placed first and
        // these CTAs land on the SMs they leave free
        k_fused_spectrum_solo<<<solo->n, kSoloThreads, kSoloSmem, solo->st>>>(
            reinterpret_cast<const FusedTab*>(descs), items, nitems, taper, tw, partial, next_item,
            solo->reserve_per_cluster * nclusters, solo->col, solo->acc);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(solo->join, solo->st)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(st, solo->join, 0)) != cudaSuccess) return e;
    }
    if (ev1 && (e = record_timing(ev1, st)) != cudaSuccess) return e;
    dim3 g((FCX * FT + 255) / 256, nimg);
    k_item_reduce<<<g, 256, 0, st>>>(partial, first + img0, inv + img0, raw);
    return cudaGetLastError();
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
constexpr size_t kNaBsumOff = kNaTwOff + (size_t)FT * sizeof(float2);                 // block sums
constexpr int kNaMaxBlocks = 2 * kNaMaxItems * kNaMaxTilesPerItem + 2;                 // (ntx+1)(nty+1)
constexpr size_t kNaMetaOff = kNaBsumOff + (size_t)kNaMaxBlocks * sizeof(double);      // descriptors
struct NaMeta {
    FusedTab desc;
    double* bsum_ptr[1];
    int4 items[kNaMaxItems];
    int first[2];
    float inv[1];
    unsigned long long next_item;
};
constexpr size_t kNaBytes = kNaMetaOff + ((sizeof(NaMeta) + 255) / 256) * 256;

// The scratch.  In host code this name is only a stand-in; its device
// address comes from cudaGetSymbolAddress at set-up (na_setup).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
unsigned char* g_na_base[kNaMaxDevices] = {};
int g_na_clusters[kNaMaxDevices] = {};
int g_na_shape[kNaMaxDevices] = {};

// Writes one call's descriptors into the scratch.  They travel as a kernel
// parameter (by value), so no host buffer has to outlive the call.
__global__ void k_na_meta(NaMeta m, NaMeta* dst)
{
    const int n = (int)(sizeof(NaMeta) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(&m);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
}

// Once per device, with that device current: find the scratch address and
// fill the constant taper / twiddle tables inside it.  The address is looked
// up on every call (cheap) and compared with the cached one, so a context
// that was torn down and re-created (cudaDeviceReset) is set up again.
gcf_status na_setup(int dev, unsigned char** base, int* clusters)
{
    std::lock_guard<std::mutex> lk(g_na_mutex);
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GCF_ERR_CUDA;
    if (g_na_base[dev] == static_cast<unsigned char*>(p)) {
        *base = g_na_base[dev];
        *clusters = g_na_clusters[dev];
        return GCF_OK;
    }
    g_na_base[dev] = nullptr;
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
    // the copies come from pageable memory and may return before their DMA
    // lands; the caller's stream may be non-blocking: wait for them here
    if (cudaDeviceSynchronize() != cudaSuccess) return GCF_ERR_CUDA;
    int n = 0, shape = 0;
    if (fused_max_clusters(&n, &shape) != cudaSuccess || n <= 0) return GCF_ERR_CUDA;
    g_na_base[dev] = b;
    g_na_clusters[dev] = n;
    g_na_shape[dev] = shape;
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
    double* bsum = reinterpret_cast<double*>(base + kNaBsumOff);
    meta.desc.img = dev_img;
    meta.desc.bsum = bsum;
    meta.desc.pitch = pitch;
    meta.desc.ntx = ntx;
    meta.desc.nty = nty;
    meta.desc.offx = (width - ntx * FT + (ntx - 1) * ov) / 2;
    meta.desc.offy = (height - nty * FT + (nty - 1) * ov) / 2;
    meta.desc.stride = stride;
    meta.desc.vec = ((meta.desc.offx % 2) == 0 && (stride % 2) == 0 && (pitch % 2) == 0 &&
                     ((uintptr_t)dev_img % 8) == 0) ? 2 : 1;
    meta.desc.nbx = ntx + 1;
    meta.bsum_ptr[0] = bsum;
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
    k_na_meta<<<1, 128, 0, st>>>(meta, dmeta);
    if (cudaGetLastError() != cudaSuccess) return GCF_ERR_CUDA;
    int ncl = clusters < nitems ? clusters : nitems;
    cudaError_t e = launch_fused(&dmeta->desc, dmeta->bsum_ptr, (ntx + 1) * (nty + 1), dmeta->items,
                                 nitems, dmeta->first, dmeta->inv, 0, 1,
                                 reinterpret_cast<const float*>(base + kNaTaperOff),
                                 reinterpret_cast<const float2*>(base + kNaTwOff),
                                 reinterpret_cast<float*>(base), dev_raw_out, &dmeta->next_item, ncl,
                                 g_na_shape[dev], st, nullptr, nullptr);
    if (e != cudaSuccess) return GCF_ERR_CUDA;
    return GCF_OK;
}
