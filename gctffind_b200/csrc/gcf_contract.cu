// gcf_contract.cu -- operands of the BF16 candidate contraction.
//
// The reference scores every defocus / astigmatism candidate against every
// in-band pixel of one spectrum (GCalcCTF2D + GCC2D per candidate,
// FindCTF/GCalcCTF2D.cu:15-38, FindCTF/GCC2D.cu:13-99, driven by
// FindCTF/CFindDefocus2D.cpp:153-380).  The model at pixel (s, theta) is
//   C = (|sin(phi + pi lambda s^2 (z(theta) - lambda^2 s^2 Cs / 2))| - 1/2) env(s)
// with z(theta) = mean + sigma cos 2(theta - alpha): for a fixed angle it is
// a function of (s^2, z) only.  So on a common polar grid -- ns bins in s^2
// (physical units, shared by micrographs of any pixel size), nth angle bins
// -- the correlation numerator of every candidate of every micrograph is
//   sum_t  P[z(theta_t)][t],   P[z][(j, t)] = sum_k A[z][k] B[(j, t)][k],
// one dense product of the model rows A (defocus grid x s^2 bins, shared by
// the whole batch) with the binned spectra B (micrograph x angle bin rows):
// the tcgen05 contraction of gcf_umma.cu.  The normaliser sum C^2 comes from
// the same product of A^2 with the per-micrograph pixel counts E.
//
// This file makes A, A2 (once per grid and optics), B, E and ss (per batch)
// and plans which row tiles of P each column block needs.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <math.h>

#include "gcf_internal.h"

namespace gcf {

namespace {

constexpr double kPiD = 3.14159265358979323846;

// A[i][k], A2[i][k]: model rows in double, rounded to BF16 once.
__global__ void k_polar_model(PolarGrid g, __nv_bfloat16* __restrict__ A, __nv_bfloat16* __restrict__ A2)
{
    const int i = blockIdx.x;
    const double z = (double)g.z0 + (double)i * g.dz;
    const double wl = g.wl, cs = g.cs;
    for (int k = threadIdx.x; k < g.ns; k += blockDim.x) {
        const double s2 = (double)g.s2_lo + ((double)k + 0.5) * g.ds2;
        // chi / pi in turns: lambda s^2 z - lambda^3 s^4 Cs / 2 + phi / pi
        const double t = wl * s2 * z - 0.5 * wl * wl * wl * s2 * s2 * cs + (double)g.amp_phase / kPiD;
        const double r = t - rint(t);
        const double h = fabs(sin(kPiD * r)) - 0.5;
        A[(size_t)i * g.ns + k] = __double2bfloat16(h);
        A2[(size_t)i * g.ns + k] = __double2bfloat16(h * h);
    }
}

// One CTA per job: the job's background-removed half spectrum (tile/2+1
// columns x tile rows, DC at (0, tile/2)) summed into (s^2, angle) cells in
// shared memory [t][k], then written as envelope-weighted BF16 rows.  One
// warp per row over the row's in-band columns.
__global__ void __launch_bounds__(1024)
k_polar_bin(const float* __restrict__ ctf, int tile, const SearchJob* __restrict__ jobs, PolarGrid g,
            __nv_bfloat16* __restrict__ B, __nv_bfloat16* __restrict__ E, double* __restrict__ ss)
{
    extern __shared__ float sm[];
    float* cell = sm;                         // [nth][ns]
    int* cnt = reinterpret_cast<int*>(sm + (size_t)g.nth * g.ns);   // [ns]
    __shared__ double s_red[32];
    const int j = blockIdx.x;
    const int cx = tile / 2 + 1, cy = tile;
    const float px = jobs[j].o.px;
    const float* S = ctf + (size_t)jobs[j].mic * cx * cy;
    for (int i = threadIdx.x; i < g.nth * g.ns; i += blockDim.x) cell[i] = 0.0f;
    for (int i = threadIdx.x; i < g.ns; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const float inv_px2 = 1.0f / (px * px);
    const float s2_hi = g.s2_lo + g.ns * g.ds2;
    const float th_scale = (float)g.nth / (float)kPiD;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    double acc = 0.0;
    // one warp per row, over the row's columns whose s^2 can be in the band
    // (one column of slack each side; the exact test below decides)
    for (int y = warp; y < cy; y += nwarps) {
        const float fy = (float)(y - cy / 2) / (float)tile;
        const float alo = g.s2_lo * px * px - fy * fy, ahi = s2_hi * px * px - fy * fy;
        const int xlo = alo > 0.0f ? max((int)(sqrtf(alo) * (float)tile) - 1, 0) : 0;
        const int xhi = min(ahi > 0.0f ? (int)(sqrtf(ahi) * (float)tile) + 2 : 2, cx);
        for (int x0 = xlo; x0 < xhi; x0 += 32) {
            const int x = x0 + lane;
            const float fx = (float)x / (float)tile;
            const float s2 = (fx * fx + fy * fy) * inv_px2;
            const bool in = x < xhi && s2 >= g.s2_lo && s2 < s2_hi;
            int k = -1;
            if (in) {
                k = min(max((int)((s2 - g.s2_lo) / g.ds2), 0), g.ns - 1);
                // angle from +x towards +y (row index), the convention of
                // GCalcCTF2D (FindCTF/GCalcCTF2D.cu:20-27): [-90, 90] degrees
                const float th = atan2f(fy, fx);
                int t = (int)((th + 0.5f * (float)kPiD) * th_scale);
                t = min(max(t, 0), g.nth - 1);
                const float v = S[(size_t)y * cx + x];
                atomicAdd(&cell[t * g.ns + k], v);
                acc += (double)v * v;
            }
            // the s^2 counts: one atomic per run of equal bins in the warp
            const unsigned grp = __match_any_sync(0xffffffffu, k);
            if (in && lane == __ffs(grp) - 1) atomicAdd(&cnt[k], __popc(grp));
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) ss[j] = v;
    }
    // envelope of GCC2D, exp(-16 s^2) with s in 1/pixel (FindCTF/GCC2D.cu:39-41),
    // at each bin's centre for this job's pixel size
    for (int i = threadIdx.x; i < g.nth * g.ns; i += blockDim.x) {
        const int t = i / g.ns, k = i - t * g.ns;
        const float s2 = g.s2_lo + ((float)k + 0.5f) * g.ds2;
        const float env = expf(-16.0f * s2 * px * px);
        B[((size_t)j * g.nth + t) * g.ns + k] = __float2bfloat16_rn(env * cell[i]);
    }
    for (int k = threadIdx.x; k < g.ns; k += blockDim.x) {
        const float s2 = g.s2_lo + ((float)k + 0.5f) * g.ds2;
        const float env = expf(-16.0f * s2 * px * px);
        E[(size_t)j * g.ns + k] = __float2bfloat16_rn(env * env * (float)cnt[k]);
    }
}

// One thread per column block: the union of its jobs' row ranges in row
// tiles of 128.
__global__ void k_plan_tiles(const int2* __restrict__ rows, int njobs, int nth, int nz, int bn,
                             int2* __restrict__ tiles, int* __restrict__ ntiles, int max_tiles)
{
    const int jobs_per_block = bn / nth;
    const int nblocks = (njobs + jobs_per_block - 1) / jobs_per_block;
    for (int cb = blockIdx.x * blockDim.x + threadIdx.x; cb < nblocks; cb += gridDim.x * blockDim.x) {
        int lo = nz, hi = 0;
        for (int q = cb * jobs_per_block; q < min(njobs, (cb + 1) * jobs_per_block); ++q) {
            lo = min(lo, max(rows[q].x, 0));
            hi = max(hi, min(rows[q].y, nz));
        }
        if (hi <= lo) continue;
        for (int m0 = (lo / 128) * 128; m0 < hi; m0 += 128) {
            const int slot = atomicAdd(ntiles, 1);
            if (slot < max_tiles) tiles[slot] = make_int2(m0, cb * bn);
        }
    }
}

// Defocus rows each job's table search can touch: CFindCtf1D's range
// [3000, 30000] px^2 A widened by the 2D search's +-10 % in the mean and
// ratio <= 0.06 (FindCTF/CFindCtf1D.cpp:78-79, FindCTF/CFindDefocus2D.cpp:
// 110-124), or, with a learned prior, its window of +-5 search steps; both
// with 4 % more for the re-score neighbourhood and the local passes.
__global__ void k_job_rows(const SearchJob* __restrict__ jobs, int njobs, const float4* __restrict__ prior,
                           PolarGrid g, int2* __restrict__ rows)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const float px2 = jobs[j].o.px * jobs[j].o.px;
    float zlo = 3000.0f * px2 * 0.82f, zhi = 30000.0f * px2 * 1.2f;
    if (prior && prior[j].x > 0.0f) {
        const float4 p = prior[j];
        const float w = p.w > 0.0f ? p.w : 1.0f;
        const float hdf = 5.0f * w * 0.2f * p.x / 31.0f;
        const float rhi = fminf(fmaxf(p.y, 0.0f) + 5.0f * w * 0.06f / 51.0f, 0.06f);
        zlo = (p.x - hdf) * (1.0f - rhi);
        zhi = (p.x + hdf) * (1.0f + rhi);
    }
    zlo *= 0.96f;
    zhi *= 1.04f;
    int lo = (int)floorf((zlo - g.z0) / g.dz), hi = (int)ceilf((zhi - g.z0) / g.dz) + 2;
    lo = max(lo, 0);
    hi = min(hi, g.nz);
    rows[j] = make_int2(lo, max(hi, lo));
}

// Seeded uniform fill (SplitMix64 finaliser of the element index): trial
// operands of the autotuner.
__device__ __forceinline__ float hash_uniform(unsigned long long seed, size_t i)
{
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}

__global__ void k_fill_f32(float* __restrict__ p, size_t n, unsigned long long seed, float lo, float hi)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = lo + (hi - lo) * hash_uniform(seed, i);
}

__global__ void k_fill_bf16(__nv_bfloat16* __restrict__ p, size_t n, unsigned long long seed)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = __float2bfloat16_rn(2.0f * hash_uniform(seed, i) - 1.0f);
}

}  // namespace

void launch_fill_f32(float* p, size_t n, unsigned long long seed, float lo, float hi, cudaStream_t st)
{
    if (n) k_fill_f32<<<1184, 256, 0, st>>>(p, n, seed, lo, hi);
}

void launch_fill_bf16(__nv_bfloat16* p, size_t n, unsigned long long seed, cudaStream_t st)
{
    if (n) k_fill_bf16<<<1184, 256, 0, st>>>(p, n, seed);
}

void launch_polar_model(const PolarGrid& g, __nv_bfloat16* A, __nv_bfloat16* A2, cudaStream_t st)
{
    if (g.nz <= 0 || g.ns <= 0) return;
    k_polar_model<<<g.nz, 256, 0, st>>>(g, A, A2);
}

cudaError_t launch_polar_bin(const float* ctf, int tile, const SearchJob* jobs, int njobs, const PolarGrid& g,
                             __nv_bfloat16* B, __nv_bfloat16* E, double* ss, cudaStream_t st)
{
    if (njobs <= 0) return cudaSuccess;
    const size_t sm = (size_t)g.nth * g.ns * sizeof(float) + (size_t)g.ns * sizeof(int);
    cudaError_t e = cudaFuncSetAttribute(k_polar_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_polar_bin<<<njobs, 1024, sm, st>>>(ctf, tile, jobs, g, B, E, ss);
    return cudaGetLastError();
}

void launch_plan_tiles(const int2* rows, int njobs, int nth, int nz, int bn, int2* tiles, int* ntiles,
                       int max_tiles, cudaStream_t st)
{
    if (njobs <= 0) return;
    k_plan_tiles<<<1, 256, 0, st>>>(rows, njobs, nth, nz, bn, tiles, ntiles, max_tiles);
}

void launch_job_rows(const SearchJob* jobs, int njobs, const float4* prior, const PolarGrid& g, int2* rows,
                     cudaStream_t st)
{
    if (njobs <= 0) return;
    k_job_rows<<<(njobs + 127) / 128, 128, 0, st>>>(jobs, njobs, prior, g, rows);
}

}  // namespace gcf
