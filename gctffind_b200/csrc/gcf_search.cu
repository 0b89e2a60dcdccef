// gcf_search.cu -- candidate x band-pixel correlation kernel of the 2D search
// (GCalcCTF2D + GCC2D fused, FindCTF/GCalcCTF2D.cu:15-38, FindCTF/GCC2D.cu:13-170).
//
// For every job (micrograph) the pending line search holds up to kMaxCand
// candidates, each reduced to four numbers:
//   q = (mean defocus [px], sigma*cos(2 alpha), sigma*sin(2 alpha), phase/pi)
// and every in-band pixel to five:
//   a = wl*s^2, d = -0.5*wl^3*s^4*Cs, env = exp(-16 s^2), cos(2 theta), sin(2 theta)
// so that the model at one (candidate, pixel) pair is
//   t   = a * (mean + sigma*cos(2(theta - alpha))) + d + phase/pi   (= chi/pi)
//   C   = (|sin(pi * (t - rint(t)))| - 1/2) * env
// and the kernel accumulates sum(C*S) and sum(C*C); sum(S*S) is per job.
//
// Grid: x = band chunk (kEvalChunk pixels), y = candidate block (kEvalCB),
// z = job.  Pixel data stay in registers; candidate parameters come from
// shared memory; partial sums leave as FP64, one slot per (candidate, chunk),
// and the update kernel reduces them in chunk order (deterministic).
#include <cuda_runtime.h>

#include "gcf_internal.h"

namespace gcf {

namespace {

__global__ void __launch_bounds__(kEvalThreads)
k_eval2d(const SearchJob* __restrict__ jobs, const BandDev* __restrict__ bands,
         const float* __restrict__ band_spec, const int* __restrict__ spec_off,
         const float4* __restrict__ cand, double2* __restrict__ part, int max_chunks)
{
    __shared__ float4 sq[kEvalCB];
    __shared__ float red[kEvalThreads / 32][2 * kEvalCB];
    const int j = blockIdx.z;
    const int ncand = jobs[j].ncand;
    if ((int)blockIdx.y * kEvalCB >= ncand) return;
    const BandDev b = bands[jobs[j].band];
    const int p0 = blockIdx.x * kEvalChunk;
    if (p0 >= b.n) return;
    const float* S = band_spec + spec_off[j];
    float pa[kEvalPPT], pd[kEvalPPT], pe[kEvalPPT], pc[kEvalPPT], ps[kEvalPPT], pv[kEvalPPT];
#pragma unroll
    for (int k = 0; k < kEvalPPT; ++k) {
        int p = p0 + k * kEvalThreads + threadIdx.x;
        if (p < b.n) {
            pa[k] = __ldg(b.a + p);
            pd[k] = __ldg(b.d + p);
            pe[k] = __ldg(b.env + p);
            pc[k] = __ldg(b.c2t + p);
            ps[k] = __ldg(b.s2t + p);
            pv[k] = __ldg(S + p);
        } else {
            pa[k] = 0.f;
            pd[k] = 0.f;
            pe[k] = 0.f;
            pc[k] = 0.f;
            ps[k] = 0.f;
            pv[k] = 0.f;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // candidate blocks y, y + gridDim.y, ... so any candidate count is covered
    for (int c0 = blockIdx.y * kEvalCB; c0 < ncand; c0 += gridDim.y * kEvalCB) {
        __syncthreads();
        if (threadIdx.x < kEvalCB) {
            int c = c0 + threadIdx.x;
            sq[threadIdx.x] =
                c < ncand ? cand[(size_t)j * kMaxCand + c] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();
        float acs[kEvalCB], acc[kEvalCB];
#pragma unroll
        for (int c = 0; c < kEvalCB; ++c) {
            const float4 q = sq[c];
            float s_cs = 0.f, s_cc = 0.f;
#pragma unroll
            for (int k = 0; k < kEvalPPT; ++k) {
                float df = fmaf(ps[k], q.z, fmaf(pc[k], q.y, q.x));
                float t = fmaf(pa[k], df, pd[k]) + q.w;
                float r = t - rintf(t);
                float sv = __sinf(r * 3.14159265358979f);
                float C = (fabsf(sv) - 0.5f) * pe[k];
                s_cs = fmaf(C, pv[k], s_cs);
                s_cc = fmaf(C, C, s_cc);
            }
            acs[c] = s_cs;
            acc[c] = s_cc;
        }
#pragma unroll
        for (int c = 0; c < kEvalCB; ++c) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                acs[c] += __shfl_xor_sync(0xffffffffu, acs[c], o);
                acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < kEvalCB; ++c) {
                red[warp][2 * c] = acs[c];
                red[warp][2 * c + 1] = acc[c];
            }
        }
        __syncthreads();
        if (threadIdx.x < kEvalCB) {
            int c = c0 + threadIdx.x;
            if (c < ncand) {
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int w = 0; w < kEvalThreads / 32; ++w) {
                    s1 += (double)red[w][2 * threadIdx.x];
                    s2 += (double)red[w][2 * threadIdx.x + 1];
                }
                part[((size_t)j * kMaxCand + c) * max_chunks + blockIdx.x] = make_double2(s1, s2);
            }
        }
    }
}

}  // namespace

void launch_eval2d(const EvalArgs& a, int cand_blocks, int max_band_n, cudaStream_t st)
{
    if (a.njobs <= 0 || cand_blocks <= 0 || max_band_n <= 0) return;
    dim3 grid((max_band_n + kEvalChunk - 1) / kEvalChunk, cand_blocks, a.njobs);
    k_eval2d<<<grid, kEvalThreads, 0, st>>>(a.jobs, a.bands, a.band_spec, a.spec_off, a.cand,
                                            a.part, a.max_chunks);
}

}  // namespace gcf
