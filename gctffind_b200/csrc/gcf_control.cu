// gcf_control.cu -- device-resident control of the CTF search.
//
// The reference drives every candidate from the host with a synchronous
// readback (FindCTF/CFindDefocus1D.cpp:76-137, FindCTF/CFindDefocus2D.cpp:153-380).
// Here the whole control flow lives on the GPU:
//   k_search1d : radial average -> 1D brute force -> 1D refine -> 2D init,
//                one CTA per Do2D job (CFindCtf1D::Do1D, FindCTF/CFindCtf1D.cpp:49-111);
//   k_eval2d   : one step of every job's line search: all pending candidates
//                against all band pixels, then (last block of each job)
//                reduce, take the first strict maximum, advance the
//                CFindDefocus2D::mIterate state machine and write the next
//                candidate set.
// The host only enqueues k_eval2d launches; no value comes back until the
// search is over.
//
// Compiled with -fmad=false: every float step/range expression is rounded
// operation by operation like the reference's host code, so candidate grids
// coincide with the reference and with the oracle.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "gcf_internal.h"

namespace gcf {

namespace {

constexpr float kD2R2D = 0.01745329f;   // FindCTF/CFindDefocus2D.cpp:11
constexpr float kD2R1D = 0.0174533f;    // FindCTF/CFindDefocus1D.cpp:11
constexpr double kPi = 3.14159265358979323846;

struct Cand {
    float ast, ang, phase, dfmean;
};

// Candidate -> (mean px, sigma*cos 2a, sigma*sin 2a, add/pi); mCorrelate +
// GCalcCTF2D::DoIt (FindCTF/CFindDefocus2D.cpp:363-380, FindCTF/GCalcCTF2D.cu:117-132).
__device__ float4 cand_params(const Cand& c, const PixOptics& o)
{
    float ph = c.phase * kD2R2D;
    float az = c.ang * kD2R2D;
    float dmin = c.dfmean * (1.0f - c.ast) / o.px;
    float dmax = c.dfmean * (1.0f + c.ast) / o.px;
    float mean = 0.5f * (dmin + dmax);
    float sig = 0.5f * (dmax - dmin);
    float add = o.amp_phase + ph;
    double a2 = 2.0 * (double)az;
    float4 q;
    q.x = mean;
    q.y = (float)((double)sig * cos(a2));
    q.z = (float)((double)sig * sin(a2));
    q.w = (float)((double)add / kPi);
    return q;
}

// rintf(t) for |t| < 2^22 with two FP32 additions, which run on the FMA
// pipe rather than the transcendental unit that the sine needs: t + 1.5*2^23
// lies in [2^23, 2^24), where floats are the integers, so the addition
// rounds t to the nearest integer (ties to even, as rintf) and the
// subtraction is exact.  The CTF phase in turns stays within a few hundred.
__device__ __forceinline__ float rint_small(float t)
{
    const float M = 12582912.0f;   // 1.5 * 2^23
    return __fsub_rn(__fadd_rn(t, M), M);
}

// sin(pi r) and cos(pi r) for |r| <= 1/2 from their Taylor series in r
// (coefficients (-1)^k pi^n / n!), truncated after r^13 and r^14: the first
// omitted terms are below (pi/2)^15/15! < 7e-10 and (pi/2)^16/16! < 7e-11,
// so the Horner evaluation's own float rounding (a few ulp) dominates.  Runs
// on the FMA pipe only.
constexpr double kPiD = 3.14159265358979323846;
constexpr double kPi2D = kPiD * kPiD;
constexpr float kS1 = (float)kPiD;
constexpr float kS3 = (float)(-kPiD * kPi2D / 6.0);
constexpr float kS5 = (float)(kPiD * kPi2D * kPi2D / 120.0);
constexpr float kS7 = (float)(-kPiD * kPi2D * kPi2D * kPi2D / 5040.0);
constexpr float kS9 = (float)(kPiD * kPi2D * kPi2D * kPi2D * kPi2D / 362880.0);
constexpr float kS11 = (float)(-kPiD * kPi2D * kPi2D * kPi2D * kPi2D * kPi2D / 39916800.0);
constexpr float kS13 = (float)(kPiD * kPi2D * kPi2D * kPi2D * kPi2D * kPi2D * kPi2D / 6227020800.0);
constexpr float kC2 = (float)(-kPi2D / 2.0);
constexpr float kC4 = (float)(kPi2D * kPi2D / 24.0);
constexpr float kC6 = (float)(-kPi2D * kPi2D * kPi2D / 720.0);
constexpr float kC8 = (float)(kPi2D * kPi2D * kPi2D * kPi2D / 40320.0);
constexpr float kC10 = (float)(-kPi2D * kPi2D * kPi2D * kPi2D * kPi2D / 3628800.0);
constexpr float kC12 = (float)(kPi2D * kPi2D * kPi2D * kPi2D * kPi2D * kPi2D / 479001600.0);
constexpr float kC14 = (float)(-kPi2D * kPi2D * kPi2D * kPi2D * kPi2D * kPi2D * kPi2D / 87178291200.0);

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// sincos_pi_half on a packed pair of arguments
__device__ __forceinline__ void sincos_pi_half2(float2 r, float2& s, float2& c)
{
    const float2 r2 = __fmul2_rn(r, r);
    float2 p = __ffma2_rn(f2(kS13), r2, f2(kS11));
    p = __ffma2_rn(p, r2, f2(kS9));
    p = __ffma2_rn(p, r2, f2(kS7));
    p = __ffma2_rn(p, r2, f2(kS5));
    p = __ffma2_rn(p, r2, f2(kS3));
    p = __ffma2_rn(p, r2, f2(kS1));
    s = __fmul2_rn(p, r);
    float2 q = __ffma2_rn(f2(kC14), r2, f2(kC12));
    q = __ffma2_rn(q, r2, f2(kC10));
    q = __ffma2_rn(q, r2, f2(kC8));
    q = __ffma2_rn(q, r2, f2(kC6));
    q = __ffma2_rn(q, r2, f2(kC4));
    q = __ffma2_rn(q, r2, f2(kC2));
    c = __ffma2_rn(q, r2, f2(1.0f));
}

__device__ __forceinline__ void sincos_pi_half(float r, float& s, float& c)
{
    const float r2 = r * r;
    float p = fmaf(kS13, r2, kS11);
    p = fmaf(p, r2, kS9);
    p = fmaf(p, r2, kS7);
    p = fmaf(p, r2, kS5);
    p = fmaf(p, r2, kS3);
    p = fmaf(p, r2, kS1);
    s = p * r;
    float q = fmaf(kC14, r2, kC12);
    q = fmaf(q, r2, kC10);
    q = fmaf(q, r2, kC8);
    q = fmaf(q, r2, kC6);
    q = fmaf(q, r2, kC4);
    q = fmaf(q, r2, kC2);
    c = fmaf(q, r2, 1.0f);
}

// Candidate i of the pending step of job J.
__device__ Cand cand_of(const SearchJob& J, int i, const float2* cval)
{
    Cand c{J.ast_ratio, J.ast_angle, J.ext_phase, J.df_mean};
    switch (J.step) {
    case STEP_CC0:
        break;
    case STEP_ASTIG: {
        int jj = i / J.gen_n1, ii = i - jj * J.gen_n1;
        c.ast = J.gen_lo + ii * J.gen_step;
        c.ang = J.gen_lo2 + jj * J.gen_step2;
        break;
    }
    case STEP_ASTMAG:
        c.ast = J.gen_lo + i * J.gen_step;
        break;
    case STEP_ASTANG:
        c.ang = J.gen_lo + i * J.gen_step;
        break;
    case STEP_DFMEAN:
        c.dfmean = J.gen_lo + i * J.gen_step;
        break;
    case STEP_PHASE:
        c.phase = cval[i].x;
        break;
    case STEP_RESCORE:   // the table's best candidates, in table order
        c.dfmean = J.rs_df[i];
        c.ast = J.rs_ast[i];
        c.ang = J.rs_ang[i];
        break;
    case STEP_LOCAL: {   // 3 x 3 x 3 grid around the current best
        const int a = i % 3 - 1, b = (i / 3) % 3 - 1, d = i / 9 - 1;
        c.dfmean = J.df_mean + (float)a * J.loc_ddf;
        c.ast = fmaxf(J.ast_ratio + (float)b * J.loc_dast, 0.0f);
        c.ang = J.ast_angle + (float)d * J.loc_dang;
        break;
    }
    default:
        break;
    }
    return c;
}

__device__ __forceinline__ float iter_scale(int i)
{
    const int iters = 20;
    return 1.0f - i * 0.5f / iters;   // FindCTF/CFindDefocus2D.cpp:167
}

// Sets the generator of J.step and returns its candidate count (0 where the
// reference returns early).  Phase candidates are compacted into cval.
__device__ int prepare_step(SearchJob& J, float2* cval)
{
    switch (J.step) {
    case STEP_CC0:
        return 1;
    case STEP_ASTIG: {   // mFindAstig, :185-199
        float tiny = (float)1e-20;
        float ar = J.ast_range[1] - J.ast_range[0];
        float gr = J.ang_range[1] - J.ang_range[0];
        if (ar < tiny && gr < tiny) return 0;
        int ns = 51, ng = 51;
        float as = ar / ns, gs = gr / ng;
        if ((double)as < 1e-5) ns = 1;
        if ((double)gs < 1e-5) ng = 1;
        if (ns == 1 && ng == 1) return 0;
        J.gen_lo = J.ast_range[0];
        J.gen_step = as;
        J.gen_n1 = ns;
        J.gen_lo2 = J.ang_range[0];
        J.gen_step2 = gs;
        J.gen_n2 = ng;
        return ns * ng;
    }
    case STEP_ASTMAG: {   // mRefineAstMag, :224-236
        float range = iter_scale(J.iter) * J.range_ast;
        if (range < (float)1e-20) return 0;
        float lo = fmaxf(J.ast_ratio - range * 0.5f, J.ast_range[0]);
        float hi = fminf(J.ast_ratio + range * 0.5f, J.ast_range[1]);
        int n = 21;
        float step = (hi - lo) / (n - 1);
        if (step < 0.001f) step = 0.001f;
        n = (int)((hi - lo) / step) / 2 * 2 + 1;
        if (n == 1) return 0;
        J.gen_lo = lo;
        J.gen_step = step;
        return n;
    }
    case STEP_ASTANG: {   // mRefineAstAng, :256-268
        float range = iter_scale(J.iter) * J.range_ang;
        if (range < (float)1e-20) return 0;
        float lo = fmaxf(J.ast_angle - range * 0.5f, J.ang_range[0]);
        float hi = fminf(J.ast_angle + range * 0.5f, J.ang_range[1]);
        int n = 51;
        float step = (hi - lo) / (n - 1);
        if (step < 1.0f) step = 1.0f;
        n = (int)((hi - lo) / step) / 2 * 2 + 1;
        if (n == 1) return 0;
        J.gen_lo = lo;
        J.gen_step = step;
        return n;
    }
    case STEP_DFMEAN: {   // mRefineDfMean, :288-301
        float range = iter_scale(J.iter) * J.range_df;
        if (range < (float)1e-30) return 0;
        int n = 31;
        float lo = fmaxf(J.df_mean - range * 0.5f, J.df_range[0]);
        float hi = fminf(J.df_mean + range * 0.5f, J.df_range[1]);
        float step = (hi - lo) / n;
        if (step < 20) step = 20.0f;
        n = (int)((hi - lo) / step) / 2 * 2 + 1;
        if (n == 1) return 0;
        J.gen_lo = lo;
        J.gen_step = step;
        return n;
    }
    case STEP_PHASE: {   // mRefinePhase, :324-347
        float range = iter_scale(J.iter) * J.phase_range[1];
        if (range < (float)1e-30) return 0;
        int n = 61;
        float step = range / n;
        if (step < 0.03f) return 0;
        if (step > 1.0f) {
            step = 1.0f;
            n = (int)(range / step);
            n = n / 2 * 2 + 1;
        }
        float pmin = J.phase_range[0] - J.phase_range[1] * 0.5f;
        float pmax = J.phase_range[0] + J.phase_range[1] * 0.5f;
        if (pmin < 0) pmin = 0.0f;
        if (pmax > 150) pmax = 150.0f;
        int k = 0;
        for (int i = 0; i < n && k < kMaxCand; ++i) {
            float ph = J.ext_phase + (i - n / 2) * step;
            if (ph < pmin || ph > pmax) continue;
            cval[k++] = make_float2(ph, 0.0f);
        }
        return k;
    }
    case STEP_RESCORE:
        return kRescore;
    case STEP_LOCAL:
        return 27;
    default:
        return 0;
    }
}

// Applies the outcome of the pending step (best CC `best` at candidate
// `bi`, best = -1e20 when the step had no candidates) and moves J.step on.
__device__ void finish_step(SearchJob& J, float best, int bi, float cc0, const float2* cval)
{
    switch (J.step) {
    case STEP_CC0:   // mIterate, :155-156
        J.cc_max = cc0;
        J.old_cc = cc0;
        J.step = STEP_ASTIG;
        return;
    case STEP_ASTIG: {   // :214-221, then mIterate :159-165
        if (bi >= 0 && best > J.cc_max) {
            Cand c = cand_of(J, bi, cval);
            J.ast_ratio = c.ast;
            J.ast_angle = c.ang;
            J.cc_max = best;
        }
        if (J.old_cc > J.cc_max) {
            J.step = STEP_DONE;
            return;
        }
        J.ext_phase = J.phase_range[0];
        J.range_df = J.df_range[1] - J.df_range[0];
        J.range_ast = J.ast_range[1] - J.ast_range[0];
        J.range_ang = J.ang_range[1] - J.ang_range[0];
        J.iter = 1;
        J.step = STEP_ASTMAG;
        return;
    }
    case STEP_ASTMAG:   // :248-253, then mIterate :171-173
        if (bi >= 0 && best > J.cc_max) {
            J.ast_ratio = cand_of(J, bi, cval).ast;
            J.cc_max = best;
        }
        if (J.old_cc > J.cc_max) {
            J.step = STEP_DONE;
            return;
        }
        J.cc_max = J.old_cc;
        J.step = STEP_ASTANG;
        return;
    case STEP_ASTANG:   // :280-285
        if (bi >= 0 && best > J.cc_max) {
            J.ast_angle = cand_of(J, bi, cval).ang;
            J.cc_max = best;
        }
        J.step = STEP_DFMEAN;
        return;
    case STEP_DFMEAN:   // :313-321
        if (bi >= 0 && best > J.cc_max) {
            J.df_mean = cand_of(J, bi, cval).dfmean;
            J.cc_max = best;
        }
        J.step = STEP_PHASE;
        return;
    case STEP_PHASE:   // :355-360
        if (bi >= 0 && best > J.cc_max) {
            J.ext_phase = cand_of(J, bi, cval).phase;
            J.cc_max = best;
        }
        J.iter += 1;
        J.step = (J.iter < 20) ? STEP_ASTMAG : STEP_DONE;
        return;
    case STEP_RESCORE:   // the best re-scored table candidate (first strict maximum)
        if (bi >= 0) {
            const Cand c = cand_of(J, bi, cval);
            J.df_mean = c.dfmean;
            J.ast_ratio = c.ast;
            J.ast_angle = c.ang;
            J.cc_max = best;
        }
        J.iter = 0;
        J.step = STEP_LOCAL;
        return;
    case STEP_LOCAL:
        if (bi >= 0 && best > J.cc_max) {
            const Cand c = cand_of(J, bi, cval);
            J.df_mean = c.dfmean;
            J.ast_ratio = c.ast;
            J.ast_angle = c.ang;
            J.cc_max = best;
        }
        J.loc_ddf *= 0.5f;
        J.loc_dast *= 0.5f;
        J.loc_dang *= 0.5f;
        J.iter += 1;
        if (J.iter >= kLocalPasses) {
            // the azimuth is defined modulo 180 degrees: report it in (-90, 90]
            if (J.ast_angle > 90.0f) J.ast_angle -= 180.0f;
            if (J.ast_angle <= -90.0f) J.ast_angle += 180.0f;
            J.step = STEP_DONE;
        }
        return;
    default:
        J.step = STEP_DONE;
        return;
    }
}

// Advance past steps without candidates; returns the pending count.
__device__ int advance(SearchJob& J, float2* cval)
{
    while (J.step != STEP_DONE) {
        int n = prepare_step(J, cval);
        if (n > 0) return n;
        finish_step(J, (float)-1e20, -1, 0.0f, cval);
    }
    return 0;
}

// Argmax with the reference's tie rule (first strict maximum in index
// order, starting from -1e20; NaN never wins).
struct ArgMax {
    float v;
    int i;
};

__device__ __forceinline__ ArgMax better(ArgMax a, ArgMax b)
{
    if (b.i < 0) return a;
    if (a.i < 0) return b;
    if (b.v > a.v) return b;
    if (a.v > b.v) return a;
    return (b.i < a.i) ? b : a;
}

__device__ ArgMax block_argmax(ArgMax m, ArgMax* sh)
{
    for (int o = 16; o > 0; o >>= 1) {
        ArgMax t;
        t.v = __shfl_xor_sync(0xffffffffu, m.v, o);
        t.i = __shfl_xor_sync(0xffffffffu, m.i, o);
        m = better(m, t);
    }
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sh[warp] = m;
    __syncthreads();
    if (warp == 0) {
        int nw = (blockDim.x + 31) >> 5;
        ArgMax t = lane < nw ? sh[lane] : ArgMax{0.0f, -1};
        for (int o = 16; o > 0; o >>= 1) {
            ArgMax u;
            u.v = __shfl_xor_sync(0xffffffffu, t.v, o);
            u.i = __shfl_xor_sync(0xffffffffu, t.i, o);
            t = better(t, u);
        }
        if (lane == 0) sh[0] = t;
    }
    __syncthreads();
    ArgMax r = sh[0];
    __syncthreads();
    return r;
}

__device__ void write_candidates(const SearchJob& J, int n, float4* cand, float2* cval)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        Cand c = cand_of(J, i, cval);
        cand[i] = cand_params(c, J.o);
    }
}

// ---------------------------------------------------------------------------
// One block finishes job j's pending line search: reduce the candidates'
// partial sums in chunk order, take the first strict maximum, advance the
// CFindDefocus2D::mIterate state machine and write the next candidates.
__device__ void update_job(int j, SearchJob* __restrict__ jobs, const BandDev* __restrict__ bands,
                           const double* __restrict__ sum_ss, float4* __restrict__ cand,
                           float2* __restrict__ cval, const double2* __restrict__ part, int max_chunks)
{
    __shared__ SearchJob sJ;
    __shared__ ArgMax shm[32];
    __shared__ float s_cc0;
    __shared__ int s_n;
    if (threadIdx.x == 0) sJ = jobs[j];
    __syncthreads();
    if (sJ.step == STEP_DONE) return;
    float4* cj = cand + (size_t)j * kMaxCand;
    float2* vj = cval + (size_t)j * kMaxCand;
    const int n = sJ.ncand;
    const BandDev b = bands[sJ.band];
    const int nch = (b.n + kEvalChunk - 1) / kEvalChunk;
    const double ss = sum_ss[j];
    ArgMax m{(float)-1e20, -1};
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        const double2* p = part + ((size_t)j * kMaxCand + c) * max_chunks;
        double cs = 0.0, cc = 0.0;
        for (int k = 0; k < nch; ++k) {
            double2 v = p[k];
            cs += v.x;
            cc += v.y;
        }
        double d = sqrt(cc * ss);
        float ccv = (d == 0.0) ? 0.0f : (float)(cs / d);   // GCC2D mGCalc1D, FindCTF/GCC2D.cu:81-87
        if (c == 0) s_cc0 = ccv;
        if (ccv > m.v) m = ArgMax{ccv, c};   // strict, in index order per thread
    }
    __syncthreads();
    m = block_argmax(m, shm);
    if (threadIdx.x == 0) {
        sJ.n_cand2d += n;
        finish_step(sJ, m.i >= 0 ? m.v : (float)-1e20, m.i, s_cc0, vj);
        s_n = advance(sJ, vj);
        sJ.ncand = s_n;
        jobs[j] = sJ;
    }
    __syncthreads();
    write_candidates(sJ, s_n, cj, vj);
}

// Fresh jobs: the pending step is CC0 with one candidate (Do2D jobs were
// set up by k_search1d; 1D-only jobs have nothing to search).
__global__ void k_init_jobs(SearchJob* __restrict__ jobs, float4* __restrict__ cand, float2* __restrict__ cval)
{
    __shared__ SearchJob sJ;
    __shared__ int s_n;
    const int j = blockIdx.x;
    if (threadIdx.x == 0) sJ = jobs[j];
    __syncthreads();
    if (sJ.mode >= 2) return;
    float4* cj = cand + (size_t)j * kMaxCand;
    float2* vj = cval + (size_t)j * kMaxCand;
    if (threadIdx.x == 0) {
        sJ.step = STEP_CC0;
        s_n = advance(sJ, vj);
        sJ.ncand = s_n;
        jobs[j] = sJ;
    }
    __syncthreads();
    write_candidates(sJ, s_n, cj, vj);
}

// ---------------------------------------------------------------------------
// Candidate x band-pixel correlation (GCalcCTF2D + GCC2D fused,
// FindCTF/GCalcCTF2D.cu:15-38, FindCTF/GCC2D.cu:13-170).
//
// For every job the pending line search holds up to kMaxCand candidates,
// each reduced to four numbers
//   q = (mean defocus [px], sigma*cos(2 alpha), sigma*sin(2 alpha), phase/pi)
// and every in-band pixel to five
//   a = wl*s^2, d = -0.5*wl^3*s^4*Cs, env = exp(-16 s^2), cos(2 theta), sin(2 theta)
// so that the model at one (candidate, pixel) pair is
//   t   = a * (mean + sigma*cos(2(theta - alpha))) + d + phase/pi   (= chi/pi)
//   C   = (|sin(pi * (t - rint(t)))| - 1/2) * env
// and the kernel accumulates sum(C*S) and sum(C*C); sum(S*S) is per job.
// The argument of the fast sine stays within [-pi/2, pi/2].
//
// Grid: x = band chunk (kEvalChunk pixels), y = candidate block (kEvalCB
// candidates, strided), z = job.  Pixel data stay in registers; candidate
// parameters come from shared memory; partial sums leave as FP64, one slot
// per (candidate, chunk).  The last block of a job to finish (an arrival
// counter, no waiting) runs update_job for it, so one launch is one step of
// every job's search.  No expression here is contracted differently by
// -fmad=false: every multiply-add is an explicit fmaf.  Three CTAs per SM
// (80 registers, 6 pixels per thread) measured faster than two at 8 pixels
// per thread: more warps hide the sine's latency better than more
// independent pixels per warp do.
__global__ void __launch_bounds__(kEvalThreads, 3)
k_eval2d(SearchJob* __restrict__ jobs, const BandDev* __restrict__ bands, const float* __restrict__ band_spec,
         const int* __restrict__ spec_off, const double* __restrict__ sum_ss, float4* __restrict__ cand,
         float2* __restrict__ cval, double2* __restrict__ part, int max_chunks, int* __restrict__ arrive)
{
    __shared__ float4 sq[kEvalCB];
    __shared__ float red[kEvalThreads / 32][2 * kEvalCB];
    __shared__ int s_last;
    const int j = blockIdx.z;
    const int ncand = jobs[j].ncand;
    const int cand_blocks = (ncand + kEvalCB - 1) / kEvalCB;
    if ((int)blockIdx.y >= cand_blocks) return;
    // steps whose candidates move one parameter by a fixed step: the mean
    // defocus, the astigmatism magnitude or the phase (in candidate order),
    // and the single candidate of CC0
    const int kind = jobs[j].step;
    const bool linear = kind == STEP_CC0 || kind == STEP_ASTMAG || kind == STEP_DFMEAN || kind == STEP_PHASE;
    const BandDev b = bands[jobs[j].band];
    const int nchunk = (b.n + kEvalChunk - 1) / kEvalChunk;
    const int p0 = blockIdx.x * kEvalChunk;
    if ((int)blockIdx.x >= max(nchunk, 1)) return;
    const float* S = band_spec + spec_off[j];
    // per pixel: a, d, envelope and -envelope/2, cos 2theta, sin 2theta, spectrum
    float pa[kEvalPPT], pd[kEvalPPT], pe[kEvalPPT], ph[kEvalPPT], pc[kEvalPPT], ps[kEvalPPT], pv[kEvalPPT];
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
        ph[k] = -0.5f * pe[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // candidate blocks y, y + gridDim.y, ... so any candidate count is covered
    for (int c0 = blockIdx.y * kEvalCB; c0 < ncand && nchunk > 0; c0 += gridDim.y * kEvalCB) {
        __syncthreads();
        if (threadIdx.x < kEvalCB) {
            int c = c0 + threadIdx.x;
            sq[threadIdx.x] =
                c < ncand ? cand[(size_t)j * kMaxCand + c] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();
        float acs[kEvalCB], acc[kEvalCB];
        if (linear) {
            // The block's candidates step one parameter evenly, so t is
            // t0 + i * dt at every pixel (dt from the block's end points) and
            // sin(pi t_i) follows from sin and cos of pi t0 and pi dt by
            // rotation: 4 FMA-pipe operations per pair instead of a sine.
            // Two chains, seeded at candidates 0 and 8, advance as one
            // packed f32x2 pair (7 rotations each instead of 15).  All
            // angles are reduced to [-pi/2, pi/2] first; shifting dt by an
            // integer m flips the sign of sin(pi t_i) for odd i * m only,
            // which |sin| ignores.
            const int nb = min(kEvalCB, ncand - c0);
            const float4 q0 = sq[0];
            float4 dq = make_float4(0.f, 0.f, 0.f, 0.f);
            if (nb > 1) {
                const float4 q1 = sq[nb - 1];
                const float inv = 1.0f / (float)(nb - 1);
                dq = make_float4((q1.x - q0.x) * inv, (q1.y - q0.y) * inv, (q1.z - q0.z) * inv,
                                 (q1.w - q0.w) * inv);
            }
            constexpr int H = kEvalCB / 2;
            float2 as2[H], ac2[H];
#pragma unroll
            for (int c = 0; c < H; ++c) {
                as2[c] = f2(0.f);
                ac2[c] = f2(0.f);
            }
#pragma unroll
            for (int k = 0; k < kEvalPPT; ++k) {
                float df = fmaf(ps[k], q0.z, fmaf(pc[k], q0.y, q0.x));
                float t = fmaf(pa[k], df, pd[k]) + q0.w;
                float dt = fmaf(pa[k], fmaf(ps[k], dq.z, fmaf(pc[k], dq.y, dq.x)), dq.w);
                float t8 = fmaf((float)H, dt, t);
                float2 s2, c2;
                sincos_pi_half2(make_float2(t - rint_small(t), t8 - rint_small(t8)), s2, c2);
                float sd, cd;
                sincos_pi_half(dt - rint_small(dt), sd, cd);
                const float2 cd2 = f2(cd), sd2 = f2(sd), nsd2 = f2(-sd);
                const float2 e2 = f2(pe[k]), h2 = f2(ph[k]), v2 = f2(pv[k]);
#pragma unroll
                for (int c = 0; c < H; ++c) {
                    float2 C = __ffma2_rn(make_float2(fabsf(s2.x), fabsf(s2.y)), e2, h2);
                    as2[c] = __ffma2_rn(C, v2, as2[c]);
                    ac2[c] = __ffma2_rn(C, C, ac2[c]);
                    float2 sn = __ffma2_rn(s2, cd2, __fmul2_rn(c2, sd2));
                    c2 = __ffma2_rn(c2, cd2, __fmul2_rn(s2, nsd2));
                    s2 = sn;
                }
            }
#pragma unroll
            for (int c = 0; c < H; ++c) {
                acs[c] = as2[c].x;
                acs[c + H] = as2[c].y;
                acc[c] = ac2[c].x;
                acc[c + H] = ac2[c].y;
            }
        } else {
#pragma unroll
        for (int c = 0; c < kEvalCB; ++c) {
            const float4 q = sq[c];
            float s_cs = 0.f, s_cc = 0.f;
#pragma unroll
            for (int k = 0; k < kEvalPPT; ++k) {
                float df = fmaf(ps[k], q.z, fmaf(pc[k], q.y, q.x));
                float t = fmaf(pa[k], df, pd[k]) + q.w;
                float r = t - rint_small(t);
                float sv = __sinf(r * 3.14159265358979f);
                float C = fmaf(fabsf(sv), pe[k], ph[k]);   // (|sin| - 1/2) * env
                s_cs = fmaf(C, pv[k], s_cs);
                s_cc = fmaf(C, C, s_cc);
            }
            acs[c] = s_cs;
            acc[c] = s_cc;
        }
        }
        // warp sums of the 2 * kEvalCB values by recursive halving: at each
        // stage a lane keeps the half of its values selected by one lane bit
        // and adds the partner's copy of that half, so lane l ends with the
        // warp total of value l (31 shuffles instead of 5 per value)
        static_assert(2 * kEvalCB == 32, "one value per lane");
        float v[32];
#pragma unroll
        for (int c = 0; c < kEvalCB; ++c) {
            v[2 * c] = acs[c];
            v[2 * c + 1] = acc[c];
        }
#pragma unroll
        for (int h = 16; h > 0; h >>= 1) {
            const bool up = (lane & h) != 0;
#pragma unroll
            for (int i = 0; i < h; ++i) {
                float send = up ? v[i] : v[i + h];
                float keep = up ? v[i + h] : v[i];
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
            }
        }
        red[warp][lane] = v[0];
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
    // arrival: the last working block of job j finishes its step
    const int expected = max(nchunk, 1) * min((int)gridDim.y, cand_blocks);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(arrive + j, 1) == expected - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) arrive[j] = 0;
    update_job(j, jobs, bands, sum_ss, cand, cval, part, max_chunks);
}

// ---------------------------------------------------------------------------
// 1D search.  Bin data of GCalcCTF1D/GCC1D (FindCTF/GCalcCTF1D.cu:17-33,
// FindCTF/GCC1D.cu:15-65) in the same turns formulation as the 2D kernel.
struct Bins1D {
    float a[kMax1DBins], d[kMax1DBins], env[kMax1DBins], s[kMax1DBins];
};

struct Brute {
    float df, ph, cc;
    int n;   // grid points evaluated
};

__device__ Brute brute_1d(const Bins1D& B, int lo_bin, int hi_bin, double ss, const PixOptics& o,
                          const float dfr[2], const float phr[2], ArgMax* shm)
{
    // CFindDefocus1D::mBrutalForceSearch (FindCTF/CFindDefocus1D.cpp:76-119)
    int ndf = 501;
    float dfrange = dfr[1] - dfr[0];
    float dfs = dfrange / (ndf - 1);
    if (dfs < 10) dfs = 10.0f;
    ndf = (int)(dfrange / dfs) / 2 * 2 + 1;
    int nps = 37;
    float psr = phr[1] - phr[0];
    float pss = psr / (nps - 1);
    if (pss == 0) nps = 1;
    else nps = (int)(psr / pss) / 2 * 2 + 1;
    int npts = ndf * nps;
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    ArgMax m{(float)-1e20, -1};
    for (int i = warp; i < npts; i += nw) {
        int f = i % ndf, p = i / ndf;
        float df = dfr[0] + f * dfs;
        float ph = phr[0] + p * pss;
        if (ph < 0) ph = 0.0f;
        else if (ph > 150.0f) ph = 150.0f;
        float pdf = df / o.px;
        float add = o.amp_phase + ph * kD2R1D;
        float tw = (float)((double)add / kPi);
        float cs = 0.f, cc = 0.f;
        for (int x = lo_bin + lane; x < hi_bin; x += 32) {
            float t = B.a[x] * pdf + B.d[x] + tw;
            float r = t - rint_small(t);
            float sv = __sinf(r * 3.14159265358979f);
            float C = (fabsf(sv) - 0.5f) * B.env[x];
            cs += C * B.s[x];
            cc += C * C;
        }
        double dcs = cs, dcc = cc;
        for (int o2 = 16; o2 > 0; o2 >>= 1) {
            dcs += __shfl_xor_sync(0xffffffffu, dcs, o2);
            dcc += __shfl_xor_sync(0xffffffffu, dcc, o2);
        }
        float v = (dcc > 0 && ss > 0) ? (float)(dcs / sqrt(dcc * ss)) : 0.0f;
        if (v > m.v) m = ArgMax{v, i};
    }
    __syncthreads();
    m = block_argmax(m, shm);
    Brute r{0.0f, 0.0f, (float)-1e20, npts};
    if (m.i >= 0) {
        int f = m.i % ndf, p = m.i / ndf;
        float ph = phr[0] + p * pss;
        if (ph < 0) ph = 0.0f;
        else if (ph > 150.0f) ph = 150.0f;
        r.df = dfr[0] + f * dfs;
        r.ph = ph;
        r.cc = m.v;
    }
    return r;
}

__global__ void k_search1d(SearchJob* __restrict__ jobs, const float* __restrict__ radial, int cx,
                           float4* __restrict__ cand, float2* __restrict__ cval)
{
    extern __shared__ unsigned char smem_raw[];
    Bins1D& B = *reinterpret_cast<Bins1D*>(smem_raw);
    __shared__ ArgMax shm[32];
    __shared__ double s_ss;
    __shared__ SearchJob sJ;
    const int j = blockIdx.x;
    if (threadIdx.x == 0) sJ = jobs[j];
    __syncthreads();
    if (sJ.mode == 1 || sJ.mode == 4) return;   // Refine and the contraction search have no 1D stage here
    const PixOptics o = sJ.o;
    const float* rad = radial + (size_t)sJ.mic * cx;
    // CFindDefocus1D::mCorrelate band (FindCTF/CFindDefocus1D.cpp:128-137)
    float r0 = 25.0f * o.px, r1 = (2.0f * o.px) / 0.8f;
    if (r1 < 3.5f) r1 = 3.5f;
    float res1 = ((cx - 1) * 2) * o.px;
    float flo = res1 / r0, fhi = res1 / r1;
    int lo_bin = cx, hi_bin = 0;
    for (int x = 0; x < cx; ++x) {
        if ((float)x >= flo && (float)x < fhi) {
            if (x < lo_bin) lo_bin = x;
            hi_bin = x + 1;
        }
    }
    for (int x = threadIdx.x; x < cx; x += blockDim.x) {
        double s = (x * 0.5) / (cx - 1.0);
        double s2 = s * s;
        double f = x / (cx - 1.0);
        B.a[x] = (float)((double)o.wl * s2);
        B.d[x] = (float)(-0.5 * (double)o.wl * o.wl * o.wl * s2 * s2 * o.cs);
        B.env[x] = (float)exp(-f * f);
        B.s[x] = rad[x];
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        double ss = 0.0;
        for (int x = lo_bin + (int)threadIdx.x; x < hi_bin; x += 32) ss += (double)B.s[x] * B.s[x];
        for (int o2 = 16; o2 > 0; o2 >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o2);
        if (threadIdx.x == 0) s_ss = ss;
    }
    __syncthreads();
    const double ss = s_ss;
    // CFindCtf1D::mFindDefocus (FindCTF/CFindCtf1D.cpp:73-90)
    float ext = sJ.ext_phase_in, prange = sJ.phase_range_in;
    float px2 = o.px * o.px;
    Brute b1;
    float range;
    if (sJ.mode == 3) {
        // CFindCtf1D::Refine1D (FindCTF/CFindCtf1D.cpp:58-67): refine pass only,
        // around the given defocus and the current extra phase
        b1 = Brute{sJ.r1d_df, ext, 0.0f, 0};
        range = sJ.r1d_range;
    } else {
        float dfr[2] = {3000.0f * px2, 30000.0f * px2};
        float phr[2];
        phr[0] = fmaxf(ext - prange / 2, 0.0f);
        phr[1] = fminf(phr[0] + prange, 150.0f);
        b1 = brute_1d(B, lo_bin, hi_bin, ss, o, dfr, phr, shm);
        range = fmaxf(0.3f * b1.df, 3000.0f);   // CFindCtf1D::Do1D (FindCTF/CFindCtf1D.cpp:49-56)
    }
    // CFindCtf1D::mRefineDefocus (FindCTF/CFindCtf1D.cpp:92-111)
    float mindf = 3000.0f * o.px * o.px;
    float dfr2[2];
    dfr2[0] = fmaxf(b1.df - range / 2, mindf);
    dfr2[1] = dfr2[0] + range;
    float pr = 0.2f * prange;
    float phr2[2];
    phr2[0] = fmaxf(b1.ph - pr / 2, 0.0f);
    phr2[1] = fminf(0.0f + pr, 150.0f);   // the reference reads the zero-initialised bound
    Brute b2 = brute_1d(B, lo_bin, hi_bin, ss, o, dfr2, phr2, shm);
    if (threadIdx.x == 0) {
        sJ.n_cand1d += b1.n + b2.n;
        sJ.n_pairs1d += (b1.n + b2.n) * max(hi_bin - lo_bin, 0);
    }
    if (sJ.mode >= 2) {   // Do1D / Refine1D alone: no 2D search follows
        if (threadIdx.x == 0) {
            sJ.df_1d = b2.df;
            sJ.phase_1d = b2.ph;
            sJ.score_1d = b2.cc;
            sJ.step = STEP_DONE;
            sJ.ncand = 0;
            jobs[j] = sJ;
        }
        return;
    }
    float2* vj = cval + (size_t)j * kMaxCand;
    __shared__ int s_n;
    if (threadIdx.x == 0) {
        sJ.df_1d = b2.df;
        sJ.phase_1d = b2.ph;
        sJ.score_1d = b2.cc;
        // CFindCtf2D::Do2D + CFindDefocus2D::Setup3/DoIt (FindCTF/CFindCtf2D.cpp:44-53,
        // FindCTF/CFindDefocus2D.cpp:98-124)
        float mu = (b2.df + b2.df) * 0.5f;
        sJ.df_mean = mu;
        sJ.ast_ratio = 0.0f;
        sJ.ast_angle = 0.0f;
        sJ.phase_range[0] = b2.ph;
        sJ.phase_range[1] = prange;
        sJ.ext_phase = sJ.held_phase;   // replaced by phase_range[0] after the astigmatism grid
        sJ.df_range[0] = mu * 0.9f;
        sJ.df_range[1] = mu * 1.1f;
        sJ.ast_range[0] = 0.0f;
        sJ.ast_range[1] = 0.06f;
        sJ.ang_range[0] = -90.0f;
        sJ.ang_range[1] = 90.0f;
        sJ.step = STEP_CC0;
        s_n = advance(sJ, vj);
        sJ.ncand = s_n;
        jobs[j] = sJ;
    }
    __syncthreads();
    write_candidates(sJ, s_n, cand + (size_t)j * kMaxCand, vj);
}

// Shell choice of GSpectralCC2D::DoIt (FindCTF/GSpectralCC2D.cu:144-172) and
// CFindDefocus2D::mCalcCtfRes (FindCTF/CFindDefocus2D.cpp:382-400).
__global__ void k_shell_select(SearchJob* __restrict__ jobs, int njobs, const float* __restrict__ cc,
                               int cx, int cy)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const float* c = cc + (size_t)j * cx;
    int imax = 1;
    float fmx = (float)-1e30;
    for (int i = 1; i < cx; ++i) {
        if (c[i] <= fmx) continue;
        fmx = c[i];
        imax = i;
    }
    int shell = imax;
    if (!(fmx < 0.143f)) {
        for (int i = imax; i < cx; ++i) {
            if (c[i] < 0.143f) break;
            shell = i;
        }
    }
    jobs[j].ctf_res = cy * jobs[j].o.px / shell;
}

// CFindCtf2D::mGetResults (FindCTF/CFindCtf2D.cpp:68-76) and the getters
// of CFindDefocus2D (FindCTF/CFindDefocus2D.cpp:38-68).
__global__ void k_results(const SearchJob* __restrict__ jobs, int njobs, const int* __restrict__ lowpassed,
                          gcf_result* __restrict__ out, int* __restrict__ counts)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const SearchJob& J = jobs[j];
    if (counts) {
        counts[3 * j] = J.n_cand2d;
        counts[3 * j + 1] = J.n_cand1d;
        counts[3 * j + 2] = J.n_pairs1d;
    }
    gcf_result r;
    if (J.mode == 2 || J.mode == 3) {   // CFindCtf1D results: m_fDfMin = m_fDfMax = 1D defocus
        r.df_min = J.df_1d;
        r.df_max = J.df_1d;
        r.azimuth = 0.0f;
        r.ext_phase = J.phase_1d;
        r.score = J.score_1d;
        r.ctf_res = 0.0f;
        r.df_1d = J.df_1d;
        r.phase_1d = J.phase_1d;
        r.score_1d = J.score_1d;
        r.lowpassed = lowpassed ? lowpassed[J.mic] : 0;
        out[j] = r;
        return;
    }
    r.df_min = J.df_mean * (1.0f - J.ast_ratio);
    r.df_max = J.df_mean * (1.0f + J.ast_ratio);
    r.azimuth = J.ast_angle;
    r.ext_phase = J.ext_phase;
    r.score = J.cc_max;
    r.ctf_res = J.ctf_res;
    r.df_1d = (J.mode == 0 || J.mode == 4) ? J.df_1d : 0.0f;
    r.phase_1d = (J.mode == 0 || J.mode == 4) ? J.phase_1d : 0.0f;
    r.score_1d = (J.mode == 0 || J.mode == 4) ? J.score_1d : 0.0f;
    r.lowpassed = lowpassed ? lowpassed[J.mic] : 0;
    out[j] = r;
}

// ---------------------------------------------------------------------------
// Search on the contraction's table (mode 4).  The table P[z][(j, t)] holds,
// for micrograph j, angle bin t and defocus row z, the correlation numerator
// of the model with defocus z over that angle bin; Dz[z][j] the normaliser
// sum C^2 over the whole band at defocus z.  A candidate (mean, ratio,
// angle) then costs nth interpolated reads instead of a pass over the band:
//   num = sum_t P[mean (1 + ratio cos 2(theta_t - angle))][t]
//   den = (1/nth) sum_t Dz[same row],     CC = num / sqrt(den * sum S^2).
// One CTA per job runs, on this evaluator, the reference's own control flow:
// a 1D scan over the defocus rows of CFindCtf1D's range (FindCTF/
// CFindCtf1D.cpp:73-90) -- or, with a learned prior, a window around it --
// then CFindDefocus2D::mIterate (FindCTF/CFindDefocus2D.cpp:153-183) through
// the same prepare_step / finish_step state machine as the FP32 search.  Its
// best candidates go to the FP32 re-score (STEP_RESCORE) and local
// refinement (STEP_LOCAL) of k_eval2d on the job's own band.
constexpr int kTabThreads = 256;
constexpr int kTabMaxTheta = 128;

struct TabCtx {
    const float* P;    // column 0 of this job's angle bins
    long long ldp;
    const float* D;    // this job's normaliser row Dz[j][.]
    int lo, hi;        // computed rows [lo, hi)
    int nth;
    float z0, dz;
    double ss;
};

__device__ __forceinline__ float table_cc(const TabCtx& T, const float* c2, const float* s2, float mean,
                                          float ratio, float angle_deg)
{
    const float a = angle_deg * kD2R2D;
    const float ca = cosf(2.0f * a), sa = sinf(2.0f * a);
    const float sig = mean * ratio;
    const float inv_dz = 1.0f / T.dz;
    const float umax = (float)(T.hi - 1) - 1e-3f;
    float num = 0.0f, den = 0.0f;
    for (int t = 0; t < T.nth; ++t) {
        const float z = fmaf(sig, fmaf(c2[t], ca, s2[t] * sa), mean);
        float u = (z - T.z0) * inv_dz;
        u = fminf(fmaxf(u, (float)T.lo), umax);
        const int i0 = (int)u;
        const float f = u - (float)i0;
        const float p0 = __ldg(T.P + (size_t)i0 * T.ldp + t), p1 = __ldg(T.P + (size_t)(i0 + 1) * T.ldp + t);
        const float d0 = __ldg(T.D + i0), d1 = __ldg(T.D + i0 + 1);
        num += fmaf(f, p1 - p0, p0);
        den += fmaf(f, d1 - d0, d0);
    }
    const double d = (double)den / T.nth * T.ss;
    return d > 0.0 ? (float)((double)num / sqrt(d)) : 0.0f;
}

__global__ void __launch_bounds__(kTabThreads)
k_table_search(TableArgs A)
{
    __shared__ SearchJob sJ;
    __shared__ ArgMax shm[32];
    __shared__ float s_c2[kTabMaxTheta], s_s2[kTabMaxTheta];
    __shared__ float2 s_cval[kMaxCand];
    __shared__ float s_cc0;
    __shared__ int s_n;
    __shared__ float s_top[45];
    const int j = blockIdx.x, tid = threadIdx.x;
    if (tid == 0) sJ = A.jobs[j];
    const int2 rr = A.rows[j];
    TabCtx T;
    T.P = A.P + (size_t)j * A.g.nth;
    T.ldp = A.ldp;
    T.D = A.Dz + (size_t)j * A.ldd;
    T.lo = max(rr.x, 0);
    T.hi = min(rr.y, A.g.nz);
    T.nth = min(A.g.nth, kTabMaxTheta);
    T.z0 = A.g.z0;
    T.dz = A.g.dz;
    T.ss = A.ss[j];
    for (int t = tid; t < T.nth; t += blockDim.x) {
        const float th = (-90.0f + ((float)t + 0.5f) * 180.0f / (float)T.nth) * kD2R2D;
        s_c2[t] = cosf(2.0f * th);
        s_s2[t] = sinf(2.0f * th);
    }
    __syncthreads();
    if (sJ.mode != 4 || T.hi - T.lo < 2) {
        if (tid == 0 && sJ.mode == 4) {   // nothing computed for this job: no search
            sJ.step = STEP_DONE;
            sJ.ncand = 0;
            A.jobs[j] = sJ;
        }
        return;
    }
    const float4 pr = A.prior ? A.prior[j] : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool learned = pr.x > 0.0f;
    const float px2 = sJ.o.px * sJ.o.px;
    float mu;
    if (!learned) {
        // 1D: the rows of CFindCtf1D's defocus range, angle bins summed
        const int r0 = max(T.lo, (int)ceilf((3000.0f * px2 - T.z0) / T.dz));
        const int r1 = min(T.hi - 1, (int)floorf((30000.0f * px2 - T.z0) / T.dz));
        ArgMax m{(float)-1e20, -1};
        for (int i = r0 + tid; i <= r1; i += blockDim.x) {
            const float* row = T.P + (size_t)i * T.ldp;
            float num = 0.0f;
            for (int t = 0; t < T.nth; ++t) num += __ldg(row + t);
            const double d = (double)__ldg(T.D + i) * T.ss;
            const float v = d > 0.0 ? (float)((double)num / sqrt(d)) : 0.0f;
            if (v > m.v) m = ArgMax{v, i};
        }
        m = block_argmax(m, shm);
        mu = T.z0 + (float)(m.i >= 0 ? m.i : r0) * T.dz;
        if (tid == 0) {
            sJ.df_1d = mu;
            sJ.phase_1d = sJ.ext_phase_in;
            sJ.score_1d = m.v;
            sJ.n_table += max(r1 - r0 + 1, 0);
            // CFindCtf2D::Do2D ranges (FindCTF/CFindDefocus2D.cpp:110-124)
            sJ.df_mean = mu;
            sJ.ast_ratio = 0.0f;
            sJ.ast_angle = 0.0f;
            sJ.df_range[0] = mu * 0.9f;
            sJ.df_range[1] = mu * 1.1f;
            sJ.ast_range[0] = 0.0f;
            sJ.ast_range[1] = 0.06f;
            sJ.ang_range[0] = -90.0f;
            sJ.ang_range[1] = 90.0f;
        }
    } else if (tid == 0) {
        // learned prior: a window of +-5 search steps around the prediction
        // (steps of the full search: mean defocus 0.2 mu / 31, ratio 0.06 / 51,
        // angle 180 / 51 degrees), scaled by pr.w
        mu = pr.x;
        const float w = pr.w > 0.0f ? pr.w : 1.0f;
        const float hdf = 5.0f * w * 0.2f * mu / 31.0f;
        const float hast = 5.0f * w * 0.06f / 51.0f;
        const float hang = 5.0f * w * 180.0f / 51.0f;
        sJ.df_1d = mu;
        sJ.phase_1d = sJ.ext_phase_in;
        sJ.score_1d = 0.0f;
        sJ.df_mean = mu;
        sJ.ast_ratio = fminf(fmaxf(pr.y, 0.0f), 0.06f);
        sJ.ast_angle = pr.z;
        sJ.df_range[0] = mu - hdf;
        sJ.df_range[1] = mu + hdf;
        sJ.ast_range[0] = fmaxf(sJ.ast_ratio - hast, 0.0f);
        sJ.ast_range[1] = fminf(sJ.ast_ratio + hast, 0.06f);
        sJ.ang_range[0] = sJ.ast_angle - hang;
        sJ.ang_range[1] = sJ.ast_angle + hang;
    }
    if (tid == 0) {
        sJ.phase_range[0] = sJ.ext_phase_in;
        sJ.phase_range[1] = 0.0f;   // no extra-phase search on the table
        sJ.ext_phase = sJ.ext_phase_in;
        sJ.step = STEP_CC0;
    }
    __syncthreads();
    // CFindDefocus2D::mIterate on the table
    for (int guard = 0; guard < 256; ++guard) {
        if (tid == 0) s_n = advance(sJ, s_cval);
        __syncthreads();
        const int n = s_n;
        if (sJ.step == STEP_DONE || n <= 0) break;
        ArgMax m{(float)-1e20, -1};
        for (int c = tid; c < n; c += blockDim.x) {
            const Cand cd = cand_of(sJ, c, s_cval);
            const float v = table_cc(T, s_c2, s_s2, cd.dfmean, cd.ast, cd.ang);
            if (c == 0) s_cc0 = v;
            if (v > m.v) m = ArgMax{v, c};
        }
        m = block_argmax(m, shm);   // synchronises: s_cc0 is visible
        if (tid == 0) {
            sJ.n_table += n;
            finish_step(sJ, m.i >= 0 ? m.v : (float)-1e20, m.i, s_cc0, s_cval);
        }
        __syncthreads();
    }
    // the table's best candidates: a 5 x 3 x 3 neighbourhood of its optimum
    // (half a final mean-defocus step, 0.001 in ratio, 2 degrees), the top
    // kRescore go to the FP32 re-score
    const float hmu = 0.5f * fmaxf(20.0f, 0.105f * sJ.df_mean / 31.0f);
    if (tid < 45) {
        const int a = tid % 5 - 2, b = (tid / 5) % 3 - 1, d = tid / 15 - 1;
        s_top[tid] = table_cc(T, s_c2, s_s2, sJ.df_mean + (float)a * hmu,
                              fmaxf(sJ.ast_ratio + 0.001f * (float)b, 0.0f), sJ.ast_angle + 2.0f * (float)d);
    }
    __syncthreads();
    if (tid == 0) {
        sJ.n_table += 45;
        unsigned long long used = 0ull;
        for (int r = 0; r < kRescore; ++r) {
            int bi = 22;   // the optimum itself
            float bv = (float)-1e30;
            for (int q = 0; q < 45; ++q)
                if (!((used >> q) & 1ull) && s_top[q] > bv) {
                    bv = s_top[q];
                    bi = q;
                }
            used |= 1ull << bi;
            const int a = bi % 5 - 2, b = (bi / 5) % 3 - 1, d = bi / 15 - 1;
            sJ.rs_df[r] = sJ.df_mean + (float)a * hmu;
            sJ.rs_ast[r] = fmaxf(sJ.ast_ratio + 0.001f * (float)b, 0.0f);
            sJ.rs_ang[r] = sJ.ast_angle + 2.0f * (float)d;
        }
        sJ.loc_ddf = hmu;
        sJ.loc_dast = 0.001f;
        sJ.loc_dang = 1.0f;
        sJ.cc_max = (float)-1e20;
        sJ.iter = 0;
        sJ.step = STEP_RESCORE;
        s_n = advance(sJ, s_cval);
        sJ.ncand = s_n;
        A.jobs[j] = sJ;
    }
    __syncthreads();
    write_candidates(sJ, s_n, A.cand + (size_t)j * kMaxCand, A.cval + (size_t)j * kMaxCand);
}

}  // namespace

void launch_eval2d(const EvalArgs& a, int cand_blocks, int max_band_n, cudaStream_t st)
{
    if (a.njobs <= 0 || cand_blocks <= 0 || max_band_n < 0) return;
    dim3 grid(std::max(1, (max_band_n + kEvalChunk - 1) / kEvalChunk), cand_blocks, a.njobs);
    k_eval2d<<<grid, kEvalThreads, 0, st>>>(a.jobs, a.bands, a.band_spec, a.spec_off, a.sum_ss, a.cand,
                                            a.cval, a.part, a.max_chunks, a.arrive);
}

void launch_init_jobs(const EvalArgs& a, cudaStream_t st)
{
    if (a.njobs <= 0) return;
    k_init_jobs<<<a.njobs, 256, 0, st>>>(a.jobs, a.cand, a.cval);
}

void launch_search1d(SearchJob* jobs, int njobs, const float* radial, int cx, float4* cand,
                     float2* cval, cudaStream_t st)
{
    if (njobs <= 0) return;
    size_t sm = sizeof(Bins1D);   // 16.4 KB, below the default dynamic limit
    k_search1d<<<njobs, 256, sm, st>>>(jobs, radial, cx, cand, cval);
}

void launch_table_search(const TableArgs& a, cudaStream_t st)
{
    if (a.njobs <= 0) return;
    k_table_search<<<a.njobs, kTabThreads, 0, st>>>(a);
}

void launch_shell_select(SearchJob* jobs, int njobs, const float* cc, int cx, int cy,
                         cudaStream_t st)
{
    if (njobs <= 0) return;
    k_shell_select<<<(njobs + 127) / 128, 128, 0, st>>>(jobs, njobs, cc, cx, cy);
}

void launch_results(const SearchJob* jobs, int njobs, const int* lowpassed, gcf_result* out, int* counts,
                    cudaStream_t st)
{
    if (njobs <= 0) return;
    k_results<<<(njobs + 127) / 128, 128, 0, st>>>(jobs, njobs, lowpassed, out, counts);
}

}  // namespace gcf
