// ref_driver.cpp -- C entry point over the reference's own CTF path, built
// from the reference sources by oracle/ref/Makefile into
// oracle/_ref/libgcfref.so.  Test infrastructure: the parity tests and the
// reference arm of bench.py call it; the product never does.
//
// One call runs CFindSeriesCtfs::DoIt (CFindSeriesCtfs.cpp:50-92) on an
// in-memory series, exactly as CProcessMain::DoIt (CProcessMain.cpp:16-40)
// does for an input file: CRescaleImage, CFindCtf2D Do2D for the first
// package in processing order, Refine for the others (Do2D again when the
// refined score is <= 0), GenFullSpectrum, CSaveCtfResults.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <sys/time.h>
#include <unistd.h>

#include "CMainInc.h"
// CFindCtf2D keeps its CFindDefocus2D private; the driver reads that
// object's GetCtfRes() (the spectral-CC resolution, FindCTF/CFindDefocus2D.cpp:
// 65-68, 382-400), so the class is seen with its members public here.  The
// reference sources themselves are compiled unchanged.
#define private public
#include "FindCTF/CFindCTFInc.h"
#undef private
#include "MrcUtil/CMrcUtilInc.h"

#include "ref_state.h"

using namespace GCTFFind;

GrefSeries& gref_series()
{
    static GrefSeries s;
    return s;
}

namespace {
struct StdoutMute {
    int saved = -1;
    explicit StdoutMute(bool on)
    {
        if (!on) return;
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) {
            dup2(devnull, 1);
            close(devnull);
        }
    }
    ~StdoutMute()
    {
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};
}  // namespace

extern "C" {

// results: n x 5 floats (df_min, df_max, azimuth, ext_phase, score) in
// input order.  full_spectra: optional n x tile x tile floats.
// out_ctf_path: optional CSaveCtfResults output (plus <stem>_Imod.txt for a
// tilt series).  seconds: optional wall time of DoIt (images already in
// host memory).  Returns 0, or a CUDA error code.
int gref_run_series(const float* const* images, int n, int width, int height,
                    float kv, float cs_mm, float amp_contrast, float pixel_size,
                    float ext_phase_deg, float ext_phase_range, int tile, int log_spect,
                    int gpu, const int* order, const float* tilts, const char* const* names,
                    int is_tomo, float* results, float* full_spectra,
                    const char* out_ctf_path, int quiet, double* seconds)
{
    if (n <= 0 || !images || !results) return -1;
    cudaError_t e = cudaSetDevice(gpu);
    if (e != cudaSuccess) return (int)e;
    StdoutMute mute(quiet != 0);

    CInput* in = CInput::GetInstance();
    in->m_fKv = kv;
    in->m_fCs = cs_mm;
    in->m_fAmpContrast = amp_contrast;
    in->m_fPixSize = pixel_size;
    in->m_afExtPhase[0] = ext_phase_deg;
    in->m_afExtPhase[1] = ext_phase_range;
    in->m_iTileSize = tile;
    in->m_iLogSpect = log_spect;
    in->m_iGpuID = gpu;
    memset(in->m_acOutCtfFile, 0, sizeof(in->m_acOutCtfFile));
    if (out_ctf_path) snprintf(in->m_acOutCtfFile, sizeof(in->m_acOutCtfFile), "%s", out_ctf_path);

    GrefSeries& s = gref_series();
    s.n = n;
    s.width = width;
    s.height = height;
    s.is_tomo = is_tomo != 0;
    s.images = images;
    s.order = order;
    s.tilts = tilts;
    s.names = names;
    s.full_spectra = full_spectra;

    CInputFolder::GetInstance()->ReadFiles();
    CLoadImages::GetInstance()->AsyncLoad();

    timeval t0, t1;
    gettimeofday(&t0, 0);
    CFindSeriesCtfs::GetInstance()->DoIt();
    cudaDeviceSynchronize();
    gettimeofday(&t1, 0);
    if (seconds) *seconds = (t1.tv_sec - t0.tv_sec) + 1e-6 * (t1.tv_usec - t0.tv_usec);

    if (out_ctf_path) {
        CSaveCtfResults::GetInstance()->SaveCTF();
        CSaveCtfResults::GetInstance()->SaveImod();
    }
    CInputFolder* folder = CInputFolder::GetInstance();
    for (int i = 0; i < n; i++) {
        CCtfPackage* p = folder->GetPackage(i, false);
        float* r = results + 5 * (size_t)i;
        r[0] = p->m_fDfMin;
        r[1] = p->m_fDfMax;
        r[2] = p->m_fAzimuth;
        r[3] = p->m_fExtPhase;
        r[4] = p->m_fScore;
    }
    CFindSeriesCtfs::DeleteInstance();
    CLoadImages::DeleteInstance();
    CAsyncSaveImages::DeleteInstance();
    CInputFolder::DeleteInstance();
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}


// One micrograph through the same steps as CFindSeriesCtfs::mRescaleImage,
// mSetupFindCtf and mProcessFull / mProcessRefine
// (CFindSeriesCtfs.cpp:94-170), with the intermediate products read back:
//   rescaled     : optional new_w x new_h floats (CRescaleImage output)
//   raw_half     : optional tile x (tile / 2 + 1), CFindCtfBase::GetHalfSpect(raw)
//   ctf_half     : optional tile x (tile / 2 + 1), GetHalfSpect(background removed)
//   full         : optional tile x tile, GenFullSpectrum
//   refine       : null for Do2D, else the four {centre, range} pairs of
//                  CFindCtf2D::Refine (defocus mean, astig ratio, astig
//                  angle, extra phase)
//   result       : df_min, df_max, azimuth, ext_phase, score, ctf_res (A)
int gref_single(const float* image, int width, int height, float kv, float cs_mm,
                float amp_contrast, float pixel_size, float ext_phase_deg, float ext_phase_range,
                int tile, int log_spect, int gpu, const float* refine, int* new_dims,
                float* new_pixel_size, float* rescaled, float* raw_half, float* ctf_half,
                float* full, float* result, int quiet)
{
    if (!image || !result) return -1;
    cudaError_t e = cudaSetDevice(gpu);
    if (e != cudaSuccess) return (int)e;
    StdoutMute mute(quiet != 0);
    CInput* in = CInput::GetInstance();
    in->m_fKv = kv;
    in->m_fCs = cs_mm;
    in->m_fAmpContrast = amp_contrast;
    in->m_fPixSize = pixel_size;
    in->m_afExtPhase[0] = ext_phase_deg;
    in->m_afExtPhase[1] = ext_phase_range;
    in->m_iTileSize = tile;
    in->m_iLogSpect = log_spect;
    in->m_iGpuID = gpu;
    memset(in->m_acOutCtfFile, 0, sizeof(in->m_acOutCtfFile));

    size_t px = (size_t)width * height;
    float* host = new float[px];
    memcpy(host, image, px * sizeof(float));
    int raw_size[2] = {width, height};
    // heap objects, as CFindSeriesCtfs::DoIt makes them (zero-filled here)
    CRescaleImage* rescale = new CRescaleImage;
    CCTFTheory* theory = new CCTFTheory;
    CFindCtf2D* find = new CFindCtf2D;
    rescale->Setup(raw_size, pixel_size);
    rescale->DoIt(host);
    if (new_dims) {
        new_dims[0] = rescale->m_aiNewSize[0];
        new_dims[1] = rescale->m_aiNewSize[1];
    }
    if (new_pixel_size) *new_pixel_size = rescale->m_fPixSizeN;
    if (rescaled) {
        cudaMemcpy2D(rescaled, sizeof(float) * rescale->m_aiNewSize[0], rescale->GetScaledImg(),
                     sizeof(float) * rescale->m_aiPadSizeN[0], sizeof(float) * rescale->m_aiNewSize[0],
                     rescale->m_aiNewSize[1], cudaMemcpyDefault);
    }
    theory->Setup(kv, cs_mm, amp_contrast, rescale->m_fPixSizeN, 100.0f, ext_phase_deg * 0.017453f);
    find->Setup1(theory);
    find->Setup2(rescale->m_aiNewSize);
    find->GenHalfSpectrum(rescale->GetScaledImg());
    size_t half = (size_t)(tile / 2 + 1) * tile;
    if (raw_half) {
        float* h = find->GetHalfSpect(true, true);
        memcpy(raw_half, h, half * sizeof(float));
        delete[] h;
    }
    if (ctf_half) {
        float* h = find->GetHalfSpect(false, true);
        memcpy(ctf_half, h, half * sizeof(float));
        delete[] h;
    }
    if (refine) {
        float df[2] = {refine[0], refine[1]}, ast[2] = {refine[2], refine[3]};
        float ang[2] = {refine[4], refine[5]}, ph[2] = {refine[6], refine[7]};
        find->Refine(df, ast, ang, ph);
    } else {
        find->SetPhase(ext_phase_deg, ext_phase_range > 0.0f ? ext_phase_range : 0.0f);
        find->Do2D();
    }
    result[0] = find->m_fDfMin;
    result[1] = find->m_fDfMax;
    result[2] = find->m_fAstAng;
    result[3] = find->m_fExtPhase;
    result[4] = find->m_fScore;
    result[5] = find->m_pFindDefocus2D ? find->m_pFindDefocus2D->GetCtfRes() : 0.0f;
    if (full) {
        float* f = find->GenFullSpectrum();
        memcpy(full, f, (size_t)tile * tile * sizeof(float));
        delete[] f;
    }
    delete find;
    delete theory;
    delete rescale;
    delete[] host;
    cudaDeviceSynchronize();
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}


// CCTFTheory host math (FindCTF/CCTFTheory.cpp) on arrays of inputs; needs
// no GPU.  param_out: the 10 CCTFParam floats after Setup + SetDefocus.
// For k < n: evaluate / phase_shift / defocus at (freq[k], azimuth[k]);
// frequency at (phase[k], azimuth[k]); zeros[k] = CalcNthZero(k + 1,
// azimuth[k]).
void gref_ctf_theory(float kv, float cs_mm, float amp_contrast, float pixel_size, float ast_tol,
                     float ext_phase_rad, float df_min, float df_max, float azimuth_rad, int n,
                     const float* freq, const float* azimuth, const float* phase, float* evaluate,
                     float* phase_shift, float* defocus, float* frequency, float* zeros,
                     float* param_out)
{
    CCTFTheory* t = new CCTFTheory;
    t->Setup(kv, cs_mm, amp_contrast, pixel_size, ast_tol, ext_phase_rad);
    t->SetDefocus(df_min, df_max, azimuth_rad);
    for (int k = 0; k < n; ++k) {
        evaluate[k] = t->Evaluate(freq[k], azimuth[k]);
        phase_shift[k] = t->CalcPhaseShift(freq[k], azimuth[k]);
        defocus[k] = t->CalcDefocus(azimuth[k]);
        frequency[k] = t->CalcFrequency(phase[k], azimuth[k]);
        zeros[k] = t->CalcNthZero(k + 1, azimuth[k]);
    }
    CCTFParam* p = t->GetParam(false);
    float v[10] = {p->m_fWavelength, p->m_fCs,      p->m_fAmpContrast, p->m_fAmpPhaseShift,
                   p->m_fExtPhase,   p->m_fDefocusMax, p->m_fDefocusMin, p->m_fAstAzimuth,
                   p->m_fAstTol,     p->m_fPixelSize};
    memcpy(param_out, v, sizeof(v));
    delete t;
}


// CFindCtf1D::Do1D (refine_1d = 0) or Refine1D(init_df, df_range)
// (FindCTF/CFindCtf1D.cpp:49-67) on one micrograph after SetPhase;
// result: 1D defocus, extra phase, CC.
int gref_single1d(const float* image, int width, int height, float kv, float cs_mm,
                  float amp_contrast, float pixel_size, float ext_phase_deg, float ext_phase_range,
                  int tile, int log_spect, int gpu, int refine_1d, float init_df, float df_range,
                  float* result, int quiet)
{
    if (!image || !result) return -1;
    cudaError_t e = cudaSetDevice(gpu);
    if (e != cudaSuccess) return (int)e;
    StdoutMute mute(quiet != 0);
    CInput* in = CInput::GetInstance();
    in->m_fKv = kv;
    in->m_fCs = cs_mm;
    in->m_fAmpContrast = amp_contrast;
    in->m_fPixSize = pixel_size;
    in->m_afExtPhase[0] = ext_phase_deg;
    in->m_afExtPhase[1] = ext_phase_range;
    in->m_iTileSize = tile;
    in->m_iLogSpect = log_spect;
    size_t px = (size_t)width * height;
    float* host = new float[px];
    memcpy(host, image, px * sizeof(float));
    int raw_size[2] = {width, height};
    CRescaleImage* rescale = new CRescaleImage;
    CCTFTheory* theory = new CCTFTheory;
    CFindCtf1D* find = new CFindCtf1D;
    rescale->Setup(raw_size, pixel_size);
    rescale->DoIt(host);
    theory->Setup(kv, cs_mm, amp_contrast, rescale->m_fPixSizeN, 100.0f, ext_phase_deg * 0.017453f);
    find->Setup1(theory);
    find->Setup2(rescale->m_aiNewSize);
    find->GenHalfSpectrum(rescale->GetScaledImg());
    find->SetPhase(ext_phase_deg, ext_phase_range > 0.0f ? ext_phase_range : 0.0f);
    if (refine_1d) find->Refine1D(init_df, df_range);
    else find->Do1D();
    result[0] = find->m_fDfMin;
    result[1] = find->m_fExtPhase;
    result[2] = find->m_fScore;
    delete find;
    delete theory;
    delete rescale;
    delete[] host;
    cudaDeviceSynchronize();
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}


// GBackground1D (FindCTF/GBackground1D.cu): DoIt on a host 1D spectrum of
// n bins -> start and background (read back through Remove1D on zeros);
// then Remove2D on a tile x (tile/2+1) half spectrum and Remove1D on an
// m-bin spectrum (m <= n), both copied in and out.
int gref_background1d(const float* spec, int n, float* bg_out, int* start_out, const float* half_in,
                      int tile, float* half_out, const float* spec1d_in, int m, float* spec1d_out,
                      int gpu)
{
    if (!spec || n <= 0 || !bg_out || !start_out || m > n) return -1;
    cudaError_t e = cudaSetDevice(gpu);
    if (e != cudaSuccess) return (int)e;
    float* host = new float[n];
    memcpy(host, spec, n * sizeof(float));
    GBackground1D* b = new GBackground1D;
    b->DoIt(host, n);
    *start_out = b->m_iStart;
    float* d = 0;
    cudaMalloc(&d, sizeof(float) * n);
    cudaMemset(d, 0, sizeof(float) * n);
    b->Remove1D(d, n);
    cudaMemcpy(bg_out, d, sizeof(float) * n, cudaMemcpyDefault);
    for (int i = 0; i < n; ++i) bg_out[i] = 0.0f - bg_out[i];
    cudaFree(d);
    if (half_in && half_out && tile > 0) {
        size_t hn = (size_t)(tile / 2 + 1) * tile;
        cudaMalloc(&d, sizeof(float) * hn);
        cudaMemcpy(d, half_in, sizeof(float) * hn, cudaMemcpyDefault);
        int size[2] = {tile / 2 + 1, tile};
        b->Remove2D(d, size);
        cudaMemcpy(half_out, d, sizeof(float) * hn, cudaMemcpyDefault);
        cudaFree(d);
    }
    if (spec1d_in && spec1d_out && m > 0) {
        cudaMalloc(&d, sizeof(float) * m);
        cudaMemcpy(d, spec1d_in, sizeof(float) * m, cudaMemcpyDefault);
        b->Remove1D(d, m);
        cudaMemcpy(spec1d_out, d, sizeof(float) * m, cudaMemcpyDefault);
        cudaFree(d);
    }
    delete b;
    delete[] host;
    cudaDeviceSynchronize();
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
