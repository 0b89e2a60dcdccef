// gcf_internal.h -- shared definitions of the B200 CTF-estimation library.
//
// Data layout in HBM (per context):
//   images     : dense float, width x height per micrograph (row pitch = width)
//   raw / ctf  : per micrograph a (tile/2+1) x tile float half spectrum,
//                row-major with cmpX = tile/2+1 floats per row and the DC at
//                (x = 0, y = tile/2), the layout of GCalcSpectrum
//                (FindCTF/GCalcSpectrum.cu:8-31)
//   band       : per (tile, pixel size, optics) the in-band pixels of the 2D
//                correlation as structure-of-arrays (index, a, d, envelope,
//                cos 2theta, sin 2theta) so the candidate kernel streams them
//   jobs       : one SearchJob per micrograph being searched
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gctf_b200.h"

namespace gcf {

constexpr int kMaxCand = 2624;        // >= 51 * 51 astigmatism grid
constexpr int kEvalThreads = 256;     // threads of the candidate kernel
constexpr int kEvalPPT = 6;           // band pixels per thread per chunk
constexpr int kEvalChunk = kEvalThreads * kEvalPPT;
constexpr int kEvalCB = 16;           // candidates per CTA
constexpr int kMax1DBins = 1025;      // tile <= 2048

// Search step kinds (CFindDefocus2D::mIterate, FindCTF/CFindDefocus2D.cpp:153-183)
enum StepKind : int {
    STEP_CC0 = 0,
    STEP_ASTIG = 1,
    STEP_ASTMAG = 2,
    STEP_ASTANG = 3,
    STEP_DFMEAN = 4,
    STEP_PHASE = 5,
    STEP_DONE = 6
};

// Optics in pixel units (CCTFTheory::Setup, FindCTF/CCTFTheory.cpp:69-86).
struct PixOptics {
    float wl;         // wavelength, pixels
    float cs;         // Cs, pixels
    float amp_phase;  // radian (GCalcCTF2D::SetParam, FindCTF/GCalcCTF2D.cu:99-104)
    float px;         // Angstrom / pixel
};

// Per-job search state: the members of CFindDefocus2D plus the position in
// the mIterate sequence.  Lives in device memory; the update kernel owns it.
struct SearchJob {
    // inputs
    int mic;            // spectrum slot
    int band;           // band-table slot
    int mode;           // 0 = Do2D (after the 1D search), 1 = Refine, 2 = Do1D, 3 = Refine1D
    int pad0;
    PixOptics o;
    float phase_range_in;   // CFindCtfBase::m_fPhaseRange (Do2D)
    float ext_phase_in;     // CFindCtfBase::m_fExtPhase   (Do2D)
    float res_lo, res_hi;   // 1D band, Fourier pixels [lo, hi)
    // CFindDefocus2D::m_fExtPhase as the search object holds it on entry:
    // Setup3 does not set it, and mIterate evaluates its first CC and the
    // whole astigmatism grid at this phase before replacing it with
    // m_afPhaseRange[0] (FindCTF/CFindDefocus2D.cpp:98-108,153-165).  It is 0
    // for an object that Setup1 has just created, else the phase the
    // previous search on the same object ended with.
    float held_phase;
    float r1d_df, r1d_range;   // Refine1D: initial defocus and window, Angstrom
    int pad2;
    // CFindDefocus2D state
    float df_mean, ast_ratio, ast_angle, ext_phase, cc_max, old_cc;
    float phase_range[2], df_range[2], ast_range[2], ang_range[2];
    float range_df, range_ast, range_ang;  // full ranges captured by mIterate
    int iter;
    int step;           // StepKind of the pending candidate set
    int ncand;          // candidates of the pending step
    // generator of the pending step
    float gen_lo, gen_step;
    int gen_n1, gen_n2;
    float gen_lo2, gen_step2;
    // results
    float df_1d, phase_1d, score_1d;
    float ctf_res;
    int lowpassed;
    // work done: 2D candidates evaluated (each over the whole band), 1D grid
    // points evaluated, and 1D (grid point, bin) pairs
    int n_cand2d, n_cand1d, n_pairs1d;
};

// Per-band device pointers (structure of arrays).
struct BandDev {
    int n;
    int cx, cy;
    int pad;
    const int* idx;
    const float* a;     // wl * s^2                     (turns / pixel defocus)
    const float* d;     // -0.5 * wl^3 * s^4 * Cs       (turns)
    const float* env;   // exp(-16 s^2)
    const float* c2t;   // cos(2 theta)
    const float* s2t;   // sin(2 theta)
};

// Arguments of the 2D candidate kernels.
struct EvalArgs {
    SearchJob* jobs;
    const BandDev* bands;
    const float* band_spec;     // [job][band pixels] spectrum gathered in band order
    const double* sum_ss;       // [job] sum of S^2 over the band
    const int* spec_off;        // [job] offset of the job's band spectrum
    float4* cand;               // [job][kMaxCand] (mean_px, sig*cos2a, sig*sin2a, phase/pi)
    float2* cval;               // [job][kMaxCand] searched parameter values
    double2* part;              // [job][kMaxCand][max_chunks] (sum CS, sum CC)
    int* arrive;                // [job] blocks of the current step done (0 between steps)
    int max_chunks;
    int njobs;
};

// ---------------------------------------------------------------------------
// Kernel launchers (defined in the .cu units).  All enqueue on `st`.
// ---------------------------------------------------------------------------

// gcf_spectrum.cu
void launch_extract_tiles(const float* img, int w, int h, int pitch, int tile, int ntx,
                          int offx, int offy, int stride, int first_tile, int ntiles,
                          const float* taper, float* out, cudaStream_t st);
void launch_amp_accumulate(const float2* cmp, int tile, int ntiles, double* acc, cudaStream_t st);
void launch_finalize_raw(const double* acc, int n, double inv, float* raw, cudaStream_t st);
void launch_fourier_crop(const float2* in, int cx_in, int cy_in, float2* out, int cx_out,
                         int cy_out, cudaStream_t st);
// gcf_fused.cu: fused tile-spectrum kernel (tile 512).
struct FusedImageDesc {          // layout must match FusedTab in gcf_fused.cu
    const float* img;
    const double* bsum;
    int pitch;
    int ntx, nty;
    int offx, offy, stride;
    int vec;
    int nbx;
};
int fused_tile_supported(int tile);
cudaError_t fused_max_clusters(int* n, int* shape);
cudaError_t fused_clusters_of(int shape, int* n);   // shape 8, 816 or 16
// CTAs of the cluster-less tile kernel beside a cluster launch (on the SMs
// the clusters leave free), with their global scratch: col holds
// solo_scratch_float2(n) float2, acc solo_scratch_floats(n) floats.  fork and
// join order `st` around the launch on the solo stream.
struct SoloLaunch {
    int n;
    int reserve_per_cluster;   // they stop taking items when <= this x clusters remain
    cudaStream_t st;
    float2* col;
    float* acc;
    cudaEvent_t fork, join;
};
size_t solo_scratch_float2(int nsolo);
size_t solo_scratch_floats(int nsolo);
// Spectra of images img0 .. img0 + nimg - 1 of descs/bsum_out/first/inv.
// items: the nitems work items of those images, (image, first tile, end
// tile, item index into partial); first[img]..first[img+1] are the items of
// image img; inv[img] = 1 / tiles of img; raw: the spectrum of image img0;
// next_item: the launch's 64-bit item queue counter (zeroed on st).
cudaError_t launch_fused(const void* descs, double* const* bsum_out, int max_blocks, const int4* items,
                         int nitems, const int* first, const float* inv, int img0, int nimg,
                         const float* taper, const float2* tw, float* partial, float* raw,
                         unsigned long long* next_item, int nclusters, int shape, cudaStream_t st,
                         cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr, const SoloLaunch* solo = nullptr);

// gcf_post.cu
void launch_bg_horizontal(const float* raw, int tile, int nmic, int log_spect, double* hsum,
                          cudaStream_t st);
void launch_bg_vertical(const float* raw, const double* hsum, int tile, int nmic, int log_spect,
                        float* ctf, cudaStream_t st);
void launch_moments(const float* spect, int n, int nmic, double* out2, cudaStream_t st);
// lowpass of CFindCtfBase::mLowpass around a batched R2C / C2R pair
void launch_lp_full(const float* ctf0, int tile, int nmic, float* full, cudaStream_t st);
void launch_lp_table(double* g, int tile, double bfactor, cudaStream_t st);
void launch_lp_filter(float2* cmp, int tile, int nmic, const double* g, cudaStream_t st);
void launch_lp_extract(const float* ctf0, const float* full, int tile, int nmic, const double* moments,
                       float* out, int* lowpassed, cudaStream_t st);
void launch_radial(const float* spect, int tile, int nmic, const int* off, const int* pix,
                   float* radial, cudaStream_t st);
void launch_band_gather(const float* ctf, int cmp_n, const SearchJob* jobs, const BandDev* bands,
                        const int* spec_off, int njobs, float* band_spec, double* sum_ss,
                        cudaStream_t st);
void launch_full_spectrum(const float* ctf, int tile, int nmic, const int* mic_of,
                          const gcf_result* res, const PixOptics* o, const double* moments,
                          float res_lo_freq_dummy, float* full, cudaStream_t st);
void launch_ctf_res(const float* ctf, int tile, const SearchJob* jobs, int njobs, const int* ring_off,
                    const int* ring_pix, const double2* ring_geo, double* ring_sums, float* cc,
                    cudaStream_t st);

// gcf_control.cu: candidate kernel with the state machine in its last blocks
void launch_eval2d(const EvalArgs& a, int cand_blocks, int max_band_n, cudaStream_t st);
void launch_init_jobs(const EvalArgs& a, cudaStream_t st);
void launch_search1d(SearchJob* jobs, int njobs, const float* radial, int cx, float4* cand,
                     float2* cval, cudaStream_t st);
void launch_shell_select(SearchJob* jobs, int njobs, const float* cc, int cx, int cy,
                         cudaStream_t st);
// counts (nullable): per job n_cand2d, n_cand1d, n_pairs1d
void launch_results(const SearchJob* jobs, int njobs, const int* lowpassed, gcf_result* out, int* counts,
                    cudaStream_t st);

// gcf_background.cu: GBackground1D
constexpr int kMaxBackgroundBins = 12288;   // one block's shared memory (48 KB)
cudaError_t launch_background1d(const float* spec, int n, float* bg, int* start, cudaStream_t st);
cudaError_t launch_remove_background1d(float* spec, int n, const float* bg, int bg_n, int start,
                                       cudaStream_t st);
cudaError_t launch_remove_background2d(float* spec, int tile, const float* bg, int bg_n, int start,
                                       cudaStream_t st);

}  // namespace gcf
