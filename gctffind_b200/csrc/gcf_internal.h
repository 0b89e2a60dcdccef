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

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gctf_b200.h"

namespace gcf {

// Device-allocation epoch: every (re)allocation of a context buffer bumps
// it, so a captured CUDA graph (which holds raw device addresses) is only
// replayed while the epoch it was captured in is current.
void note_device_alloc();
unsigned long long device_alloc_epoch();
// Records a timing event on st; inside a stream capture it becomes an event
// node of the graph (recorded again on every replay).
cudaError_t record_timing(cudaEvent_t ev, cudaStream_t st);

// gcf_resize.cu: the Fourier-crop rescale as line transforms.  A line of
// length n (<= kResizeMaxLine) is transformed whole, or (split = 1) as the
// DFTs of its even and odd samples combined by one radix-2 step with the
// twiddles ts[k] = exp(-2 pi i k / n), k < n/2.  The transform of length
// n (or n/2 when split): FFT length M (that length when a power of two,
// else the power of two >= 2 length - 1 of Bluestein's convolution), and for
// Bluestein the chirp exp(-i pi j^2 / length) and the spectrum of its
// conjugate over M, divided by M.
constexpr int kResizeMaxLine = 4096;
struct ResizeLine {
    int n, M;
    const float2* chirp;
    const float2* bf;
    int split;
    const float2* ts;
};
bool resize_line_ok(int n);
cudaError_t resize_line(int n, ResizeLine* out);
// exp(sign 2 pi i k / len), k < count
cudaError_t resize_twiddles(int len, int sign, int count, const float2** out);
size_t resize_cols_smem(int h, int m_max, int e_max);
// img (w x h, w even) -> out (nw x nh); T1: (nw/2 + 1) x h, T2: (nw/2 + 1) x nh
// complex scratch; tA = exp(-2 pi i k / w), k <= w/2; tC = exp(2 pi i k / nw),
// k < nw/2.
cudaError_t launch_resize(const float* img, int w, int h, int nw, int nh, const ResizeLine& rowA,
                          const float2* tA, const ResizeLine& colF, const ResizeLine& colI, const ResizeLine& rowC,
                          const float2* tC, float2* T1, float2* T2, float* out, cudaStream_t st);

// gcf_mrc.cpp: section layout of an MRC file (false if unreadable) and the
// bytes per pixel of a mode (0 if unsupported).
bool mrc_layout(const char* path, int dims[3], int* mode, bool* swap, long long* data_off);
int mrc_mode_bytes(int mode);
// gcf_ingest.cu: raw MRC section bytes (mode 0/5 unsigned char, 1 short,
// 6 unsigned short, 2 float; `swap`: big-endian file) to float.
cudaError_t launch_mrc_to_float(const void* raw, int mode, int swap, size_t npx, float* out, cudaStream_t st);
// dst (device) = bytes read by a kernel from mapped page-locked host memory
// (src_mapped: its device-side address).  Small uploads take this route
// instead of a copy-engine transfer, so they never queue behind the bulk
// image uploads on the copy engines.
cudaError_t launch_copy_from_host(void* dst, const void* src_mapped, size_t bytes, cudaStream_t st);

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
    STEP_DONE = 6,
    // finish of the BF16 contraction search (mode 4): the best of the
    // table's top candidates re-scored in FP32, then local 3 x 3 x 3 grids
    STEP_RESCORE = 7,
    STEP_LOCAL = 8
};

constexpr int kRescore = 4;      // table candidates re-scored in FP32
constexpr int kLocalPasses = 4;  // local 3 x 3 x 3 passes after the re-score

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
    int mode;           // 0 = Do2D (after the 1D search), 1 = Refine, 2 = Do1D, 3 = Refine1D,
                        // 4 = contraction search (table search, then the FP32 finish)
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
    // contraction search (mode 4): candidates scored on the BF16 table, the
    // table's best candidates for the FP32 re-score, the local steps
    int n_table;
    float rs_df[kRescore], rs_ast[kRescore], rs_ang[kRescore];
    float loc_ddf, loc_dast, loc_dang;
    int pad3;
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
// gcf_fused.cu: the whole lowpass of 512 x 512 spectra (ctf0 -> out, the
// variance gate included) with the warp FFT; rowf: 512 x 512 floats per
// spectrum of scratch; tw: exp(-2 pi i k / 512), k < 512.
cudaError_t launch_lowpass512(const float* ctf0, const float2* tw, double bfactor, int nmic, const double* moments,
                              float* rowf, float* out, int* lowpassed, cudaStream_t st);
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

// gcf_umma.cu: BF16 x BF16 -> FP32 tensor-core product D = A * B^T (A: M x K,
// B: N x K, both K-major), 128 x bn tiles (bn = 32, 64, 128 or 256),
// `stages`-deep TMA ring (see the file for the supported pairs).
struct GemmArgs {
    int M = 0, N = 0, K = 0;
    float* D = nullptr;            // FP32 row-major output (nullable), pitch ldd
    long long ldd = 0;
    __nv_bfloat16* Db = nullptr;   // BF16 row-major copy (nullable), pitch ldd
    __nv_bfloat16* Dt = nullptr;   // BF16 transposed copy Dt[n][m] (nullable), pitch ldt
    long long ldt = 0;
    const float* bias = nullptr;   // added per column n before the ReLU (nullable)
    int relu = 0;
    int accumulate = 0;            // D += A B^T (FP32 output only)
    int vec4 = 0;                  // set by the launcher
    const int2* tiles = nullptr;   // (m0, n0) of each CTA's tile; null: the whole grid
    const int* ntiles = nullptr;   // device count of `tiles` (CTAs beyond it exit at once)
    int* err = nullptr;            // device flag: 0 ok, else the wait that ran out
};
int umma_tile_n_supported(int bn);
cudaError_t launch_umma_gemm(const __nv_bfloat16* A, long long lda, const __nv_bfloat16* B, long long ldb,
                             GemmArgs g, int bn, int stages, int ntiles, cudaStream_t st);
// The same product by one persistent CTA per SM over all tiles, the
// accumulator double-buffered in tensor memory (pairs 256 x 3/4, 128 x 4/6,
// 64 x 4, 32 x 4).
cudaError_t launch_umma_gemm_persistent(const __nv_bfloat16* A, long long lda, const __nv_bfloat16* B,
                                        long long ldb, GemmArgs g, int bn, int stages, int ntiles, cudaStream_t st);

// gcf_rsgemm.cu: the Fourier-crop rescale as two BF16 tensor-core products
// (raw sides up to kRescaleGemmMax).  Scratch: bf16_elems BF16 and
// f32_elems FP32 elements, laid out as below (offsets in elements).
constexpr int kRescaleGemmMax = 16384;
struct RescaleGemmLayout {
    long long ldw, ldk;                   // row pitches: K = w, K = h + 1
    long long off_x, off_w, off_k, off_t; // BF16 image, row map, column map, T^T
    long long bf16_elems;
    long long off_uc, off_bias;           // FP32: partial column sums at 0, (u, cos, sin, cos) per
    long long f32_elems;                  // column, the per-column bias
};
bool rescale_gemm_supported(int w, int h, int nw, int nh);
RescaleGemmLayout rescale_gemm_layout(int w, int h, int nw, int nh);
// img (w x h, row pitch `pitch` floats) -> out (nw x nh, dense); err: the
// products' device flag (0 on entry; set if a bounded wait gave up).
cudaError_t launch_rescale_gemm(const float* img, long long pitch, int w, int h, int nw, int nh,
                                __nv_bfloat16* bf, float* f32, int* err, float* out, cudaStream_t st);

// gcf_contract.cu: the BF16 candidate contraction.
// Common polar grid of a batch: ns bins uniform in s^2 (1/A^2) over the
// band [s2_lo, s2_lo + ns * ds2), nth angle bins over [-90, 90) degrees, and
// nz defocus rows z_i = z0 + i * dz (Angstrom).
struct PolarGrid {
    int ns, nth, nz, pad;
    float s2_lo, ds2;
    float z0, dz;
    float wl, cs;          // wavelength and Cs, Angstrom
    float amp_phase;       // amplitude-contrast phase + extra phase, radian
    float pad2;
};
// Model rows A[i][k] = |sin(chi(z_i, s2_k))| - 1/2 and A2 = A^2, BF16,
// nz x ns (row pitch ns).
void launch_polar_model(const PolarGrid& g, __nv_bfloat16* A, __nv_bfloat16* A2, cudaStream_t st);
// Per job j (spectrum slot mic[j], pixel size px[j]): the background-
// removed half spectrum summed into (s^2, angle) cells, times the job's
// envelope exp(-16 s^2 px^2), as BF16 rows B[j * nth + t][k]; the
// envelope^2-weighted pixel count per s^2 bin E[j][k]; sum of S^2 over the
// band's pixels ss[j].
cudaError_t launch_polar_bin(const float* ctf, int tile, const SearchJob* jobs, int njobs, const PolarGrid& g,
                             __nv_bfloat16* B, __nv_bfloat16* E, double* ss, cudaStream_t st);
// Rows [lo, hi) of the defocus grid each job's table search can touch
// (prior: optional learned (mean, ratio, angle, window scale) per job).
void launch_job_rows(const SearchJob* jobs, int njobs, const float4* prior, const PolarGrid& g, int2* rows,
                     cudaStream_t st);
// Row tiles of P = A B^T that the jobs need: job j needs rows rows[j] =
// [lo, hi); a column block of bn columns (bn / nth jobs) gets the row tiles
// covering the union of its jobs' rows.  tiles: (m0, n0), *ntiles their
// count (capacity max_tiles).
void launch_plan_tiles(const int2* rows, int njobs, int nth, int nz, int bn, int2* tiles, int* ntiles,
                       int max_tiles, cudaStream_t st);

// gcf_control.cu: the search on the contraction's table (one CTA per job).
struct TableArgs {
    SearchJob* jobs;
    int njobs;
    const float* P;          // [nz][ldp]: job j's angle bins at columns j * nth ..
    long long ldp;
    const float* Dz;         // [njobs][ldd]: job j's normaliser sum C^2 at each row
    long long ldd;
    const double* ss;        // [njobs]
    PolarGrid g;
    const int2* rows;        // [njobs] rows computed for each job
    const float4* prior;     // [njobs] (mean A, ratio, angle deg, window scale) or null
    float4* cand;
    float2* cval;
};
void launch_table_search(const TableArgs& a, cudaStream_t st);
// Seeded uniform fills (autotuner trial operands): floats in [lo, hi), BF16 in [-1, 1).
void launch_fill_f32(float* p, size_t n, unsigned long long seed, float lo, float hi, cudaStream_t st);
void launch_fill_bf16(__nv_bfloat16* p, size_t n, unsigned long long seed, cudaStream_t st);

// gcf_nn.cu: the learned initialiser's kernels (see the file for the network).
constexpr int kNnProfile = 256;            // x1 bins
constexpr int kNnMap = 256;                // x2 is kNnMap x kNnMap
constexpr int kNnOut = 3;                  // (mean, ax, ay)
constexpr int kNnPredPitch = 16;           // FP32 prediction rows
// spectra in slots 0 .. n-1 of ctf; px[j * px_stride]: pixel size of slot j
cudaError_t launch_nn_input(const float* ctf, int tile, const float* px, int px_stride, int n, __nv_bfloat16* x1,
                            __nv_bfloat16* x2, cudaStream_t st);
// params: 8 floats per sample; target: 3 floats per sample
void launch_synth_params(unsigned long long seed, unsigned long long first, int n, float* params, float* target,
                         cudaStream_t st);
// base: optics with the wavelength and Cs in Angstrom
void launch_synth_raw(unsigned long long seed, unsigned long long first, const float* params, int n, int tile,
                      const PixOptics& base, float* raw, cudaStream_t st);
void launch_im2col_p4(const __nv_bfloat16* x, int B, __nv_bfloat16* cols, cudaStream_t st);
// the first layer (4 x 4 stride-4 patches of x, 16 outputs, bias + ReLU)
// without im2col rows; w: [16][16] BF16; x 8-byte and y 16-byte aligned (the
// network's own buffers)
void launch_conv1_direct(const __nv_bfloat16* x, int B, const __nv_bfloat16* w, const float* bias,
                         __nv_bfloat16* y, cudaStream_t st);
void launch_im2col_3s2(const __nv_bfloat16* x, int B, int H, int W, int C, __nv_bfloat16* cols, cudaStream_t st);
void launch_col2im_3s2_relu(const float* dcols, const __nv_bfloat16* y, int B, int H, int W, int C,
                            __nv_bfloat16* dz, cudaStream_t st);
void launch_relu_bwd(const float* dy, long long ldy, const __nv_bfloat16* y, long long ldyy, int rows, int n,
                     __nv_bfloat16* dz, long long ldz, cudaStream_t st);
void launch_concat(const __nv_bfloat16* x1, const __nv_bfloat16* y4, int B, __nv_bfloat16* h0, cudaStream_t st);
void launch_wgrad(const __nv_bfloat16* dz, long long ldz, const __nv_bfloat16* x, long long ldx, int rows, int nout,
                  int nin, float* dw, float* db, cudaStream_t st);
void launch_mse(const float* pred, long long ldp, const float* target, int B, float* loss, __nv_bfloat16* dpred,
                cudaStream_t st);
void launch_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                 float c1, float c2, int nout, int nin, __nv_bfloat16* wb, __nv_bfloat16* wt, long long ldt,
                 cudaStream_t st);
void launch_copy_weights(const float* w, int nout, int nin, __nv_bfloat16* wb, __nv_bfloat16* wt, long long ldt,
                         cudaStream_t st);
void launch_prior(const float* pred, long long ldp, int n, float4* prior, cudaStream_t st);

// gcf_learned.cpp: the network's state and passes (device buffers, one stream).
struct NnNet;
NnNet* nn_create();
void nn_destroy(NnNet* n);
size_t nn_param_count();
// He-normal weights from the seed, zero biases
cudaError_t nn_init_random(NnNet* n, unsigned long long seed, cudaStream_t st);
cudaError_t nn_set_params(NnNet* n, const float* host, cudaStream_t st);
cudaError_t nn_get_params(NnNet* n, float* host, cudaStream_t st);
cudaError_t nn_get_grads(NnNet* n, float* host, cudaStream_t st);
// x1 [B][256], x2 [B][256][256] BF16 (device) -> pred [B][kNnPredPitch] FP32 (device, owned by the net)
cudaError_t nn_forward(NnNet* n, const __nv_bfloat16* x1, const __nv_bfloat16* x2, int B, cudaStream_t st);
const float* nn_pred(NnNet* n);
// after nn_forward: gradients of the mean squared error against target
// [B][3] (device) into the net's FP32 gradient buffer, loss (device) += mean
cudaError_t nn_backward(NnNet* n, const float* target, int B, float* loss, cudaStream_t st);
cudaError_t nn_adam(NnNet* n, float lr, cudaStream_t st);
int* nn_err_flag(NnNet* n);

// gcf_background.cu: GBackground1D
constexpr int kMaxBackgroundBins = 12288;   // one block's shared memory (48 KB)
cudaError_t launch_background1d(const float* spec, int n, float* bg, int* start, cudaStream_t st);
cudaError_t launch_remove_background1d(float* spec, int n, const float* bg, int bg_n, int start,
                                       cudaStream_t st);
cudaError_t launch_remove_background2d(float* spec, int tile, const float* bg, int bg_n, int start,
                                       cudaStream_t st);

}  // namespace gcf
