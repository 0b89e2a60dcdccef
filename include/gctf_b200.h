/*
 * gctf_b200.h -- C ABI of the B200-native GCtfFind CTF-estimation path.
 *
 * Plain C types only (no CUDA or torch types in any signature).  Every entry
 * point returns a gcf_status; none asserts, exits or resets the device.
 * A context owns all device memory and one CUDA stream; the caller owns
 * every host buffer.  Use one context per host thread.
 *
 * The reference surface each entry point replaces is cited beside it
 * (paths are relative to the GCtfFind source tree).
 */
#ifndef GCTF_B200_H
#define GCTF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GCF_OK = 0,
    GCF_ERR_INVALID_ARG = 1,     /* bad pointer, size or flag           */
    GCF_ERR_CUDA = 2,            /* CUDA runtime error                  */
    GCF_ERR_CUFFT = 3,           /* cuFFT error (rescale, cuFFT variant) */
    GCF_ERR_NO_MEMORY = 4,       /* device or host allocation failed    */
    GCF_ERR_IMAGE_TOO_SMALL = 5, /* image holds no full tile            */
    GCF_ERR_STATE = 6,           /* call out of order (e.g. Do2D before
                                    a spectrum was generated)           */
    GCF_ERR_IO = 7,              /* file could not be read or written   */
    GCF_ERR_TIMEOUT = 8          /* bounded device wait gave up         */
} gcf_status;

typedef struct gcf_ctx gcf_ctx;

/* Optics of CCTFTheory::Setup (FindCTF/CCTFTheory.cpp:69-86) and the
 * -ExtPhase pair of CInput (CInput.cpp:43-58, :152-155). */
typedef struct {
    float kv;               /* keV                                    */
    float cs_mm;            /* spherical aberration, mm               */
    float amp_contrast;     /* amplitude contrast fraction            */
    float pixel_size;       /* raw pixel size, Angstrom               */
    float ext_phase_deg;    /* initial extra phase, degree            */
    float ext_phase_range;  /* extra-phase search range, degree (<=0: off) */
} gcf_optics;

/* Result row (CFindSeriesCtfs::mGetResults, CFindSeriesCtfs.cpp:378-386)
 * plus the 1D estimate and the spectral-CC resolution that the reference
 * computes but does not report (FindCTF/CFindDefocus2D.cpp:382-400). */
typedef struct {
    float df_min;      /* Angstrom */
    float df_max;      /* Angstrom */
    float azimuth;     /* degree   */
    float ext_phase;   /* degree   */
    float score;       /* CC       */
    float ctf_res;     /* Angstrom */
    float df_1d;       /* 1D estimate, Angstrom (0 after Refine) */
    float phase_1d;    /* 1D estimate, degree   */
    float score_1d;    /* 1D CC                 */
    int   lowpassed;   /* 1 if the B-factor lowpass ran           */
} gcf_result;

/* Spectrum-stage implementation. */
typedef enum {
    GCF_SPECT_FUSED = 0,   /* hand-written fused tile-FFT kernel (default) */
    GCF_SPECT_CUFFT = 1    /* batched cuFFT comparison variant            */
} gcf_spectrum_impl;

/* Rescale implementation (CRescaleImage::DoIt, FindCTF/CRescaleImage.cpp:76-99). */
typedef enum {
    GCF_RESCALE_CUFFT = 0, /* cuFFT R2C + crop + C2R, the reference's calls
                              (default: the faster once a size's plans exist) */
    GCF_RESCALE_LINES = 1, /* hand-written line transforms (gcf_resize.cu): no
                              plans to make, so new sizes cost nothing extra;
                              raw width even and every line of the raw and new
                              sizes <= 4096 long, else cuFFT */
    GCF_RESCALE_GEMM = 2   /* the crop as two BF16 tensor-core products
                              (gcf_rsgemm.cu): img -> Rh img Rw^T with closed-form
                              maps; BF16 operands, so within ~0.5 % of rms of
                              cuFFT, not bit-identical; raw sides <= 16384,
                              else cuFFT */
} gcf_rescale_impl;

/* ---------------------------------------------------------------------- */
/* Context                                                                  */
/* ---------------------------------------------------------------------- */

/* Replaces the CInput tile/log-spectrum globals read by CFindCtfBase
 * (FindCTF/CFindCtfBase.cpp:52-54, :111-112) and the device choice of
 * CProcessMain::DoIt (CProcessMain.cpp:26). */
gcf_status gcf_create(int gpu, int tile_size, int log_spect, gcf_ctx** out);
void       gcf_destroy(gcf_ctx* ctx);
const char* gcf_strerror(gcf_status s);
/* Last error detail of this context (CUDA/cuFFT message), never NULL. */
const char* gcf_last_error(gcf_ctx* ctx);
gcf_status gcf_set_spectrum_impl(gcf_ctx* ctx, int impl);
/* GCF_RESCALE_CUFFT (default), GCF_RESCALE_LINES or GCF_RESCALE_GEMM for
 * the images below 1.2 A/px. */
gcf_status gcf_set_rescale_impl(gcf_ctx* ctx, int impl);
/* Cluster shape of the fused tile kernel: 0 = the shape that keeps the most
 * SMs busy (default), 8 = 8 CTAs x 8 warps, 816 = 8 CTAs x 16 warps,
 * 16 = 16 CTAs x 16 warps, 162 = 16 CTAs x 8 warps with two CTAs per SM,
 * 168 = 16 CTAs x 8 warps with a double-buffered column buffer.
 * For tuning (gcf_autotune picks one by timing); results do not depend on it. */
gcf_status gcf_set_fused_shape(gcf_ctx* ctx, int shape);

/* ---------------------------------------------------------------------- */
/* CFindCtf2D call shape (FindCTF/CFindCTFInc.h:541-623)                    */
/* ---------------------------------------------------------------------- */

/* CFindCtf2D::Setup1 + Setup2 (FindCTF/CFindCtf2D.cpp:33-42,
 * FindCTF/CFindCtfBase.cpp:48-76): optics with the pixel size of the image
 * that will be passed to gcf_gen_half_spectrum (i.e. after rescaling). */
gcf_status gcf_setup(gcf_ctx* ctx, const gcf_optics* optics, int width, int height);

/* CFindCtfBase::GenHalfSpectrum (FindCTF/CFindCtfBase.cpp:109-116): average
 * amplitude spectrum of the tiles of `img` (width x height floats, row
 * pitch `pitch` floats), background removal and lowpass.  `img_is_device`
 * = 1 when img is a device pointer on the context's GPU. */
gcf_status gcf_gen_half_spectrum(gcf_ctx* ctx, const float* img, int pitch, int img_is_device);

/* CFindCtfBase::SetPhase (FindCTF/CFindCtfBase.cpp:78-82). */
gcf_status gcf_set_phase(gcf_ctx* ctx, float phase_deg, float range_deg);

/* CFindCtf2D::Do2D (FindCTF/CFindCtf2D.cpp:44-53). */
gcf_status gcf_do2d(gcf_ctx* ctx, gcf_result* out);

/* CFindCtf2D::Refine (FindCTF/CFindCtf2D.cpp:55-66): {centre, range} pairs. */
gcf_status gcf_refine(gcf_ctx* ctx, const float df_mean[2], const float ast_ratio[2],
                      const float ast_angle[2], const float ext_phase[2], gcf_result* out);

/* CFindCtf1D::Do1D (FindCTF/CFindCtf1D.cpp:49-56): radial average, brute-
 * force defocus x extra-phase search, refinement; out->df_min = df_max =
 * the 1D defocus, out->ext_phase / score its phase and CC.  Like the
 * reference it moves the context's extra phase (SetPhase) to the result. */
gcf_status gcf_do1d(gcf_ctx* ctx, gcf_result* out);
/* CFindCtf1D::Refine1D (FindCTF/CFindCtf1D.cpp:58-67): the refinement pass
 * alone around init_df (Angstrom) over df_range, centred on the context's
 * extra phase. */
gcf_status gcf_refine1d(gcf_ctx* ctx, float init_df, float df_range, gcf_result* out);

/* GBackground1D (FindCTF/GBackground1D.cu:61-169).  The reference keeps
 * this 1D background model without calling it; it is offered here behind
 * the same three operations.  `on_device` says whether every array
 * argument is device memory (else host).  n <= 12288 bins. */
/* DoIt + mFindStart: start = first bin from 2 on where the spectrum falls to
 * the least-squares line fitted over bins [n/5, n - n/5) (n/5 if none);
 * background[i] = mean of the start/2*2-1 bins centred on i (mirrored at
 * the end) for i >= start, 0 below. */
gcf_status gcf_background1d(gcf_ctx* ctx, const float* spectrum, int n, int on_device,
                            float* background, int* start);
/* Remove1D: spectrum[i] -= background[i] for start <= i < min(n, bg_n),
 * 0 for i < start (in place). */
gcf_status gcf_remove_background1d(gcf_ctx* ctx, float* spectrum, int n, const float* background,
                                   int bg_n, int start, int on_device);
/* Remove2D: on a tile x (tile/2+1) half spectrum (DC at (0, tile/2)),
 * subtract the background at radius r (pixels, linear interpolation;
 * background[bg_n-1] from r >= bg_n - 1), 0 inside r < start (in place). */
gcf_status gcf_remove_background2d(gcf_ctx* ctx, float* half_spectrum, int tile,
                                   const float* background, int bg_n, int start, int on_device);

/* CFindCtfBase::GetSpectSize (FindCTF/CFindCtfBase.cpp:102-107). */
gcf_status gcf_get_spect_size(gcf_ctx* ctx, int size[2], int half);

/* CFindCtfBase::GetHalfSpect (FindCTF/CFindCtfBase.cpp:90-100): raw (1) or
 * background-removed (0) half spectrum, (tile/2+1) x tile floats, DC at
 * (0, tile/2), copied to host. */
gcf_status gcf_get_half_spectrum(gcf_ctx* ctx, int raw, float* host_out);

/* CFindCtfBase::GenFullSpectrum (FindCTF/CFindCtfBase.cpp:118-133): the
 * tile x tile diagnostic spectrum with the fitted |CTF| in the left half,
 * for the result `res` (normally the last Do2D/Refine result). */
gcf_status gcf_gen_full_spectrum(gcf_ctx* ctx, const gcf_result* res, float* host_out);

/* GRadialAvg of the current spectrum (FindCTF/GRadialAvg.cu:43-53):
 * tile/2+1 floats to host. */
gcf_status gcf_get_radial_average(gcf_ctx* ctx, float* host_out);

/* ---------------------------------------------------------------------- */
/* CTF theory (CCTFTheory / CCTFParam, FindCTF/CCTFTheory.cpp:9-301,         */
/* FindCTF/CFindCTFInc.h:8-91): host math, no GPU, bit-identical to the      */
/* reference's float/double arithmetic.                                      */
/* ---------------------------------------------------------------------- */
/* Field order and units of CCTFParam: lengths in pixels, angles in radian. */
typedef struct {
    float wavelength;    /* pixel                                   */
    float cs;            /* spherical aberration, pixel             */
    float amp_contrast;  /* fraction                                */
    float amp_phase;     /* atan(Ac / sqrt(1 - Ac^2)), radian       */
    float ext_phase;     /* extra phase mod pi, radian              */
    float df_max;        /* pixel                                   */
    float df_min;        /* pixel                                   */
    float azimuth;       /* astigmatism azimuth, radian             */
    float ast_tol;       /* pixel                                   */
    float pixel_size;    /* Angstrom                                */
} gcf_ctf_param;

/* CCTFTheory::Setup(kV, Cs mm, Ac, pixel A, astigmatism tolerance A,
 * extra phase radian); clears the defocus. */
gcf_status gcf_ctf_setup(gcf_ctf_param* p, float kv, float cs_mm, float amp_contrast,
                         float pixel_size, float ast_tol, float ext_phase_rad);
gcf_status gcf_ctf_set_ext_phase(gcf_ctf_param* p, float phase, int degree);
gcf_status gcf_ctf_get_ext_phase(const gcf_ctf_param* p, int degree, float* out);
/* CCTFTheory::SetDefocus (Angstrom) / SetDefocusInPixel. */
gcf_status gcf_ctf_set_defocus(gcf_ctf_param* p, float df_min_a, float df_max_a, float azimuth_rad);
gcf_status gcf_ctf_set_defocus_px(gcf_ctf_param* p, float df_min_px, float df_max_px,
                                  float azimuth_rad);
gcf_status gcf_ctf_change_pixel_size(gcf_ctf_param* p, float new_pixel_size);
/* CCTFTheory::Evaluate: -sin(phase shift) at a relative frequency in
 * [-0.5, 0.5] (1/pixel) along `azimuth` (radian). */
gcf_status gcf_ctf_evaluate(const gcf_ctf_param* p, float freq, float azimuth, float* out);
gcf_status gcf_ctf_phase_shift(const gcf_ctf_param* p, float freq, float azimuth, float* out);
/* CCTFTheory::CalcDefocus: defocus (pixel) along an azimuth. */
gcf_status gcf_ctf_defocus(const gcf_ctf_param* p, float azimuth, float* out);
/* CCTFTheory::CalcFrequency / CalcNthZero: relative frequency where the
 * phase shift reaches `phase` (n pi); 0 if none. */
gcf_status gcf_ctf_frequency(const gcf_ctf_param* p, float phase, float azimuth, float* out);
gcf_status gcf_ctf_nth_zero(const gcf_ctf_param* p, int n, float azimuth, float* out);
/* CCTFTheory::EqualTo: *out = 1 when p and q agree within the tolerances. */
gcf_status gcf_ctf_equal(const gcf_ctf_param* p, const gcf_ctf_param* q, float df_tol, int* out);

/* ---------------------------------------------------------------------- */
/* Rescale (CRescaleImage, FindCTF/CRescaleImage.cpp:47-99)                  */
/* ---------------------------------------------------------------------- */
void       gcf_rescale_dims(int width, int height, float pixel_size, int* new_width,
                            int* new_height, float* new_pixel_size);
/* Fourier-crop `img` (host or device) to >= 1.2 A/px; output dense
 * new_width x new_height floats to host. */
gcf_status gcf_rescale(gcf_ctx* ctx, const float* img, int width, int height, float pixel_size,
                       int img_is_device, float* host_out);

/* ---------------------------------------------------------------------- */
/* Batched paths                                                            */
/* ---------------------------------------------------------------------- */

/* CFindSeriesCtfs::DoIt policy (CFindSeriesCtfs.cpp:50-213) over n
 * equally-sized raw images: images[i] is image i (host or device, dense
 * width x height floats); `order` is the processing order (order[0] gets the
 * full search; every later image is refined around the best-scoring earlier
 * one; a refine with score <= 0 falls back to the full search).  is_tomo
 * selects the tilt-series refine windows (CFindSeriesCtfs.cpp:168-193).
 * results[i] receives image i.  full_spectra (nullable) receives n
 * tile x tile diagnostic spectra in image order. */
gcf_status gcf_run_series(gcf_ctx* ctx, const float* const* images, int n, int width,
                          int height, int images_are_device, const gcf_optics* optics,
                          const int* order, int is_tomo, gcf_result* results,
                          float* full_spectra);

/* Called on the calling host thread during gcf_run_series each time one
 * more package's result is final, in processing order: `done` packages are
 * final so far, the last being image `image` with `result`.  This is the
 * hook of the reference's crash-safety flush, which rewrites the CTF and
 * Imod files after every 21st package (CFindSeriesCtfs.cpp:97-101).  The
 * callback must not call into this context.  fn = NULL removes it. */
typedef void (*gcf_package_fn)(void* user, int done, int image, const gcf_result* result);
gcf_status gcf_set_package_callback(gcf_ctx* ctx, gcf_package_fn fn, void* user);

/* Independent full searches (CFindCtf2D::Do2D per image, the single-file
 * mode of CInputFolder::mReadSingle, CInputFolder.cpp:159-192) of n images
 * of possibly different sizes and pixel sizes, batched on the GPU. */
typedef struct {
    const float* image;      /* host or device, dense width x height */
    int width, height;
    float pixel_size;        /* raw pixel size, Angstrom */
} gcf_item;
gcf_status gcf_run_batch(gcf_ctx* ctx, const gcf_item* items, int n, int images_are_device,
                         const gcf_optics* optics, gcf_result* results);

/* Search method of a batch. */
typedef enum {
    GCF_SEARCH_PLAIN = 0,    /* the reference's FP32 search per micrograph
                                (CFindCtf1D::Do1D + CFindCtf2D::Do2D)       */
    GCF_SEARCH_BF16 = 1,     /* all candidates x all spectra as one BF16
                                tensor-core contraction, the table searched
                                with the reference's control flow, the best
                                candidates re-scored in FP32 (FP64 sums) and
                                refined locally                             */
    GCF_SEARCH_LEARNED = 2   /* as BF16, the search window set by the learned
                                initialiser, full search as the fallback    */
} gcf_search_mode;

/* gcf_run_batch with a search method.  GCF_SEARCH_PLAIN is gcf_run_batch.
 * The contraction has no extra-phase dimension: with ext_phase_range > 0
 * every mode runs the plain search.  Replaces the per-candidate
 * GCalcCTF2D + GCC2D loop of CFindDefocus2D (FindCTF/CFindDefocus2D.cpp:
 * 153-380) and the 1D brute force of CFindDefocus1D
 * (FindCTF/CFindDefocus1D.cpp:76-119) in the contraction modes. */
gcf_status gcf_run_batch_mode(gcf_ctx* ctx, const gcf_item* items, int n, int images_are_device,
                              const gcf_optics* optics, int mode, gcf_result* results);

/* ---------------------------------------------------------------------- */
/* Learned initialiser.  No counterpart in the reference: it replaces the    */
/* coarse searches of CFindCtf1D::mFindDefocus (FindCTF/CFindCtf1D.cpp:73-90)*/
/* and CFindDefocus2D::mFindAstig (FindCTF/CFindDefocus2D.cpp:185-222) with  */
/* a window of +-5 search steps around a prediction.                        */
/* ---------------------------------------------------------------------- */
/* A small network (4 convolutions over the 256 x 256 polar half spectrum,
 * a 3-layer MLP over the 256-bin rotational profile and those features)
 * predicts mean defocus, astigmatism and angle; its BF16 forward and
 * backward passes and Adam run in this library's kernels.  Parameters are
 * FP32, gcf_nn_param_count() of them. */
size_t gcf_nn_param_count(void);
gcf_status gcf_nn_init(gcf_ctx* ctx, unsigned long long seed);
gcf_status gcf_nn_set_params(gcf_ctx* ctx, const float* params, size_t n);
gcf_status gcf_nn_get_params(gcf_ctx* ctx, float* params, size_t n);
/* Weights file: 8-byte tag "GCFNN001", the count (uint64), FP32 params. */
gcf_status gcf_nn_save(gcf_ctx* ctx, const char* path);
gcf_status gcf_nn_load(gcf_ctx* ctx, const char* path);
/* CUDA graphs for batch calls (gcf_run_batch, gcf_run_batch_mode), off by
 * default.  With graphs on, a call that repeats an earlier call's inputs
 * (the same image buffers, sizes, pixel sizes, optics and method; device
 * images, or host images in page-locked memory) is captured once and then
 * replayed as a single graph launch: rescale, spectra, post-processing and
 * the search kernels, and the small uploads they read.  The image contents
 * may change between calls; the results are those of an eager call.  No
 * counterpart in the reference, whose package loop launches every kernel
 * from the host (CFindSeriesCtfs.cpp:50-213). */
gcf_status gcf_set_graphs(gcf_ctx* ctx, int on);
/* Project autotuner.  Times, on this context's GPU, every cluster shape of
 * the fused tile kernel that the device can hold (four synthetic 4096 x 4096
 * micrographs) and the (tile N, pipeline depth) pairs of the contraction's
 * tensor-core product (a 1024 x 8192 x 512 table), and makes the fastest of
 * each this context's choice.  The trials run once per device and process;
 * later calls (and other contexts) reuse them unless `force`.  Results do
 * not depend on the choice, only speed.  No counterpart in the reference,
 * whose kernels have fixed launch shapes. */
typedef struct {
    int fused_shape;     /* tile-kernel cluster shape picked: 8, 816, 16, 162 or 168 */
    int gemm_tile_n;     /* contraction product tile picked: 128 x gemm_tile_n */
    int gemm_stages;     /* its load-pipeline depth */
    int gemm_persistent; /* 1: the persistent product (gcf_gemm_bf16_ex) */
    float fused_ms[5];   /* trial ms of shapes 8, 816, 16, 162, 168 (-1: cannot be resident) */
    float gemm_ms[10];   /* trial ms of (256,2) (256,3) (256,4) (128,4) (128,6) (64,4) one tile per
                            CTA, then (256,3) (256,4) (128,4) (128,6) persistent */
} gcf_tuning;
gcf_status gcf_autotune(gcf_ctx* ctx, int force, gcf_tuning* out);

/* [0] graph launches of the last batch call (0: it ran eagerly), [1] nodes
 * of the cached graph, [2] kernels of this library captured in it, [3] why
 * the last capture gave no graph (0: it did; 1 staging memory, 2 capture
 * could not begin, 3 an enqueued step failed, 4 capture could not end,
 * 5 a buffer was reallocated during it, 6 instantiation failed; the
 * detail is in gcf_last_error). */
gcf_status gcf_get_graph_info(gcf_ctx* ctx, long long info[4]);

/* Refined CC below which a learned search falls back to the full search
 * (default 0.1); a result at the edge of its window always falls back. */
gcf_status gcf_set_learned_threshold(gcf_ctx* ctx, float tau);
/* `steps` Adam steps of `batch` synthetic pairs each, generated on the GPU
 * from the seed (samples first, first + 1, ...): the expected averaged
 * spectrum of the micrograph model (white object x CTF x B-factor
 * envelope, smooth background, shot noise, tile averaging) for parameters
 * drawn like the uneven batch, background-removed and lowpassed by this
 * library's own post-processing.  Starts from random weights if none are
 * set.  losses (nullable, host): the mean squared error of each step. */
gcf_status gcf_nn_train(gcf_ctx* ctx, const gcf_optics* optics, int steps, int batch, unsigned long long seed,
                        unsigned long long first, float lr, float* losses);
/* The network inputs of n <= 512 synthetic samples, as host floats:
 * x1 n x 256, x2 n x 256 x 256, target n x 3, params n x 8 (mean defocus,
 * astigmatism, angle radian, pixel size, dose, tiles, raw pixel size,
 * scale); each output nullable. */
gcf_status gcf_nn_synth_inputs(gcf_ctx* ctx, const gcf_optics* optics, unsigned long long seed,
                               unsigned long long first, int n, float* x1, float* x2, float* target,
                               float* params);
/* The network inputs of n <= 512 given background-removed half spectra
 * (host, n x tile x (tile/2+1) floats in the layout of
 * gcf_get_half_spectrum) of pixel sizes px[n]: x1 n x 256 (s^2 profile),
 * x2 n x 256 x 256 (angle rows x s^2 bins), as host floats (the BF16 values
 * the network reads); each output nullable. */
gcf_status gcf_nn_inputs(gcf_ctx* ctx, const float* spectra, const float* px, int n, float* x1, float* x2);
/* One forward and backward pass on given inputs (rounded to BF16): loss,
 * the FP32 gradient of every parameter (gcf_nn_param_count floats) and the
 * predictions (n x 3); outputs nullable.  For gradient checks. */
gcf_status gcf_nn_forward_backward(gcf_ctx* ctx, const float* x1, const float* x2, const float* target, int n,
                                   float* loss, float* grads, float* pred);
/* Searches of n synthetic spectra (samples first .. first + n - 1 of the
 * seed) with the given method: results and (nullable) the samples'
 * parameters (n x 8 as above).  gcf_get_fast_counts then holds the work. */
gcf_status gcf_nn_eval_synthetic(gcf_ctx* ctx, const gcf_optics* optics, unsigned long long seed,
                                 unsigned long long first, int n, int mode, gcf_result* results, float* params);

/* ---------------------------------------------------------------------- */
/* MRC input/output (Mrc::CLoadMrc / Mrc::CSaveMrc subset,                  */
/* Include/Mrcfile/CMrcFileInc.h:52-120, MrcUtil/CLoadImages.cpp:108-181)   */
/* ---------------------------------------------------------------------- */
/* dims = {nx, ny, nz}; mode; pixel size from the cell (0 if absent);
 * ext_floats = floats per section in the extended header. */
gcf_status gcf_mrc_info(const char* path, int dims[3], int* mode, float* pixel_size,
                        int* ext_floats);
/* Section z as float (modes 0, 1, 2, 5, 6). */
gcf_status gcf_mrc_read(const char* path, int z, float* out);
/* Tilt angle of each of the first n sections from the extended header. */
gcf_status gcf_mrc_read_tilts(const char* path, float* tilts, int n);
/* Sections z0 .. z0+n-1 of an MRC file (modes 0, 1, 2, 5, 6) as float
 * images in device memory owned by the context (CLoadImages::mLoadPackage +
 * mToFloat, MrcUtil/CLoadImages.cpp:108-181).  The section bytes cross PCIe
 * as stored (1, 2 or 4 bytes per pixel) through two pinned staging buffers
 * -- the next section is read from disk while the GPU copies and widens the
 * previous one -- and a kernel converts them to float.  dev_images[k]
 * receives section z0+k's device address (dense nx x ny floats), valid
 * until the next gcf_mrc_load on this context or gcf_destroy; pass them to
 * gcf_run_series / gcf_run_batch with images_are_device = 1. */
gcf_status gcf_mrc_load(gcf_ctx* ctx, const char* path, int z0, int n, const float** dev_images);
/* float32 (mode 2) stack of nz sections. */
gcf_status gcf_mrc_write(const char* path, const float* data, int nx, int ny, int nz,
                         float pixel_size);

/* ---------------------------------------------------------------------- */
/* Result files (CSaveCtfResults::SaveCTF / SaveImod,                       */
/* CSaveCtfResults.cpp:34-117)                                              */
/* ---------------------------------------------------------------------- */
/* Writes the CTF text file (header + one row per image, 0-based index)
 * and, when is_tomo, "<path without extension>_Imod.txt" with defocus in
 * nm.  tilts and names may be NULL (0 and "" then). */
gcf_status gcf_write_ctf_file(const char* path, const gcf_result* results, const float* tilts,
                              const char* const* names, int n, int is_tomo);
/* gcf_write_ctf_file with output options.  GCF_CTF_COLUMN_RES adds the
 * spectral-CC resolution (gcf_result.ctf_res, Angstrom) as a last
 * "ctfRes" column of the CTF file; the reference computes it
 * (FindCTF/CFindDefocus2D.cpp:382-400) but writes no such column, so the
 * default (flags = 0) output is the reference's, byte for byte. */
enum { GCF_CTF_COLUMN_RES = 1 };
gcf_status gcf_write_ctf_file_ex(const char* path, const gcf_result* results, const float* tilts,
                                 const char* const* names, int n, int is_tomo, int flags);

/* ---------------------------------------------------------------------- */
/* Tensor-core building block.  No counterpart in the reference (its        */
/* candidate loop is one GCalcCTF2D + GCC2D launch pair per candidate,      */
/* FindCTF/CFindDefocus2D.cpp:363-380); this is the dense product the       */
/* batched candidate contraction is built on.                               */
/* ---------------------------------------------------------------------- */
/* d[m][n] = sum_k a[m][k] * b[n][k] on the tcgen05 tensor cores: a (m x k,
 * row pitch lda) and b (n x k, row pitch ldb) are BF16 device arrays with
 * 16-byte aligned bases and pitches, d (m x n, pitch ldd) FP32, FP32
 * accumulation.  tile_n (32, 64, 128, 256) and stages pick the kernel's
 * 128 x tile_n output tile and its load-pipeline depth (pairs: 256 x 2/3/4,
 * 128 x 2/4/6, 64 x 2/4, 32 x 2/4).  Runs on `cuda_stream` of the current
 * device and waits for it; GCF_ERR_TIMEOUT if a bounded device wait gave up. */
gcf_status gcf_gemm_bf16(const void* a, long long lda, const void* b, long long ldb, int m, int n, int k,
                         float* d, long long ldd, int tile_n, int stages, void* cuda_stream);
/* gcf_gemm_bf16 with persistent = 1: one CTA per SM walks all output tiles
 * and double-buffers the accumulator in tensor memory, so each tile's
 * epilogue overlaps the next tile's MMAs (pairs 256 x 3/4, 128 x 4/6,
 * 64 x 4, 32 x 4).  Same results as persistent = 0. */
gcf_status gcf_gemm_bf16_ex(const void* a, long long lda, const void* b, long long ldb, int m, int n, int k,
                            float* d, long long ldd, int tile_n, int stages, int persistent, void* cuda_stream);

/* ---------------------------------------------------------------------- */
/* Allocation-free spectrum.  No counterpart in the reference.              */
/* ---------------------------------------------------------------------- */
/* Averaged amplitude spectrum (512 x 512 tiles, the fused tile kernel) of
 * the device image dev_img (width x height floats, row pitch `pitch` floats)
 * into dev_raw_out (257 x 512 floats, DC at (0, 256)), on `cuda_stream`
 * (NULL = default stream) of the current device, without allocating any
 * device memory.  For callers that cannot call cudaMalloc: applications
 * whose framework owns every device allocation, or acquisition loops that
 * must not allocate because cudaMalloc can synchronise the device.
 * Its scratch is one static device array of about 9.5 MB that every GPU
 * loading this library holds until exit; it takes at most 4096 tiles
 * (e.g. 16384 x 16384 pixels) and returns GCF_ERR_INVALID_ARG beyond that.
 * The first call on a device finds the array's address and fills its
 * constant tables; make that first call before any stream capture.  All
 * calls share the array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller. */
gcf_status gcf_avg_spectrum_noalloc(const float* dev_img, int width, int height, int pitch,
                                    float* dev_raw_out, void* cuda_stream);

/* Device time (ms, CUDA events on the context streams) of the stages of the
 * last batched call: [0] upload of host inputs (it overlaps [2]), [1] time
 * in which fused tile-spectrum launches ran (the union of their intervals,
 * inside [2]; 0 for the cuFFT variant), [2] rescale + tile spectra,
 * [3] background + lowpass + radial, [4] 1D search, [5] 2D search,
 * [6] total. */
gcf_status gcf_get_stage_times(gcf_ctx* ctx, float times_ms[7]);
/* Contraction work of the last gcf_run_batch_mode call: [0] candidates
 * scored on the BF16 table, [1] tensor-core multiply-adds of the
 * contraction, [2] candidates re-scored in FP32 on the micrographs' own
 * bands, [3] learned searches that fell back to the full search. */
gcf_status gcf_get_fast_counts(gcf_ctx* ctx, long long counts[4]);
/* Device time (ms, CUDA events) of the contraction stages of the last
 * gcf_run_batch_mode call: [0] polar binning of the spectra, [1] the
 * tensor-core products (table and normaliser), [2] the table search,
 * [3] FP32 re-score and local passes, [4] the learned initialiser's
 * network (its inputs and layers; 0 for the other methods). */
gcf_status gcf_get_fast_times(gcf_ctx* ctx, float times_ms[5]);
/* Number of kernels this library launched in the last batched call. */
gcf_status gcf_get_launch_count(gcf_ctx* ctx, long long* count);
/* Search work counted on the device since the last gcf_run_series /
 * gcf_run_batch began (single-micrograph calls add to it): [0] 2D candidates
 * evaluated (each is one GCalcCTF2D + GCC2D evaluation of the reference,
 * FindCTF/CFindDefocus2D.cpp:363-380), [1] 2D (candidate, in-band pixel)
 * pairs, [2] 1D grid points (CFindDefocus1D::mBrutalForceSearch,
 * FindCTF/CFindDefocus1D.cpp:76-119), [3] 1D (grid point, bin) pairs.
 * The pair counts are the multiply-adds of model x spectrum: twice them is
 * the candidate contraction's algorithmic flop count. */
gcf_status gcf_get_search_counts(gcf_ctx* ctx, long long counts[4]);

#ifdef __cplusplus
}
#endif
#endif /* GCTF_B200_H */
