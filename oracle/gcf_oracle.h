/*
 * gcf_oracle.h -- FP64 CPU restatement of GCtfFind's CTF-estimation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product in gctffind_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product never links it and
 * never falls back to it.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths are relative to the GCtfFind source tree).  Grids, step counts and
 * integer truncations are evaluated in float32 exactly as the reference
 * writes them so that candidate grids coincide; sums, FFTs and the CTF model
 * are evaluated in double.
 */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Result row of one package (CFindSeriesCtfs::mGetResults,
 * CFindSeriesCtfs.cpp:378-386), plus the 1D estimate and the unused
 * spectral-CC resolution (CFindDefocus2D::mCalcCtfRes). */
typedef struct {
    float df_min;        /* Angstrom */
    float df_max;        /* Angstrom */
    float azimuth;       /* degree   */
    float ext_phase;     /* degree   */
    float score;         /* CC       */
    float ctf_res;       /* Angstrom (GSpectralCC2D shell), 0 if not run */
    float df_1d;         /* 1D estimate, Angstrom */
    float phase_1d;      /* 1D estimate, degree   */
    float score_1d;      /* 1D CC                 */
    int   lowpassed;     /* 1 if the B-factor lowpass ran (variance >= 1) */
} orc_result;

/* Optics and run flags (CInput.cpp:43-58 defaults). */
typedef struct {
    float kv;              /* keV          */
    float cs_mm;           /* mm           */
    float amp_contrast;    /* fraction     */
    float pixel_size;      /* raw A/pixel  */
    float ext_phase_deg;   /* -ExtPhase v0 */
    float ext_phase_range; /* -ExtPhase v1 (search range, deg; <=0 = none) */
    int   tile_size;       /* -TileSize    */
    int   log_spect;       /* -LogSpect    */
    float held_phase;      /* CFindDefocus2D::m_fExtPhase on entry to DoIt/Refine (deg):
                              Setup3 leaves it alone, mIterate evaluates its first CC
                              and the astigmatism grid there; 0 for a search object
                              Setup1 has just created */
} orc_params;

int  orc_num_threads(int n);           /* set OpenMP threads (n<=0: keep); returns current */

/* CRescaleImage::Setup (FindCTF/CRescaleImage.cpp:47-66). */
void orc_rescale_dims(int w, int h, float px, int* new_w, int* new_h,
                      float* new_px, float* binning);
/* CRescaleImage::DoIt (FindCTF/CRescaleImage.cpp:68-99): dense new_w x new_h
 * output (row pitch new_w).  c2r_mode selects how the non-Hermitian Nyquist
 * row/column of the cropped spectrum is treated by the inverse transform
 * (0 = y-pass then Hermitian x-pass, imaginary parts of kx=0 and kx=N/2
 * dropped). */
int  orc_rescale(const float* img, int w, int h, float px, float* out, int c2r_mode);

/* Tile geometry of CGenAvgSpectrum::SetSizes (FindCTF/CGenAvgSpectrum.cpp:40-75). */
void orc_tile_layout(int w, int h, int tile, int* n_tiles_x, int* n_tiles_y,
                     int* off_x, int* off_y, int* overlap);
/* CGenAvgSpectrum::DoIt (FindCTF/CGenAvgSpectrum.cpp:77-139): raw averaged
 * amplitude spectrum, (tile/2+1) x tile, DC at (0, tile/2). */
int  orc_avg_spectrum(const float* img, int w, int h, int pitch, int tile, double* raw);
/* Taper of GRoundEdge (FindCTF/GRoundEdge.cu:7-25), tile x tile. */
void orc_taper(int tile, double* w);

/* CFindCtfBase::mRemoveBackground + mLowpass (FindCTF/CFindCtfBase.cpp:158-219).
 * raw -> ctf spectrum; returns 1 if the lowpass ran, 0 if skipped. */
int  orc_ctf_spectrum(const double* raw, int tile, int log_spect, double* ctf,
                      double* bg_out /* nullable: background estimate */);
/* GRmBackground2D only (FindCTF/GRmBackground2D.cu:11-70). */
void orc_remove_background(const double* raw, int tile, int log_spect, double* out);
/* GLowpass2D::DoBFactor applied through the full spectrum
 * (FindCTF/CFindCtfBase.cpp:191-219, FindCTF/GLowpass2D.cu:9-23). */
void orc_lowpass(const double* in, int tile, double bfactor, double* out);
/* GRadialAvg (FindCTF/GRadialAvg.cu:11-33). */
void orc_radial_average(const double* spect, int tile, double* radial);

/* Model + correlation primitives.  wl_px, cs_px in pixels; phases radian. */
void   orc_ctf1d(int n, float wl_px, float cs_px, float add_phase, float df_px, double* ctf);
double orc_cc1d(const double* ctf, const double* radial, int n, float lo, float hi, float bfac);
void   orc_ctf2d(int tile, float wl_px, float cs_px, float add_phase,
                 float df_min_px, float df_max_px, float azimuth_rad, double* ctf);
double orc_cc2d(const double* ctf, const double* spect, int tile, float lo, float hi, float bfac);

/* One package through CFindCtf2D: spectrum (already rescaled image `img`,
 * new pixel size px_n) then Do2D (mode 0) or Refine (mode 1) with
 * refine_in = {df_mean, df_range, ast, ast_range, ang, ang_range, phase, phase_range}.
 * raw/ctf/full are optional outputs. */
int orc_find_ctf_image(const float* img, int w, int h, int pitch, float px_n,
                       const orc_params* p, int mode, const float* refine_in,
                       orc_result* res, double* raw_out, double* ctf_out,
                       float* full_out);

/* Search only, on a given ctf spectrum (mode/refine_in as above). */
int orc_search(const double* ctf, int tile, float px_n, const orc_params* p,
               int mode, const float* refine_in, orc_result* res);

/* CFindCtf1D::Do1D on a given ctf spectrum (FindCTF/CFindCtf1D.cpp:49-59). */
int orc_search1d(const double* ctf, int tile, float px_n, const orc_params* p,
                 float* df, float* phase, float* score);
/* CFindCtf1D::Refine1D: refinement pass around init_df over df_range (A). */
int orc_refine1d(const double* ctf, int tile, float px_n, const orc_params* p, float init_df,
                 float df_range, float* df, float* phase, float* score);

/* CSpectrumImage (FindCTF/CSpectrumImage.cpp:21-71): tile x tile float. */
void orc_full_spectrum(const double* ctf, int tile, float px_n, const orc_params* p,
                       const orc_result* res, float* full);

/* CFindSeriesCtfs::DoIt policy (CFindSeriesCtfs.cpp:50-213) over n raw
 * images (each w x h, dense) in processing `order`; is_tomo selects the
 * tilt-series refine windows.  Results are written at res[image index]. */
int orc_series(const float* const* imgs, int n, int w, int h, const orc_params* p,
               const int* order, int is_tomo, orc_result* res);

/* GBackground1D: start bin and moving-average background of a 1D spectrum,
 * and its removal from a 1D spectrum / a half spectrum (float, in place). */
int  orc_background1d(const float* spec, int n, float* bg, int* start);
void orc_remove_bg1d(float* spec, int n, const float* bg, int bg_n, int start);
void orc_remove_bg2d(float* spec, int tile, const float* bg, int bg_n, int start);

/* Work counters: out[0] = 2D candidates (GCC2D evaluations), out[1] = 1D
 * grid points evaluated since the last reset; reset != 0 zeroes them. */
void orc_counts(long long out[2], int reset);

#ifdef __cplusplus
}
#endif
