/*
 * gcf_oracle.cpp -- FP64 CPU restatement of GCtfFind's CTF-estimation path.
 *
 * TEST INFRASTRUCTURE ONLY (see gcf_oracle.h).  This file restates the
 * reference algorithm in plain C++/OpenMP so that the CUDA product can be
 * checked against it; it is never linked into the product.
 *
 * Numerics policy:
 *  - every grid, step count, truncation and band membership test is
 *    evaluated in float32 exactly as the reference writes it, so candidate
 *    grids and pixel sets coincide with the reference;
 *  - FFTs, the CTF model, all sums and the correlation are evaluated in
 *    double (own radix-2 / Bluestein FFT, published Cooley-Tukey and
 *    chirp-z methods);
 *  - this file is compiled with -ffp-contract=off so float expressions are
 *    rounded operation by operation.
 *
 * Deliberate, documented deviations from the reference (all on pixels that
 * are outside every correlation band, or on uninitialised reads):
 *  - GCalcSpectrum::GenFullSpect reads half-spectrum row cmpY for y = 0
 *    (FindCTF/GCalcSpectrum.cu:64-68, one row past the buffer); the mirror
 *    row is taken modulo cmpY here.
 *  - CFindCtfBase::mLowpass copies the x = cmpX-1 column from the row
 *    padding of the in-place C2R buffer (FindCTF/CFindCtfBase.cpp:211-218);
 *    the periodic neighbour (column 0 of the full spectrum) is used here.
 *  - GRadialAvg reads row cmpY for r = cmpX-1 near +90 degrees
 *    (FindCTF/GRadialAvg.cu:23-24); the row index is clamped here.
 *  - CFindDefocus2D::mIterate correlates with an uninitialised m_fExtPhase
 *    on its first call (FindCTF/CFindDefocus2D.cpp:155); the phase passed to
 *    Setup3 is used here.
 */
#include "gcf_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

/* ------------------------------------------------------------------------ */
/* FFT: iterative radix-2 for powers of two, Bluestein chirp-z otherwise.   */
/* ------------------------------------------------------------------------ */
// Work counters (test instrumentation): 2D candidates and 1D grid points
// evaluated since the last orc_counts(..., reset = 1).
static std::atomic<long long> g_cand2d{0}, g_cand1d{0};

namespace {

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

struct Plan {
    int n = 0;
    bool pow2 = false;
    int m = 0;                 // Bluestein FFT size (power of two)
    std::vector<cd> tw;        // exp(-2 pi i k / N), k < N/2, N = n or m
    std::vector<cd> chirp;     // exp(+i pi k^2 / n), k < n
    std::vector<cd> bhat;      // FFT_m of the wrapped chirp
};

std::mutex g_plan_mutex;
std::map<int, std::shared_ptr<Plan>> g_plans;

void radix2(cd* a, int n, const std::vector<cd>& tw, int tw_n, bool inverse)
{
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1;
        int stride = tw_n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < half; ++k) {
                cd w = tw[(size_t)k * stride];
                if (inverse) w = std::conj(w);
                cd u = a[i + k];
                cd v = a[i + k + half] * w;
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
        }
    }
}

std::vector<cd> twiddles(int n)
{
    std::vector<cd> t(n / 2 > 0 ? n / 2 : 1);
    for (int k = 0; k < n / 2; ++k) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        t[k] = cd(std::cos(a), std::sin(a));
    }
    return t;
}

std::shared_ptr<Plan> get_plan(int n)
{
    std::lock_guard<std::mutex> lk(g_plan_mutex);
    auto it = g_plans.find(n);
    if (it != g_plans.end()) return it->second;
    auto p = std::make_shared<Plan>();
    p->n = n;
    p->pow2 = is_pow2(n);
    if (p->pow2) {
        p->tw = twiddles(n);
    } else {
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        p->m = m;
        p->tw = twiddles(m);
        p->chirp.resize(n);
        for (int k = 0; k < n; ++k) {
            long long k2 = ((long long)k * k) % (2LL * n);
            double a = M_PI * (double)k2 / (double)n;
            p->chirp[k] = cd(std::cos(a), std::sin(a));
        }
        p->bhat.assign(m, cd(0, 0));
        p->bhat[0] = p->chirp[0];
        for (int k = 1; k < n; ++k) {
            p->bhat[k] = p->chirp[k];
            p->bhat[m - k] = p->chirp[k];
        }
        radix2(p->bhat.data(), m, p->tw, m, false);
    }
    g_plans[n] = p;
    return p;
}

/* In-place complex DFT of length n; forward uses exp(-2 pi i jk/n).
 * Unnormalised in both directions. */
void fft(cd* a, int n, bool inverse)
{
    if (n <= 1) return;
    auto p = get_plan(n);
    if (p->pow2) {
        radix2(a, n, p->tw, n, inverse);
        return;
    }
    // Bluestein: X[k] = conj(c_k) * sum_j (x_j conj(c_j)) c_{k-j}, c_k = exp(i pi k^2/n)
    // Inverse via conj(DFT(conj(x))).
    int m = p->m;
    std::vector<cd> buf(m, cd(0, 0));
    for (int j = 0; j < n; ++j) {
        cd x = inverse ? std::conj(a[j]) : a[j];
        buf[j] = x * std::conj(p->chirp[j]);
    }
    radix2(buf.data(), m, p->tw, m, false);
    for (int k = 0; k < m; ++k) buf[k] *= p->bhat[k];
    radix2(buf.data(), m, p->tw, m, true);
    double s = 1.0 / (double)m;
    for (int k = 0; k < n; ++k) {
        cd y = buf[k] * s * std::conj(p->chirp[k]);
        a[k] = inverse ? std::conj(y) : y;
    }
}

/* Real-to-half-complex 2D transform of a w x h real image (row pitch
 * `pitch`), unnormalised; output (w/2+1) x h, row-major. */
void r2c_2d(const double* in, int w, int h, int pitch, std::vector<cd>& out)
{
    int cx = w / 2 + 1;
    out.assign((size_t)cx * h, cd(0, 0));
#pragma omp parallel
    {
        std::vector<cd> row(w);
#pragma omp for schedule(static)
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) row[x] = cd(in[(size_t)y * pitch + x], 0.0);
            fft(row.data(), w, false);
            for (int x = 0; x < cx; ++x) out[(size_t)y * cx + x] = row[x];
        }
        std::vector<cd> col(h);
#pragma omp for schedule(static)
        for (int x = 0; x < cx; ++x) {
            for (int y = 0; y < h; ++y) col[y] = out[(size_t)y * cx + x];
            fft(col.data(), h, false);
            for (int y = 0; y < h; ++y) out[(size_t)y * cx + x] = col[y];
        }
    }
}

/* Half-complex to real 2D inverse, unnormalised: inverse pass along y on
 * every kx column, then a Hermitian inverse along x in which the imaginary
 * parts of the kx = 0 and kx = w/2 bins do not contribute. */
void c2r_2d(const std::vector<cd>& in, int w, int h, double* out, int pitch)
{
    int cx = w / 2 + 1;
    std::vector<cd> tmp(in);
#pragma omp parallel
    {
        std::vector<cd> col(h);
#pragma omp for schedule(static)
        for (int x = 0; x < cx; ++x) {
            for (int y = 0; y < h; ++y) col[y] = tmp[(size_t)y * cx + x];
            fft(col.data(), h, true);
            for (int y = 0; y < h; ++y) tmp[(size_t)y * cx + x] = col[y];
        }
        std::vector<cd> row(w);
#pragma omp for schedule(static)
        for (int y = 0; y < h; ++y) {
            const cd* src = &tmp[(size_t)y * cx];
            for (int k = 0; k < cx && k < w; ++k) row[k] = src[k];
            for (int k = 1; k < (w + 1) / 2; ++k) row[w - k] = std::conj(src[k]);
            fft(row.data(), w, true);
            for (int x = 0; x < w; ++x) out[(size_t)y * pitch + x] = row[x].real();
        }
    }
}

inline float d2rf_2d() { return 0.01745329f; }   // FindCTF/CFindDefocus2D.cpp:11
inline float d2rf_1d() { return 0.0174533f; }    // FindCTF/CFindDefocus1D.cpp:11

/* Optics in pixel units as CCTFTheory::Setup stores them
 * (FindCTF/CCTFTheory.cpp:69-86, :283-287). */
struct PixOptics {
    float wl;        // wavelength, pixels
    float cs;        // Cs, pixels
    float amp_phase; // radian, GCalcCTF1D/2D::SetParam (FindCTF/GCalcCTF2D.cu:99-104)
    float px;        // Angstrom / pixel
};

PixOptics make_optics(const orc_params* p, float px_n)
{
    PixOptics o;
    double wl = 12.26 / std::sqrt((double)p->kv * 1000.0 + 0.9784 * (double)p->kv * p->kv);
    o.wl = (float)wl / px_n;
    o.cs = (float)((double)p->cs_mm * 1e7 / px_n);
    float ac = p->amp_contrast;
    o.amp_phase = (float)atanf(ac / sqrtf(1.0f - ac * ac));
    o.px = px_n;
    return o;
}

}  // namespace

/* ------------------------------------------------------------------------ */
extern "C" int orc_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* CRescaleImage::Setup, FindCTF/CRescaleImage.cpp:47-66 */
extern "C" void orc_rescale_dims(int w, int h, float px, int* new_w, int* new_h,
                                 float* new_px, float* binning)
{
    float bin = 1.2f / px;
    if (bin <= 1) bin = 1.0f;
    float pxn = px * bin;
    int nw = (int)(w / bin + 0.5f);
    int nh = (int)(h / bin + 0.5f);
    nw = nw / 2 * 2;
    nh = nh / 2 * 2;
    if (new_w) *new_w = nw;
    if (new_h) *new_h = nh;
    if (new_px) *new_px = pxn;
    if (binning) *binning = bin;
}

/* CRescaleImage::DoIt (FindCTF/CRescaleImage.cpp:68-99) with the Fourier
 * crop of GFtResize2D::DownSample (Util/GFtResize2D.cu:7-32,124-143). */
extern "C" int orc_rescale(const float* img, int w, int h, float px, float* out, int c2r_mode)
{
    (void)c2r_mode;
    int nw, nh;
    float pxn, bin;
    orc_rescale_dims(w, h, px, &nw, &nh, &pxn, &bin);
    if (bin == 1.0f) {
        for (int y = 0; y < nh; ++y)
            for (int x = 0; x < nw; ++x) out[(size_t)y * nw + x] = img[(size_t)y * w + x];
        return 0;
    }
    std::vector<double> in((size_t)w * h);
    for (size_t i = 0; i < in.size(); ++i) in[i] = img[i];
    std::vector<cd> cmp;
    r2c_2d(in.data(), w, h, w, cmp);
    int cxi = w / 2 + 1, cxo = nw / 2 + 1;
    std::vector<cd> crop((size_t)cxo * nh);
    for (int y = 0; y < nh; ++y) {
        int ys = (y > nh / 2) ? y - nh + h : y;
        for (int x = 0; x < cxo; ++x) crop[(size_t)y * cxo + x] = cmp[(size_t)ys * cxi + x];
    }
    std::vector<double> res((size_t)nw * nh);
    c2r_2d(crop, nw, nh, res.data(), nw);
    for (size_t i = 0; i < res.size(); ++i) out[i] = (float)res[i];
    return 0;
}

/* CGenAvgSpectrum::SetSizes, FindCTF/CGenAvgSpectrum.cpp:40-75 */
extern "C" void orc_tile_layout(int w, int h, int tile, int* ntx, int* nty, int* offx,
                                int* offy, int* overlap)
{
    int ov = (int)(tile * 0.50f);
    ov = ov / 2 * 2;
    int size = tile - ov;
    int nx = (w - ov) / size, ny = (h - ov) / size;
    if (ntx) *ntx = nx;
    if (nty) *nty = ny;
    if (offx) *offx = (w - nx * tile + (nx - 1) * ov) / 2;
    if (offy) *offy = (h - ny * tile + (ny - 1) * ov) / 2;
    if (overlap) *overlap = ov;
}

/* GRoundEdge mask (FindCTF/GRoundEdge.cu:7-25) with centre tile/2 and size
 * tile (FindCTF/CGenAvgSpectrum.cpp:113-117). */
extern "C" void orc_taper(int tile, double* wout)
{
    double c = tile * 0.5, s = tile;
    for (int y = 0; y < tile; ++y) {
        for (int x = 0; x < tile; ++x) {
            double fx = 2.0 * std::fabs(x - c) / s, fy = 2.0 * std::fabs(y - c) / s;
            double r = std::sqrt(fx * fx + fy * fy);
            double v = 0.0;
            if (r < 1.0) {
                double q = 0.5 * (1.0 - std::cos(M_PI * r));
                v = 1.0 - q * q * q;
            }
            wout[(size_t)y * tile + x] = v;
        }
    }
}

/* CGenAvgSpectrum::DoIt/mCalcTileSpectrum/mExtractPadTile
 * (FindCTF/CGenAvgSpectrum.cpp:77-139): per tile mean removal
 * (Util/GCalcMoment2D.cu, Util/GNormalize2D.cu), taper, R2C, amplitude with
 * the DC moved to (0, tile/2) (FindCTF/GCalcSpectrum.cu:15-31), average. */
extern "C" int orc_avg_spectrum(const float* img, int w, int h, int pitch, int tile, double* raw)
{
    int ntx, nty, offx, offy, ov;
    orc_tile_layout(w, h, tile, &ntx, &nty, &offx, &offy, &ov);
    int ntiles = ntx * nty;
    if (ntiles <= 0 || tile < 8) return -1;
    int cx = tile / 2 + 1, cy = tile;
    std::vector<double> taper((size_t)tile * tile);
    orc_taper(tile, taper.data());
    int nthr = orc_num_threads(0);
    std::vector<std::vector<double>> acc(nthr, std::vector<double>((size_t)cx * cy, 0.0));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        std::vector<double> t((size_t)tile * tile);
        std::vector<cd> rowbuf(tile), colbuf(tile), half((size_t)cx * cy);
#pragma omp for schedule(static)
        for (int it = 0; it < ntiles; ++it) {
            int tx = it % ntx, ty = it / ntx;
            int sx = offx + tx * (tile - ov), sy = offy + ty * (tile - ov);
            double sum = 0.0;
            for (int y = 0; y < tile; ++y)
                for (int x = 0; x < tile; ++x) {
                    double v = img[(size_t)(sy + y) * pitch + sx + x];
                    t[(size_t)y * tile + x] = v;
                    sum += v;
                }
            double mean = sum / ((double)tile * tile);
            for (size_t i = 0; i < t.size(); ++i) t[i] = (t[i] - mean) * taper[i];
            for (int y = 0; y < tile; ++y) {
                for (int x = 0; x < tile; ++x) rowbuf[x] = cd(t[(size_t)y * tile + x], 0.0);
                fft(rowbuf.data(), tile, false);
                for (int x = 0; x < cx; ++x) half[(size_t)y * cx + x] = rowbuf[x];
            }
            std::vector<double>& a = acc[tid];
            for (int x = 0; x < cx; ++x) {
                for (int y = 0; y < cy; ++y) colbuf[y] = half[(size_t)y * cx + x];
                fft(colbuf.data(), cy, false);
                for (int y = 0; y < cy; ++y) {
                    int yd = y + cy / 2;
                    if (yd >= cy) yd -= cy;
                    a[(size_t)yd * cx + x] += std::abs(colbuf[y]);
                }
            }
        }
    }
    for (size_t i = 0; i < (size_t)cx * cy; ++i) {
        double s = 0.0;
        for (int k = 0; k < nthr; ++k) s += acc[k][i];
        raw[i] = s / ntiles;
    }
    return ntiles;
}

/* GRmBackground2D (FindCTF/GRmBackground2D.cu:11-95) with fMinFreq = 1/15
 * (FindCTF/CFindCtfBase.cpp:162-165). */
extern "C" void orc_remove_background(const double* in, int tile, int log_spect, double* out)
{
    int cx = tile / 2 + 1, cy = tile;
    int half_x = cx - 1, half_y = cy / 2;
    float fmin = 1.0f / 15.0f;
    int box = (int)(fmin * cy);
    if (box > (0.3f * cy)) box = (int)(0.3f * cy);
    box = box / 2 * 2 + 1;
    if (box < 7) box = 7;
    int hb = box / 2;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < cy; ++y) {
        int yr = y - half_y;
        for (int x = 0; x < cx; ++x) {
            size_t i = (size_t)y * cx + x;
            float fr = x * 0.5f / (cx - 1);
            fr = sqrtf(fr * fr + yr * yr / (float)(cy * cy));
            if ((double)fr < 0.04) {
                out[i] = 0.0;
                continue;
            }
            double s = 0.0;
            for (int k = -hb; k <= hb; ++k) {
                int yy = k + yr;
                for (int j = -hb; j <= hb; ++j) {
                    int xx = j + x, ix, iy;
                    if (xx >= half_x) xx -= 2 * half_x;
                    if (xx >= 0) {
                        ix = xx;
                        iy = half_y + yy;
                    } else {
                        ix = -xx;
                        iy = half_y - yy;
                    }
                    if (iy < 0) iy += cy;
                    else if (iy >= cy) iy -= cy;
                    double v = in[(size_t)iy * cx + ix];
                    s += log_spect ? v : std::sqrt(v);
                }
            }
            s /= (double)box * box;
            if (!log_spect) s *= s;
            out[i] = in[i] - s;
        }
    }
}

/* Half -> full spectrum, DC at (tile/2, tile/2) (FindCTF/GCalcSpectrum.cu:47-69);
 * mirror row taken modulo tile. */
static void full_from_half(const double* half, int tile, double* full)
{
    int cx = tile / 2 + 1, hx = cx - 1;
    for (int y = 0; y < tile; ++y)
        for (int X = 0; X < tile; ++X) {
            int xd = X - hx, xs, ys;
            if (xd >= 0) {
                xs = xd;
                ys = y;
            } else {
                xs = -xd;
                ys = (tile - y) % tile;
            }
            full[(size_t)y * tile + X] = half[(size_t)ys * cx + xs];
        }
}

/* CFindCtfBase::mLowpass (FindCTF/CFindCtfBase.cpp:191-219) and
 * GLowpass2D::DoBFactor (FindCTF/GLowpass2D.cu:9-23,57-87). */
extern "C" void orc_lowpass(const double* in, int tile, double bfactor, double* out)
{
    int cx = tile / 2 + 1, hx = cx - 1;
    std::vector<double> full((size_t)tile * tile);
    full_from_half(in, tile, full.data());
    std::vector<cd> f;
    r2c_2d(full.data(), tile, tile, tile, f);
    double scale = -bfactor / ((double)tile * tile + (double)tile * tile);
    double norm = 1.0 / ((double)tile * tile);
    for (int y = 0; y < tile; ++y) {
        int ky = (y > tile / 2) ? y - tile : y;
        for (int x = 0; x < cx; ++x) {
            double g = std::exp(scale * ((double)x * x + (double)ky * ky)) * norm;
            f[(size_t)y * cx + x] *= g;
        }
    }
    c2r_2d(f, tile, tile, full.data(), tile);
    for (int y = 0; y < tile; ++y)
        for (int x = 0; x < cx; ++x) out[(size_t)y * cx + x] = full[(size_t)y * tile + (x + hx) % tile];
}

/* CFindCtfBase::mRemoveBackground (FindCTF/CFindCtfBase.cpp:158-189). */
extern "C" int orc_ctf_spectrum(const double* raw, int tile, int log_spect, double* ctf, double* bg_out)
{
    int cx = tile / 2 + 1, cy = tile;
    size_t n = (size_t)cx * cy;
    orc_remove_background(raw, tile, log_spect, ctf);
    if (bg_out)
        for (size_t i = 0; i < n; ++i) bg_out[i] = raw[i] - ctf[i];
    double s1 = 0.0, s2 = 0.0;
    for (size_t i = 0; i < n; ++i) {
        s1 += ctf[i];
        s2 += ctf[i] * ctf[i];
    }
    double mean = s1 / (double)n, var = s2 / (double)n - mean * mean;
    if (var < 1.0) return 0;
    std::vector<double> tmp(ctf, ctf + n);
    orc_lowpass(tmp.data(), tile, 10.0, ctf);
    return 1;
}

/* GRadialAvg (FindCTF/GRadialAvg.cu:11-33). */
extern "C" void orc_radial_average(const double* spect, int tile, double* radial)
{
    int cx = tile / 2 + 1, cy = tile;
    for (int r = 0; r < cx; ++r) {
        int np = (int)(3.1415926f * r + 0.5f);
        if (np < 1) np = 1;
        else if (np > 180) np = 180;
        float step = 180.0f / np;
        double s = 0.0;
        for (int i = 0; i < np; ++i) {
            float rad = (-90.0f + i * step) * 0.017453f;
            int x = (int)(r * cosf(rad) + 0.5f);
            int y = (int)(r * sinf(rad) + cy / 2 + 0.5f);
            if (y > cy - 1) y = cy - 1;
            if (x > cx - 1) x = cx - 1;
            s += spect[(size_t)y * cx + x];
        }
        radial[r] = s / np;
    }
}

/* GCalcCTF1D (FindCTF/GCalcCTF1D.cu:17-33). */
extern "C" void orc_ctf1d(int n, float wl, float cs, float add_phase, float df, double* ctf)
{
    for (int i = 0; i < n; ++i) {
        double s2 = (i * 0.5) / (n - 1.0);
        s2 *= s2;
        double chi = (double)add_phase + M_PI * wl * s2 * (df - 0.5 * (double)wl * wl * s2 * cs);
        ctf[i] = -std::sin(chi);
    }
}

/* GCC1D (FindCTF/GCC1D.cu:15-125). */
extern "C" double orc_cc1d(const double* ctf, const double* radial, int n, float lo, float hi, float bfac)
{
    double cc = 0, s1 = 0, s2 = 0;
    for (int x = 0; x < n; ++x) {
        if (!((float)x >= lo && (float)x < hi)) continue;
        double f = x / (n - 1.0);
        double c = (std::fabs(ctf[x]) - 0.5) * std::exp(-(double)bfac * f * f);
        double s = radial[x];
        cc += c * s;
        s1 += c * c;
        s2 += s * s;
    }
    if (s1 > 0 && s2 > 0) return cc / std::sqrt(s1 * s2);
    return 0.0;
}

/* GCalcCTF2D (FindCTF/GCalcCTF2D.cu:15-38,117-132). */
extern "C" void orc_ctf2d(int tile, float wl, float cs, float add_phase, float dfmin, float dfmax,
                          float azimuth, double* ctf)
{
    int cx = tile / 2 + 1, cy = tile;
    float mean = 0.5f * (dfmin + dfmax), sigma = 0.5f * (dfmax - dfmin);
    for (int y = 0; y < cy; ++y) {
        double fy = (double)(y - cy / 2) / cy;
        for (int x = 0; x < cx; ++x) {
            double fx = x * 0.5 / (cx - 1);
            double s2 = fx * fx + fy * fy;
            double th = std::atan(fy / (fx + 1e-30));
            double df = mean + sigma * std::cos(2.0 * (th - azimuth));
            double chi = add_phase + M_PI * wl * s2 * (df - 0.5 * s2 * (double)wl * wl * cs);
            ctf[(size_t)y * cx + x] = -std::sin(chi);
        }
    }
}

namespace {
/* Band membership of GCC2D::DoIt/mGCalc2D (FindCTF/GCC2D.cu:13-37,148-160),
 * evaluated in float. */
struct Band2D {
    float lo2, hi2;
    Band2D(float lo, float hi, int cy)
    {
        float l = lo / cy, h = hi / cy;
        if (h > 0.75f) h = 0.75f;
        lo2 = l * l;
        hi2 = h * h;
    }
    bool in(int x, int y, int cx, int cy) const
    {
        float fy = (y - cy * 0.5f) / cy;
        float fx = (0.5f * x) / (cx - 1);
        float s2 = fx * fx + fy * fy;
        return !(s2 < lo2 || s2 > hi2);
    }
};
}  // namespace

extern "C" double orc_cc2d(const double* ctf, const double* spect, int tile, float lo, float hi, float bfac)
{
    int cx = tile / 2 + 1, cy = tile;
    Band2D b(lo, hi, cy);
    double cc = 0, s1 = 0, s2 = 0;
    for (int y = 0; y < cy; ++y) {
        double fy = (y - cy * 0.5) / cy;
        for (int x = 0; x < cx; ++x) {
            if (!b.in(x, y, cx, cy)) continue;
            double fx = 0.5 * x / (cx - 1);
            double q = fx * fx + fy * fy;
            size_t i = (size_t)y * cx + x;
            double c = (std::fabs(ctf[i]) - 0.5) * std::exp(-(double)bfac * q);
            double s = spect[i];
            cc += c * s;
            s1 += c * c;
            s2 += s * s;
        }
    }
    double d = std::sqrt(s1 * s2);
    return d == 0.0 ? 0.0 : cc / d;
}

/* ------------------------------------------------------------------------ */
/* Searches                                                                 */
/* ------------------------------------------------------------------------ */
namespace {

/* Precomputed in-band pixels for fast CC2D of many candidates. */
struct Band2DPix {
    std::vector<double> s2, theta, env, spec;
    double sum_ss = 0.0;
};

Band2DPix make_band(const double* spect, int tile, float lo, float hi, float bfac)
{
    int cx = tile / 2 + 1, cy = tile;
    Band2D b(lo, hi, cy);
    Band2DPix p;
    for (int y = 0; y < cy; ++y) {
        double fy = (double)(y - cy / 2) / cy;
        for (int x = 0; x < cx; ++x) {
            if (!b.in(x, y, cx, cy)) continue;
            double fx = x * 0.5 / (cx - 1);
            double q = fx * fx + fy * fy;
            p.s2.push_back(q);
            p.theta.push_back(std::atan(fy / (fx + 1e-30)));
            p.env.push_back(std::exp(-(double)bfac * q));
            double s = spect[(size_t)y * cx + x];
            p.spec.push_back(s);
            p.sum_ss += s * s;
        }
    }
    return p;
}

/* One mCorrelate (FindCTF/CFindDefocus2D.cpp:363-380): dfmin/dfmax in
 * pixels, angles radian, add_phase = amp phase + ext phase. */
double cc_band(const Band2DPix& b, const PixOptics& o, float add_phase, float dfmin, float dfmax,
               float az)
{
    float mean = 0.5f * (dfmin + dfmax), sigma = 0.5f * (dfmax - dfmin);
    double wl = o.wl, w2cs = 0.5 * (double)o.wl * o.wl * o.cs;
    double cs_ = 0, cc_ = 0;
    size_t n = b.s2.size();
    for (size_t i = 0; i < n; ++i) {
        double q = b.s2[i];
        double df = mean + sigma * std::cos(2.0 * (b.theta[i] - az));
        double chi = add_phase + M_PI * wl * q * (df - q * w2cs);
        double c = (std::fabs(std::sin(chi)) - 0.5) * b.env[i];
        cs_ += c * b.spec[i];
        cc_ += c * c;
    }
    double d = std::sqrt(cc_ * b.sum_ss);
    return d == 0.0 ? 0.0 : cs_ / d;
}

/* CFindDefocus2D state machine (FindCTF/CFindDefocus2D.cpp:13-413). */
struct Search2D {
    const Band2DPix* band;
    PixOptics o;
    float df_mean, ast_ratio, ast_angle, ext_phase, cc_max;
    float phase_range[2], df_range[2], ast_range[2], ang_range[2];

    struct Cand {
        float ast, ang, phase, dfmean;
    };

    /* Evaluate a line of candidates in parallel, return CCs in order. */
    std::vector<float> eval(const std::vector<Cand>& c)
    {
        g_cand2d += (long long)c.size();
        std::vector<float> out(c.size());
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < (int)c.size(); ++i) out[i] = corr(c[i].dfmean, c[i].ast, c[i].ang, c[i].phase);
        return out;
    }

    float corr(float dfmean, float ast, float ang, float phase)
    {
        float ph = phase * d2rf_2d();
        float az = ang * d2rf_2d();
        float dmin = dfmean * (1.0f - ast) / o.px;   // CFindCtfHelp::CalcDfMin
        float dmax = dfmean * (1.0f + ast) / o.px;   // CFindCtfHelp::CalcDfMax
        float add = o.amp_phase + ph;
        return (float)cc_band(*band, o, add, dmin, dmax, az);
    }

    void find_astig()  // mFindAstig, :185-222
    {
        float tiny = (float)1e-20;
        float ar = ast_range[1] - ast_range[0];
        float gr = ang_range[1] - ang_range[0];
        if (ar < tiny && gr < tiny) return;
        int ns = 51, ng = 51;
        float as = ar / ns, gs = gr / ng;
        if (as < 1e-5) ns = 1;
        if (gs < 1e-5) ng = 1;
        if (ns == 1 && ng == 1) return;
        std::vector<Cand> c;
        for (int j = 0; j < ng; ++j) {
            float ang = ang_range[0] + j * gs;
            for (int i = 0; i < ns; ++i) {
                float a = ast_range[0] + i * as;
                c.push_back({a, ang, ext_phase, df_mean});
            }
        }
        std::vector<float> cc = eval(c);
        float best = (float)-1e20, ba = 0, bg = 0;
        for (size_t k = 0; k < c.size(); ++k) {
            if (cc[k] <= best) continue;
            best = cc[k];
            ba = c[k].ast;
            bg = c[k].ang;
        }
        if (best <= cc_max) return;
        ast_ratio = ba;
        ast_angle = bg;
        cc_max = best;
    }

    void refine_ast_mag(float range)  // :224-254
    {
        if (range < (float)1e-20) return;
        float lo_ = fmax(ast_ratio - range * 0.5f, ast_range[0]);
        float hi_ = fmin(ast_ratio + range * 0.5f, ast_range[1]);
        int n = 21;
        float step = (hi_ - lo_) / (n - 1);
        if (step < 0.001f) step = 0.001f;
        n = (int)((hi_ - lo_) / step) / 2 * 2 + 1;
        if (n == 1) return;
        std::vector<Cand> c;
        for (int i = 0; i < n; ++i) c.push_back({lo_ + i * step, ast_angle, ext_phase, df_mean});
        std::vector<float> cc = eval(c);
        float best = (float)-1e20, ba = 0;
        for (int i = 0; i < n; ++i) {
            if (cc[i] <= best) continue;
            best = cc[i];
            ba = c[i].ast;
        }
        if (best <= cc_max) return;
        ast_ratio = ba;
        cc_max = best;
    }

    void refine_ast_ang(float range)  // :256-286
    {
        if (range < (float)1e-20) return;
        float lo_ = fmax(ast_angle - range * 0.5f, ang_range[0]);
        float hi_ = fmin(ast_angle + range * 0.5f, ang_range[1]);
        int n = 51;
        float step = (hi_ - lo_) / (n - 1);
        if (step < 1.0f) step = 1.0f;
        n = (int)((hi_ - lo_) / step) / 2 * 2 + 1;
        if (n == 1) return;
        std::vector<Cand> c;
        for (int i = 0; i < n; ++i) c.push_back({ast_ratio, lo_ + i * step, ext_phase, df_mean});
        std::vector<float> cc = eval(c);
        float best = (float)-1e20, bg = 0;
        for (int i = 0; i < n; ++i) {
            if (cc[i] <= best) continue;
            best = cc[i];
            bg = c[i].ang;
        }
        if (best <= cc_max) return;
        ast_angle = bg;
        cc_max = best;
    }

    void refine_df_mean(float range)  // :288-322
    {
        if (range < (float)1e-30) return;
        int n = 31;
        float lo_ = fmax(df_mean - range * 0.5f, df_range[0]);
        float hi_ = fmin(df_mean + range * 0.5f, df_range[1]);
        float step = (hi_ - lo_) / n;
        if (step < 20) step = 20.0f;
        n = (int)((hi_ - lo_) / step) / 2 * 2 + 1;
        if (n == 1) return;
        std::vector<Cand> c;
        for (int i = 0; i < n; ++i) c.push_back({ast_ratio, ast_angle, ext_phase, lo_ + i * step});
        std::vector<float> cc = eval(c);
        float best = (float)-1e20, bd = 0;
        for (int i = 0; i < n; ++i) {
            if (cc[i] <= best) continue;
            bd = c[i].dfmean;
            best = cc[i];
        }
        if (best <= cc_max) return;
        df_mean = bd;
        cc_max = best;
    }

    void refine_phase(float range)  // :324-361
    {
        if (range < (float)1e-30) return;
        int n = 61;
        float step = range / n;
        if (step < 0.03f) return;
        if (step > 1.0f) {
            step = 1.0f;
            n = (int)(range / step);
            n = n / 2 * 2 + 1;
        }
        float pmin = phase_range[0] - phase_range[1] * 0.5f;
        float pmax = phase_range[0] + phase_range[1] * 0.5f;
        if (pmin < 0) pmin = 0.0f;
        if (pmax > 150) pmax = 150.0f;
        std::vector<Cand> c;
        for (int i = 0; i < n; ++i) {
            float ph = ext_phase + (i - n / 2) * step;
            if (ph < pmin || ph > pmax) continue;
            c.push_back({ast_ratio, ast_angle, ph, df_mean});
        }
        std::vector<float> cc = eval(c);
        float best = (float)-1e20, bp = 0;
        for (size_t i = 0; i < c.size(); ++i) {
            if (cc[i] <= best) continue;
            bp = c[i].phase;
            best = cc[i];
        }
        if (best <= cc_max) return;
        ext_phase = bp;
        cc_max = best;
    }

    void iterate()  // mIterate, :153-183
    {
        cc_max = corr(df_mean, ast_ratio, ast_angle, ext_phase);
        g_cand2d += 1;
        float old = cc_max;
        find_astig();
        if (old > cc_max) return;
        const int iters = 20;
        ext_phase = phase_range[0];
        float dfr = df_range[1] - df_range[0];
        float ar = ast_range[1] - ast_range[0];
        float gr = ang_range[1] - ang_range[0];
        for (int i = 1; i < iters; ++i) {
            float scale = 1.0f - i * 0.5f / iters;
            refine_ast_mag(scale * ar);
            if (old > cc_max) return;
            cc_max = old;
            refine_ast_ang(scale * gr);
            refine_df_mean(scale * dfr);
            refine_phase(scale * phase_range[1]);
        }
    }
};

/* GSpectralCC2D (FindCTF/GSpectralCC2D.cu:12-173) via mCalcCtfRes
 * (FindCTF/CFindDefocus2D.cpp:382-400). */
float ctf_resolution(const double* spect, int tile, const PixOptics& o, float dfmean, float ast,
                     float ang, float phase)
{
    int cx = tile / 2 + 1, cy = tile;
    float dmin = dfmean * (1.0f - ast) / o.px, dmax = dfmean * (1.0f + ast) / o.px;
    std::vector<double> ctf((size_t)cx * cy);
    orc_ctf2d(tile, o.wl, o.cs, o.amp_phase + phase * d2rf_2d(), dmin, dmax, ang * d2rf_2d(),
              ctf.data());
    const int width = 10;
    std::vector<float> cc(cx, 0.0f);
    for (int b = 0; b < cx; ++b) {
        int lo = b - width / 2, hi = lo + width;
        if (lo < 0) {
            lo = 0;
            hi = width;
        } else if (hi > cx) {
            lo = cx - width;
            hi = cx;
        }
        double scs = 0, mc = 0, ms = 0, sc = 0, ss = 0, cnt = 0;
        for (int y = 0; y < cy; ++y) {
            float fy = fabsf(y - cy * 0.5f);
            if (fy >= hi) continue;
            for (int x = 0; x < cx && x < hi; ++x) {
                float r = sqrtf((float)(x * x) + fy * fy);
                if (r < lo || r >= hi) continue;
                size_t i = (size_t)y * cx + x;
                double c = ctf[i], s = spect[i];
                mc += c;
                ms += s;
                scs += c * s;
                sc += c * c;
                ss += s * s;
                cnt += 1;
            }
        }
        if (cnt == 0) continue;
        mc /= cnt;
        ms /= cnt;
        scs /= cnt;
        sc /= cnt;
        ss /= cnt;
        sc -= mc * mc;
        ss -= ms * ms;
        if (sc <= 0 || ss <= 0) continue;
        cc[b] = (float)((scs - mc * ms) / std::sqrt(sc * ss));
    }
    int imax = 1;
    float fmx = (float)-1e30;
    for (int i = 1; i < cx; ++i) {
        if (cc[i] <= fmx) continue;
        fmx = cc[i];
        imax = i;
    }
    int shell = imax;
    if (!(fmx < 0.143f)) {
        for (int i = imax; i < cx; ++i) {
            if (cc[i] < 0.143f) break;
            shell = i;
        }
    }
    return cy * o.px / shell;
}

/* CFindDefocus1D::mBrutalForceSearch (FindCTF/CFindDefocus1D.cpp:76-137). */
void brute_1d(const double* radial, int cx, const PixOptics& o, const float res_range[2],
              const float df_range[2], const float ph_range[2], float out[3])
{
    int ndf = 501;
    float dfr = df_range[1] - df_range[0];
    float dfs = dfr / (ndf - 1);
    if (dfs < 10) dfs = 10.0f;
    ndf = (int)(dfr / dfs) / 2 * 2 + 1;
    int nps = 37;
    float psr = ph_range[1] - ph_range[0];
    float pss = psr / (nps - 1);
    if (pss == 0) nps = 1;
    else nps = (int)(psr / pss) / 2 * 2 + 1;
    int npts = ndf * nps;
    g_cand1d += npts;
    float res1 = ((cx - 1) * 2) * o.px;
    float lo = res1 / res_range[0], hi = res1 / res_range[1];
    std::vector<float> cc(npts), dfv(npts), phv(npts);
#pragma omp parallel
    {
        std::vector<double> ctf(cx);
#pragma omp for schedule(static)
        for (int i = 0; i < npts; ++i) {
            int f = i % ndf, p = i / ndf;
            float df = df_range[0] + f * dfs;
            float ph = ph_range[0] + p * pss;
            if (ph < 0) ph = 0.0f;
            else if (ph > 150.0f) ph = 150.0f;
            float ph_rad = ph * d2rf_1d();
            float pdf = df / o.px;
            orc_ctf1d(cx, o.wl, o.cs, o.amp_phase + ph_rad, pdf, ctf.data());
            cc[i] = (float)orc_cc1d(ctf.data(), radial, cx, lo, hi, 1.0f);
            dfv[i] = df;
            phv[i] = ph;
        }
    }
    out[0] = 0.0f;
    out[1] = 0.0f;
    out[2] = (float)-1e20;
    for (int i = 0; i < npts; ++i) {
        if (cc[i] > out[2]) {
            out[0] = dfv[i];
            out[1] = phv[i];
            out[2] = cc[i];
        }
    }
}

/* CFindCtfBase::Setup1 resolution range (FindCTF/CFindCtfBase.cpp:64-68). */
void res_range_of(float px, float r[2])
{
    r[0] = 25.0f * px;
    r[1] = (2.0f * px) / 0.8f;
    if (r[1] < 3.5f) r[1] = 3.5f;
}

}  // namespace

/* CFindCtf1D::Do1D/mFindDefocus/mRefineDefocus (FindCTF/CFindCtf1D.cpp:49-111). */
extern "C" int orc_search1d(const double* ctf, int tile, float px_n, const orc_params* p,
                            float* df, float* phase, float* score)
{
    int cx = tile / 2 + 1;
    PixOptics o = make_optics(p, px_n);
    float rr[2];
    res_range_of(px_n, rr);
    std::vector<double> radial(cx);
    orc_radial_average(ctf, tile, radial.data());
    float ext = p->ext_phase_deg;
    float prange = fmaxf(p->ext_phase_range, 0.0f);
    float px2 = px_n * px_n;
    float dfr[2] = {3000.0f * px2, 30000.0f * px2};
    float phr[2];
    phr[0] = fmax(ext - prange / 2, 0.0f);
    phr[1] = fmin(phr[0] + prange, 150.0f);
    float out[3];
    brute_1d(radial.data(), cx, o, rr, dfr, phr, out);
    float dfmin = out[0], ext1 = out[1];
    // mRefineDefocus(max(0.3*dfmin, 3000))
    float range = fmaxf(0.3f * dfmin, 3000.0f);
    float mindf = 3000.0f * px_n * px_n;
    float dfr2[2];
    dfr2[0] = fmaxf(dfmin - range / 2, mindf);
    dfr2[1] = dfr2[0] + range;
    float pr = 0.2f * prange;
    float phr2[2] = {0.0f, 0.0f};
    phr2[0] = fmax(ext1 - pr / 2, 0.0f);
    phr2[1] = fmin(phr2[1] + pr, 150.0f);   // reads the zero-initialised [1]
    brute_1d(radial.data(), cx, o, rr, dfr2, phr2, out);
    *df = out[0];
    *phase = out[1];
    *score = out[2];
    return 0;
}

/* CFindCtf1D::Refine1D (FindCTF/CFindCtf1D.cpp:58-67): the refinement pass
 * alone around init_df, centred on the current extra phase. */
extern "C" int orc_refine1d(const double* ctf, int tile, float px_n, const orc_params* p,
                            float init_df, float df_range, float* df, float* phase, float* score)
{
    int cx = tile / 2 + 1;
    PixOptics o = make_optics(p, px_n);
    float rr[2];
    res_range_of(px_n, rr);
    std::vector<double> radial(cx);
    orc_radial_average(ctf, tile, radial.data());
    float prange = fmaxf(p->ext_phase_range, 0.0f);
    float mindf = 3000.0f * px_n * px_n;
    float dfr2[2];
    dfr2[0] = fmaxf(init_df - df_range / 2, mindf);
    dfr2[1] = dfr2[0] + df_range;
    float pr = 0.2f * prange;
    float phr2[2] = {0.0f, 0.0f};
    phr2[0] = fmax(p->ext_phase_deg - pr / 2, 0.0f);
    phr2[1] = fmin(phr2[1] + pr, 150.0f);   // reads the zero-initialised [1]
    float out[3];
    brute_1d(radial.data(), cx, o, rr, dfr2, phr2, out);
    *df = out[0];
    *phase = out[1];
    *score = out[2];
    return 0;
}

extern "C" int orc_search(const double* ctf, int tile, float px_n, const orc_params* p, int mode,
                          const float* refine_in, orc_result* res)
{
    PixOptics o = make_optics(p, px_n);
    float rr[2];
    res_range_of(px_n, rr);
    int cy = tile;
    // CFindDefocus2D::Setup2 (FindCTF/CFindDefocus2D.cpp:86-92)
    float res1 = cy * px_n;
    float lo = res1 / rr[0], hi = res1 / rr[1];
    Band2DPix band = make_band(ctf, tile, lo, hi, 16.0f);
    Search2D s;
    s.band = &band;
    s.o = o;
    std::memset(res, 0, sizeof(*res));
    if (mode == 0) {
        float df1, ph1, sc1;
        orc_search1d(ctf, tile, px_n, p, &df1, &ph1, &sc1);
        res->df_1d = df1;
        res->phase_1d = ph1;
        res->score_1d = sc1;
        // CFindCtf2D::Do2D (FindCTF/CFindCtf2D.cpp:44-53), CFindDefocus2D::DoIt (:110-124)
        s.df_mean = (df1 + df1) * 0.5f;
        s.ast_ratio = 0.0f;
        s.ast_angle = 0.0f;
        s.phase_range[0] = ph1;
        s.ext_phase = p->held_phase;   // mIterate replaces it by phase_range[0] after mFindAstig
        s.phase_range[1] = fmaxf(p->ext_phase_range, 0.0f);
        s.df_range[0] = s.df_mean * 0.9f;
        s.df_range[1] = s.df_mean * 1.1f;
        s.ast_range[0] = 0.0f;
        s.ast_range[1] = 0.06f;
        s.ang_range[0] = -90.0f;
        s.ang_range[1] = 90.0f;
    } else {
        // CFindCtf2D::Refine (FindCTF/CFindCtf2D.cpp:55-66), CFindDefocus2D::Refine (:126-151)
        s.df_mean = refine_in[0];
        s.ast_ratio = refine_in[2];
        s.ast_angle = refine_in[4];
        s.phase_range[0] = refine_in[6];
        s.ext_phase = p->held_phase;
        float h = 0.5f * refine_in[1];
        s.df_range[0] = fmaxf(s.df_mean - h, 3000.0f);
        s.df_range[1] = s.df_mean + h;
        h = 0.5f * refine_in[3];
        s.ast_range[0] = fmaxf(s.ast_ratio - h, 0.0f);
        s.ast_range[1] = fminf(s.ast_ratio + h, 0.02f);
        h = 0.5f * refine_in[5];
        s.ang_range[0] = fmaxf(s.ast_angle - h, -90.0f);
        s.ang_range[1] = fminf(s.ast_angle + h, 90.0f);
        s.phase_range[1] = refine_in[7];
    }
    s.iterate();
    // mGetResults / getters (FindCTF/CFindCtf2D.cpp:68-76, CFindDefocus2D.cpp:38-68)
    res->df_min = s.df_mean * (1.0f - s.ast_ratio);
    res->df_max = s.df_mean * (1.0f + s.ast_ratio);
    res->azimuth = s.ast_angle;
    res->ext_phase = s.ext_phase;
    res->score = s.cc_max;
    res->ctf_res = ctf_resolution(ctf, tile, o, s.df_mean, s.ast_ratio, s.ast_angle, s.ext_phase);
    return 0;
}

/* CSpectrumImage::DoIt (FindCTF/CSpectrumImage.cpp:21-71) with
 * GCalcCTF2D::EmbedCtf (FindCTF/GCalcCTF2D.cu:49-78). */
extern "C" void orc_full_spectrum(const double* ctf, int tile, float px_n, const orc_params* p,
                                  const orc_result* res, float* full_out)
{
    int cx = tile / 2 + 1, cy = tile, hx = cx - 1;
    std::vector<double> full((size_t)tile * tile);
    full_from_half(ctf, tile, full.data());
    size_t n = (size_t)cx * cy;
    double s1 = 0, s2 = 0;
    for (size_t i = 0; i < n; ++i) {
        s1 += ctf[i];
        s2 += ctf[i] * ctf[i];
    }
    double mean = s1 / n, var = s2 / n - mean * mean;
    double sd = var < 0 ? 0.0 : std::sqrt(var);
    PixOptics o = make_optics(p, px_n);
    float rr[2];
    res_range_of(px_n, rr);
    float fmn = px_n / rr[0], fmx = px_n / rr[1];
    double gain = sd * 1.5;
    // CFindCtfBase::GenFullSpectrum (FindCTF/CFindCtfBase.cpp:118-133)
    float ast_rad = res->azimuth * 0.017453f;
    float dmin = res->df_min / px_n, dmax = res->df_max / px_n;
    float ph = fmodf(res->ext_phase * d2rf_2d(), (float)(4.0 * atan(1.0)));
    std::vector<double> c(n);
    orc_ctf2d(tile, o.wl, o.cs, o.amp_phase + ph, dmin, dmax, ast_rad, c.data());
    for (int y = 0; y < cy; ++y) {
        float fy = (y - cy * 0.5f) / cy;
        for (int bx = 0; bx < hx; ++bx) {
            float fx = (bx - (float)hx) * 0.5f / hx;
            float r = sqrtf(fx * fx + fy * fy);
            if (r < fmn || r > fmx) continue;
            int ix = hx - bx, iy = (cy - y) % cy;
            double v = std::fabs(c[(size_t)iy * cx + ix]);
            full[(size_t)y * tile + bx] = (v - 0.5) * gain + mean;
        }
    }
    for (size_t i = 0; i < full.size(); ++i) full_out[i] = (float)full[i];
}

extern "C" int orc_find_ctf_image(const float* img, int w, int h, int pitch, float px_n,
                                  const orc_params* p, int mode, const float* refine_in,
                                  orc_result* res, double* raw_out, double* ctf_out, float* full_out)
{
    int tile = p->tile_size;
    int cx = tile / 2 + 1, cy = tile;
    size_t n = (size_t)cx * cy;
    std::vector<double> raw(n), ctf(n);
    if (orc_avg_spectrum(img, w, h, pitch, tile, raw.data()) <= 0) return -1;
    int lp = orc_ctf_spectrum(raw.data(), tile, p->log_spect, ctf.data(), nullptr);
    orc_search(ctf.data(), tile, px_n, p, mode, refine_in, res);
    res->lowpassed = lp;
    if (raw_out) std::memcpy(raw_out, raw.data(), n * sizeof(double));
    if (ctf_out) std::memcpy(ctf_out, ctf.data(), n * sizeof(double));
    if (full_out) orc_full_spectrum(ctf.data(), tile, px_n, p, res, full_out);
    return 0;
}

/* CFindSeriesCtfs::DoIt/mProcessPackage/mProcessFull/mProcessRefine
 * (CFindSeriesCtfs.cpp:50-213). */
extern "C" int orc_series(const float* const* imgs, int n, int w, int h, const orc_params* p,
                          const int* order, int is_tomo, orc_result* res)
{
    int nw, nh;
    float pxn, bin;
    orc_rescale_dims(w, h, p->pixel_size, &nw, &nh, &pxn, &bin);
    std::vector<float> scaled((size_t)nw * nh);
    int ref = -1;
    for (int k = 0; k < n; ++k) {
        int idx = order[k];
        orc_rescale(imgs[idx], w, h, p->pixel_size, scaled.data(), 0);
        orc_result* r = &res[idx];
        bool full = (k == 0);
        orc_params pk = *p;    // CFindSeriesCtfs::mSetupFindCtf: Setup1 per package
        pk.held_phase = 0.0f;
        if (!full) {
            const orc_result* rp = &res[ref];
            float rin[8] = {0};
            float dmin = rp->df_min, dmax = rp->df_max;
            float dfr = 5000.0f * p->pixel_size * p->pixel_size;
            rin[0] = 0.5f * (dmin + dmax);
            rin[1] = fmaxf(rin[0] * 0.5f, dfr);
            // CFindCtfHelp::CalcAstRatio (FindCTF/CFindCtfHelp.cpp:5-12)
            float diff = (dmax - dmin) * 0.5f, mean = (dmax + dmin) * 0.5f;
            rin[2] = mean <= 0.0f ? 0.0f : diff / mean;
            rin[4] = rp->azimuth;
            rin[6] = rp->ext_phase;
            if (!is_tomo) {
                rin[3] = 0.04f;
                rin[5] = 30.0f;
                if (p->ext_phase_range > 0) rin[7] = 40.0f;
            }
            if (orc_find_ctf_image(scaled.data(), nw, nh, nw, pxn, &pk, 1, rin, r, nullptr, nullptr,
                                   nullptr))
                return -1;
            if (res[ref].score < r->score) ref = idx;
            if (r->score <= 0) full = true;
        }
        if (full) {
            // Setup1 made a new search object for this package; a fallback
            // after a refine reuses it and starts at the refine's phase
            orc_params pf = pk;
            if (k > 0) pf.held_phase = r->ext_phase;
            if (orc_find_ctf_image(scaled.data(), nw, nh, nw, pxn, &pf, 0, nullptr, r, nullptr,
                                   nullptr, nullptr))
                return -1;
            ref = idx;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* GBackground1D (FindCTF/GBackground1D.cu:13-169)                          */
/* ------------------------------------------------------------------------ */

/* DoIt + mFindStart (:95-169): double line fit over [n/5, n - n/5), first
 * bin from 2 where the spectrum is at or below the line, moving average of
 * width start/2*2-1 mirrored at the end. */
extern "C" int orc_background1d(const float* spec, int n, float* bg, int* start_out)
{
    if (n <= 0) return -1;
    int i0 = n / 5, i1 = n - i0;
    double dx = 0, dy = 0, dx2 = 0, dxy = 0;
    for (int i = i0; i < i1; ++i) {
        dx += i;
        dx2 += (i * i);
        dy += spec[i];
        dxy += (i * spec[i]);
    }
    int cnt = i1 - i0;
    dx /= cnt;
    dy /= cnt;
    dx2 /= cnt;
    dxy /= cnt;
    double a = (dx * dy - dxy) / (dx * dx - dx2);
    double b = dy - a * dx;
    int start = i0;
    for (int i = 2; i < n; ++i) {
        double y = a * i + b;
        if (y < spec[i]) continue;
        start = i;
        break;
    }
    int win = start / 2 * 2 - 1;
    for (int i = 0; i < n; ++i) {
        if (i < start) {
            bg[i] = 0.0f;
            continue;
        }
        float m = 0.0f;
        for (int j = 0; j < win; ++j) {
            int k = i + j - win / 2;
            if (k >= n) k = 2 * n - 1 - k;
            m += spec[k];
        }
        bg[i] = m / win;
    }
    *start_out = start;
    return 0;
}

/* Remove1D (:13-30): bins >= bg_n are left alone (the reference sends them
 * all to bin bg_n - 1 at once, a write race). */
extern "C" void orc_remove_bg1d(float* spec, int n, const float* bg, int bg_n, int start)
{
    for (int i = 0; i < n; ++i) {
        if (i < start) spec[i] = 0.0f;
        else if (i < bg_n) spec[i] -= bg[i];
    }
}

/* Remove2D (:32-59) on a tile x (tile/2+1) half spectrum. */
extern "C" void orc_remove_bg2d(float* spec, int tile, const float* bg, int bg_n, int start)
{
    int cx = tile / 2 + 1;
    for (int y = 0; y < tile; ++y) {
        int yc = y - tile / 2;
        for (int x = 0; x < cx; ++x) {
            float* v = spec + (size_t)y * cx + x;
            float r = sqrtf((float)(x * x + yc * yc));
            if (r < start) {
                *v = 0.0f;
                continue;
            }
            if (r >= (bg_n - 1)) {
                *v -= bg[bg_n - 1];
                continue;
            }
            int ir = (int)r;
            *v -= bg[ir] * (ir + 1 - r) + bg[ir + 1] * (r - ir);
        }
    }
}

extern "C" void orc_counts(long long out[2], int reset)
{
    out[0] = g_cand2d.load();
    out[1] = g_cand1d.load();
    if (reset) {
        g_cand2d = 0;
        g_cand1d = 0;
    }
}
