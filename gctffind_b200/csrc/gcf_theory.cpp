// gcf_theory.cpp -- CCTFTheory / CCTFParam host math (FindCTF/CCTFTheory.cpp,
// FindCTF/CFindCTFInc.h:8-91) behind the C ABI.  Every quantity keeps the
// reference's float/double mix so the results are bit-identical to it:
// wavelength, Cs and defocus in pixels, angles in radian, the amplitude
// phase atan(Ac / sqrt(1 - Ac^2)) in float, the phase shift in float, the
// zero-crossing quadratic in double.  Compiled with -ffp-contract=off.
#include <cmath>
#include <cstring>

#include "../../include/gctf_b200.h"

namespace {

const float kPiF = (float)(4.0 * std::atan(1.0));
const float kD2R = 0.01745329f;

// CCTFTheory::mCalcWavelength (FindCTF/CCTFTheory.cpp:283-287): 12.26 /
// sqrt(V + 0.9784e-6 V^2) Angstrom with V in volts, written in keV.
float wavelength_angstrom(float kv)
{
    double wl = 12.26 / std::sqrt(kv * 1000 + 0.9784 * kv * kv);
    return (float)wl;
}

// CCTFTheory::CalcDefocus: defocus (pixel) along an azimuth (radian).
float defocus_at(const gcf_ctf_param* p, float azimuth)
{
    float sum = p->df_max + p->df_min;
    float dif = p->df_max - p->df_min;
    double c = std::cos(2.0 * (azimuth - p->azimuth));
    return (float)(0.5 * (sum + dif * c));
}

float phase_shift(const gcf_ctf_param* p, float freq, float azimuth)
{
    float s2 = freq * freq;
    float w2 = p->wavelength * p->wavelength;
    float df = defocus_at(p, azimuth);
    return kPiF * p->wavelength * s2 * (df - 0.5f * w2 * s2 * p->cs) + p->amp_phase + p->ext_phase;
}

// CCTFTheory::CalcFrequency: smallest positive root s of the phase-shift
// quadratic in s^2.
float frequency_of(const gcf_ctf_param* p, float phase, float azimuth)
{
    float df = defocus_at(p, azimuth);
    double w3 = std::pow(p->wavelength, 3.0);
    double a = -0.5 * kPiF * w3 * p->cs;
    double b = kPiF * p->wavelength * df;
    double c = p->ext_phase + p->amp_phase;
    double det = b * b - 4.0 * a * (c - phase);
    if (p->cs == 0) {
        double f2 = (phase - c) / b;
        return f2 > 0 ? (float)std::sqrt(f2) : 0.0f;
    }
    if (det < 0.0) return 0.0f;
    double s1 = (-b + std::sqrt(det)) / (2 * a);
    double s2 = (-b - std::sqrt(det)) / (2 * a);
    if (s1 > 0) return (float)std::sqrt(s1);
    if (s2 > 0) return (float)std::sqrt(s2);
    return 0.0f;
}

}  // namespace

extern "C" {

gcf_status gcf_ctf_setup(gcf_ctf_param* p, float kv, float cs_mm, float amp_contrast, float pixel_size,
                         float ast_tol, float ext_phase_rad)
{
    if (!p || !(pixel_size > 0.0f) || !(kv > 0.0f) || amp_contrast < 0.0f || amp_contrast >= 1.0f)
        return GCF_ERR_INVALID_ARG;
    std::memset(p, 0, sizeof(*p));
    p->wavelength = wavelength_angstrom(kv) / pixel_size;
    p->cs = (float)(cs_mm * 1e7 / pixel_size);
    p->ast_tol = ast_tol / pixel_size;
    p->pixel_size = pixel_size;
    p->amp_contrast = amp_contrast;
    p->amp_phase = std::atan(amp_contrast / std::sqrt(1 - amp_contrast * amp_contrast));
    p->ext_phase = std::fmod(ext_phase_rad, kPiF);
    return GCF_OK;
}

gcf_status gcf_ctf_set_ext_phase(gcf_ctf_param* p, float phase, int degree)
{
    if (!p) return GCF_ERR_INVALID_ARG;
    if (degree) phase *= kD2R;
    p->ext_phase = std::fmod(phase, kPiF);
    return GCF_OK;
}

gcf_status gcf_ctf_get_ext_phase(const gcf_ctf_param* p, int degree, float* out)
{
    if (!p || !out) return GCF_ERR_INVALID_ARG;
    *out = degree ? p->ext_phase / kD2R : p->ext_phase;
    return GCF_OK;
}

gcf_status gcf_ctf_set_defocus(gcf_ctf_param* p, float df_min_a, float df_max_a, float azimuth_rad)
{
    if (!p) return GCF_ERR_INVALID_ARG;
    p->df_min = df_min_a / p->pixel_size;
    p->df_max = df_max_a / p->pixel_size;
    p->azimuth = azimuth_rad;
    return GCF_OK;
}

gcf_status gcf_ctf_set_defocus_px(gcf_ctf_param* p, float df_min_px, float df_max_px, float azimuth_rad)
{
    if (!p) return GCF_ERR_INVALID_ARG;
    p->df_min = df_min_px;
    p->df_max = df_max_px;
    p->azimuth = azimuth_rad;
    return GCF_OK;
}

gcf_status gcf_ctf_change_pixel_size(gcf_ctf_param* p, float new_pixel_size)
{
    if (!p || !(new_pixel_size > 0.0f)) return GCF_ERR_INVALID_ARG;
    float scale = p->pixel_size / new_pixel_size;
    if (scale == 1.0) return GCF_OK;
    p->wavelength *= scale;
    p->cs *= scale;
    p->df_max *= scale;
    p->df_min *= scale;
    p->ast_tol *= scale;
    p->pixel_size = new_pixel_size;
    return GCF_OK;
}

gcf_status gcf_ctf_evaluate(const gcf_ctf_param* p, float freq, float azimuth, float* out)
{
    if (!p || !out) return GCF_ERR_INVALID_ARG;
    float ps = phase_shift(p, freq, azimuth);
    *out = (float)(-std::sin(ps));
    return GCF_OK;
}

gcf_status gcf_ctf_phase_shift(const gcf_ctf_param* p, float freq, float azimuth, float* out)
{
    if (!p || !out) return GCF_ERR_INVALID_ARG;
    *out = phase_shift(p, freq, azimuth);
    return GCF_OK;
}

gcf_status gcf_ctf_defocus(const gcf_ctf_param* p, float azimuth, float* out)
{
    if (!p || !out) return GCF_ERR_INVALID_ARG;
    *out = defocus_at(p, azimuth);
    return GCF_OK;
}

gcf_status gcf_ctf_frequency(const gcf_ctf_param* p, float phase, float azimuth, float* out)
{
    if (!p || !out) return GCF_ERR_INVALID_ARG;
    *out = frequency_of(p, phase, azimuth);
    return GCF_OK;
}

gcf_status gcf_ctf_nth_zero(const gcf_ctf_param* p, int n, float azimuth, float* out)
{
    if (!p || !out) return GCF_ERR_INVALID_ARG;
    *out = frequency_of(p, n * kPiF, azimuth);
    return GCF_OK;
}

// CCTFTheory::EqualTo, including its extra-phase test, which takes the
// remainder of the amplitude-contrast difference rather than of the phase
// difference (FindCTF/CCTFTheory.cpp:230-258).
gcf_status gcf_ctf_equal(const gcf_ctf_param* p, const gcf_ctf_param* q, float df_tol, int* out)
{
    if (!p || !q || !out) return GCF_ERR_INVALID_ARG;
    *out = 0;
    float dif = p->df_max - q->df_max;
    if (std::fabs(dif) > df_tol) return GCF_OK;
    dif = p->df_min - q->df_min;
    if (std::fabs(dif) > df_tol) return GCF_OK;
    dif = p->cs - q->cs;
    if (std::fabs(dif) > 0.01) return GCF_OK;
    dif = p->wavelength - q->wavelength;
    if (std::fabs(dif) > 1e-4) return GCF_OK;
    dif = p->amp_contrast - q->amp_contrast;
    if (std::fabs(dif) > 1e-4) return GCF_OK;
    const float five_deg = 0.0277f;
    double d = std::fmod(dif, 2.0 * kPiF);
    if (d > five_deg) return GCF_OK;
    d = std::fabs(p->azimuth - q->azimuth);
    d = std::fmod(d, kPiF);
    if (d > five_deg) return GCF_OK;
    *out = 1;
    return GCF_OK;
}

}  // extern "C"
