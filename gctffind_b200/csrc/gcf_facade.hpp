// gcf_facade.hpp -- C++ classes with the reference's names and call shape
// (GCTFFind::CCTFTheory, FindCTF/CCTFTheory.cpp:69-86; GCTFFind::CFindCtf2D,
// FindCTF/CFindCTFInc.h:541-623) over the C ABI of include/gctf_b200.h, so
// code written against the reference's L2 interface compiles against the
// B200 library.  Header-only; every call forwards to libgctf_b200.so.
#pragma once

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/gctf_b200.h"

namespace GCTFFind {

class CGcfError : public std::runtime_error {
public:
    CGcfError(gcf_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    gcf_status status;
};

inline void gcf_check(gcf_status s, gcf_ctx* ctx = nullptr)
{
    if (s == GCF_OK) return;
    std::string msg = gcf_strerror(s);
    if (ctx && gcf_last_error(ctx)[0]) msg += std::string(": ") + gcf_last_error(ctx);
    throw CGcfError(s, msg);
}

// CCTFTheory (FindCTF/CCTFTheory.cpp:9-301): the CTF parameters in pixels
// and radian (gcf_ctf_param has CCTFParam's fields in order) plus the
// optics the search takes.
class CCTFTheory {
public:
    CCTFTheory() { m_param.pixel_size = 1.0f; }
    // fExtPhase in radian, as in the reference.
    void Setup(float fKv, float fCs, float fAmpContrast, float fPixelSize, float fAstTol, float fExtPhase)
    {
        gcf_check(gcf_ctf_setup(&m_param, fKv, fCs, fAmpContrast, fPixelSize, fAstTol, fExtPhase));
        m_optics.kv = fKv;
        m_optics.cs_mm = fCs;
        m_optics.amp_contrast = fAmpContrast;
        m_optics.pixel_size = fPixelSize;
        m_optics.ext_phase_deg = fExtPhase / 0.017453f;
        m_optics.ext_phase_range = 0.0f;
    }
    void SetExtPhase(float fExtPhase, bool bDegree) { gcf_check(gcf_ctf_set_ext_phase(&m_param, fExtPhase, bDegree)); }
    float GetExtPhase(bool bDegree) const { return get(gcf_ctf_get_ext_phase, bDegree ? 1 : 0); }
    void SetPixelSize(float fPixSize) { m_param.pixel_size = fPixSize; }
    void ChangePixelSize(float fNewPixSize) { gcf_check(gcf_ctf_change_pixel_size(&m_param, fNewPixSize)); }
    void SetDefocus(float fDfMin, float fDfMax, float fAstAzimuth)
    {
        gcf_check(gcf_ctf_set_defocus(&m_param, fDfMin, fDfMax, fAstAzimuth));
    }
    void SetDefocusInPixel(float fDfMin, float fDfMax, float fAstAzimuth)
    {
        gcf_check(gcf_ctf_set_defocus_px(&m_param, fDfMin, fDfMax, fAstAzimuth));
    }
    void SetParam(const gcf_ctf_param* p) { m_param = *p; }
    gcf_ctf_param* GetParam() { return &m_param; }
    float Evaluate(float fFreq, float fAzimuth) const { return get(gcf_ctf_evaluate, fFreq, fAzimuth); }
    float CalcPhaseShift(float fFreq, float fAzimuth) const { return get(gcf_ctf_phase_shift, fFreq, fAzimuth); }
    float CalcDefocus(float fAzimuth) const { return get(gcf_ctf_defocus, fAzimuth); }
    float CalcFrequency(float fPhase, float fAzimuth) const { return get(gcf_ctf_frequency, fPhase, fAzimuth); }
    float CalcNthZero(int iNthZero, float fAzimuth) const { return get(gcf_ctf_nth_zero, iNthZero, fAzimuth); }
    bool EqualTo(const CCTFTheory* other, float fDfTol) const
    {
        int eq = 0;
        gcf_check(gcf_ctf_equal(&m_param, &other->m_param, fDfTol, &eq));
        return eq != 0;
    }
    float GetPixelSize() const { return m_param.pixel_size; }
    CCTFTheory* GetCopy() const { return new CCTFTheory(*this); }

    gcf_ctf_param m_param{};
    gcf_optics m_optics{300.0f, 2.7f, 0.07f, 1.0f, 0.0f, 0.0f};

private:
    template <class F, class... A>
    float get(F fn, A... a) const
    {
        float v = 0.0f;
        gcf_check(fn(&m_param, a..., &v));
        return v;
    }
};

// CFindCtf2D: Setup1 -> Setup2 -> GenHalfSpectrum -> SetPhase -> Do2D or
// Refine -> GenFullSpectrum, with the public result members of CFindCtfBase.
class CFindCtf2D {
public:
    explicit CFindCtf2D(int iGpu = 0, int iTileSize = 512, int iLogSpect = 0)
    {
        gcf_check(gcf_create(iGpu, iTileSize, iLogSpect, &m_ctx));
    }
    ~CFindCtf2D() { gcf_destroy(m_ctx); }
    CFindCtf2D(const CFindCtf2D&) = delete;
    CFindCtf2D& operator=(const CFindCtf2D&) = delete;

    void Setup1(CCTFTheory* pCtfTheory) { m_optics = pCtfTheory->m_optics; }
    // Same object for code written against CFindCtf1D.
    void Setup2(const int* piImgSize)
    {
        m_aiImgSize[0] = piImgSize[0];
        m_aiImgSize[1] = piImgSize[1];
        gcf_check(gcf_setup(m_ctx, &m_optics, piImgSize[0], piImgSize[1]), m_ctx);
    }
    // The reference takes the device image with the row padding of an
    // in-place R2C, (width / 2 + 1) * 2 floats per row.
    void GenHalfSpectrum(const float* gfPadImg)
    {
        GenHalfSpectrum(gfPadImg, (m_aiImgSize[0] / 2 + 1) * 2, true);
    }
    void GenHalfSpectrum(const float* pfImg, int iPitch, bool bDevice)
    {
        gcf_check(gcf_gen_half_spectrum(m_ctx, pfImg, iPitch, bDevice ? 1 : 0), m_ctx);
    }
    void SetPhase(float fInitPhase, float fPhaseRange)
    {
        gcf_check(gcf_set_phase(m_ctx, fInitPhase, fPhaseRange), m_ctx);
    }
    void Do2D()
    {
        gcf_check(gcf_do2d(m_ctx, &m_result), m_ctx);
        mGetResults();
    }
    void Refine(const float afDfMean[2], const float afAstRatio[2], const float afAstAngle[2],
                const float afExtPhase[2])
    {
        gcf_check(gcf_refine(m_ctx, afDfMean, afAstRatio, afAstAngle, afExtPhase, &m_result), m_ctx);
        mGetResults();
    }
    // CFindCtf1D::Do1D / Refine1D (FindCTF/CFindCtf1D.cpp:49-67).
    void Do1D()
    {
        gcf_check(gcf_do1d(m_ctx, &m_result), m_ctx);
        mGetResults();
    }
    void Refine1D(float fInitDf, float fDfRange)
    {
        gcf_check(gcf_refine1d(m_ctx, fInitDf, fDfRange, &m_result), m_ctx);
        mGetResults();
    }
    // Caller frees with delete[] (FindCTF/CFindCtfBase.cpp:118-133).
    float* GenFullSpectrum()
    {
        int sz[2];
        GetSpectSize(sz, false);
        float* out = new float[(size_t)sz[0] * sz[1]];
        gcf_status s = gcf_gen_full_spectrum(m_ctx, &m_result, out);
        if (s != GCF_OK) {
            delete[] out;
            gcf_check(s, m_ctx);
        }
        return out;
    }
    void GetSpectSize(int* piSize, bool bHalf) { gcf_check(gcf_get_spect_size(m_ctx, piSize, bHalf ? 1 : 0), m_ctx); }
    const gcf_result& GetResult() const { return m_result; }
    gcf_ctx* GetContext() { return m_ctx; }

    float m_fDfMin = 0.0f;
    float m_fDfMax = 0.0f;
    float m_fAstAng = 0.0f;     // degree
    float m_fExtPhase = 0.0f;   // degree
    float m_fScore = 0.0f;

private:
    void mGetResults()
    {
        m_fDfMin = m_result.df_min;
        m_fDfMax = m_result.df_max;
        m_fAstAng = m_result.azimuth;
        m_fExtPhase = m_result.ext_phase;
        m_fScore = m_result.score;
    }
    gcf_ctx* m_ctx = nullptr;
    gcf_optics m_optics{300.0f, 2.7f, 0.07f, 1.0f, 0.0f, 0.0f};
    gcf_result m_result{};
    int m_aiImgSize[2] = {0, 0};
};

using CFindCtf1D = CFindCtf2D;

}  // namespace GCTFFind
