// ref_fft.cu -- CuUtilFFT::GFFT2D (declared in Include/CuUtilFFT/GFFT2D.h;
// its library, libcuutilfft.a, is not in the reference tree) written over
// cuFFT plans for the reference build.  Test infrastructure only.
#include <cufft.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include <CuUtilFFT/GFFT2D.h>

static __global__ void k_scale(cufftComplex* c, size_t n, float s)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) {
        c[i].x *= s;
        c[i].y *= s;
    }
}

namespace CuUtilFFT {

GFFT2D::GFFT2D(void) : m_cufftType(CUFFT_R2C), m_cufftPlan(0), m_aStream(0)
{
    m_aiFFTSize[0] = m_aiFFTSize[1] = 0;
}

GFFT2D::~GFFT2D(void) { DestroyPlan(); }

void GFFT2D::SetStream(cudaStream_t stream)
{
    m_aStream = stream;
    if (m_cufftPlan != 0) cufftSetStream(m_cufftPlan, stream);
}

void GFFT2D::DestroyPlan(void)
{
    if (m_cufftPlan != 0) cufftDestroy(m_cufftPlan);
    m_cufftPlan = 0;
}

// piFFTSize = real-space {nx, ny}; forward = R2C, inverse = C2R.
void GFFT2D::CreatePlan(int* piFFTSize, bool bForward)
{
    DestroyPlan();
    m_aiFFTSize[0] = piFFTSize[0];
    m_aiFFTSize[1] = piFFTSize[1];
    m_cufftType = bForward ? CUFFT_R2C : CUFFT_C2R;
    mCheckError(cufftPlan2d(&m_cufftPlan, m_aiFFTSize[1], m_aiFFTSize[0], m_cufftType), "CreatePlan");
    if (m_aStream != 0) cufftSetStream(m_cufftPlan, m_aStream);
}

// In place on a row-padded image ((nx / 2 + 1) * 2 floats per row);
// bNorm scales the transform by 1 / (nx * ny).
void GFFT2D::Forward(float* gfPadImg, bool bNorm)
{
    Forward(gfPadImg, reinterpret_cast<cufftComplex*>(gfPadImg), bNorm);
}

void GFFT2D::Forward(float* gfImg, cufftComplex* gCmp, bool bNorm)
{
    mCheckError(cufftExecR2C(m_cufftPlan, gfImg, gCmp), "Forward");
    if (bNorm) mNormalize(gCmp);
}

void GFFT2D::Inverse(cufftComplex* gCmp)
{
    Inverse(gCmp, reinterpret_cast<float*>(gCmp));
}

void GFFT2D::Inverse(cufftComplex* gCmp, float* gfImg)
{
    mCheckError(cufftExecC2R(m_cufftPlan, gCmp, gfImg), "Inverse");
}

void GFFT2D::mNormalize(cufftComplex* gCmpImg)
{
    size_t n = (size_t)(m_aiFFTSize[0] / 2 + 1) * m_aiFFTSize[1];
    float s = 1.0f / ((float)m_aiFFTSize[0] * (float)m_aiFFTSize[1]);
    k_scale<<<(unsigned)((n + 255) / 256), 256, 0, m_aStream>>>(gCmpImg, n, s);
}

void GFFT2D::mCheckError(cufftResult error, const char* pcFunc)
{
    if (error != CUFFT_SUCCESS) fprintf(stderr, "GFFT2D::%s: cuFFT error %d\n", pcFunc, (int)error);
}

}  // namespace CuUtilFFT

