// ref_pad.h -- force-included (-include) into every translation unit of the
// reference build.  Test infrastructure only: nothing in the product links
// this.
//
// Two kernels of the reference read one row past the end of a spectrum
// buffer: GRadialAvg (FindCTF/GRadialAvg.cu:27, y reaches iCmpY for
// r = iCmpX - 1 near +90 degrees) and GCalcSpectrum's mGenFullSpect
// (FindCTF/GCalcSpectrum.cu:53, ySrc = iCmpY for yDst = 0 on the mirrored
// half), both on CFindCtfBase::m_gfFullSpect whose last quarter is
// m_gfCtfSpect (FindCTF/CFindCtfBase.cpp:58-60).  Every device allocation of
// the reference build therefore gets a zeroed tail, so those reads stay
// inside the allocation and read 0.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

cudaError_t gref_cuda_malloc(void** ptr, size_t bytes);

template <class T>
static inline cudaError_t gref_cuda_malloc(T** ptr, size_t bytes)
{
    return gref_cuda_malloc(reinterpret_cast<void**>(ptr), bytes);
}

#define cudaMalloc gref_cuda_malloc
