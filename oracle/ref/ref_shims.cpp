// ref_shims.cpp -- the pieces the reference's CTF path links against that
// are not part of its source tree, written here from their declarations
// (test infrastructure; only oracle/ref/ref_driver.cpp uses them):
//
//   CuUtilFFT::GFFT2D  -> ref_fft.cu
//   Util_Thread, Util_Time (Include/Util/Util_Thread.h, Util_Time.h)
//                       -> no threads, gettimeofday
//   Mrc::CSaveMrc, CSaveImages ctor/dtor (only a static instance in
//                       FindCTF/CGenAvgSpectrum.cpp:16 is constructed)
//   CLoadImages, CAsyncSaveImages, CInputFolder (MrcUtil/CMrcUtilInc.h,
//                       CMainInc.h) -> an in-memory series supplied by the
//                       driver instead of MRC files on disk
//
// Heap allocations of the reference code are zero-filled (operator new
// below; the library links with -Bsymbolic so its own calls bind to
// them).  The path reads one member it never
// writes first -- CFindDefocus2D::m_fExtPhase, used by mIterate's first
// CC and astigmatism grid (FindCTF/CFindDefocus2D.cpp:153-165) -- so with
// a plain allocator its value is whatever the heap held.  Zero-filled, it
// is 0 for every search object Setup1 creates, as in a fresh process.
#include <cufft.h>
#include <cuda_runtime.h>
#include <new>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "CMainInc.h"
#include "FindCTF/CFindCTFInc.h"
#include "MrcUtil/CMrcUtilInc.h"
#include <Util/Util_Thread.h>
#include <Util/Util_Time.h>

#include "ref_state.h"


static void* gref_zalloc(size_t n)
{
    void* p = calloc(1, n ? n : 1);
    if (!p) throw std::bad_alloc();
    return p;
}

void* operator new(size_t n) { return gref_zalloc(n); }
void* operator new[](size_t n) { return gref_zalloc(n); }
void* operator new(size_t n, const std::nothrow_t&) noexcept { return calloc(1, n ? n : 1); }
void* operator new[](size_t n, const std::nothrow_t&) noexcept { return calloc(1, n ? n : 1); }
void operator delete(void* p) noexcept { free(p); }
void operator delete[](void* p) noexcept { free(p); }
void operator delete(void* p, size_t) noexcept { free(p); }
void operator delete[](void* p, size_t) noexcept { free(p); }

#undef cudaMalloc
cudaError_t gref_cuda_malloc(void** ptr, size_t bytes)
{
    const size_t tail = 65536;
    cudaError_t e = cudaMalloc(ptr, bytes + tail);
    if (e != cudaSuccess) return e;
    return cudaMemset(static_cast<char*>(*ptr) + bytes, 0, tail);
}

// ---------------------------------------------------------------- Util_*
Util_Thread::Util_Thread(void) : m_bCreated(false), m_bStop(false)
{
    pthread_mutex_init(&m_aMutex, 0);
    pthread_cond_init(&m_aCond, 0);
}
Util_Thread::~Util_Thread()
{
    pthread_cond_destroy(&m_aCond);
    pthread_mutex_destroy(&m_aMutex);
}
void Util_Thread::ThreadMain(void) {}
bool Util_Thread::WaitForExit(float) { return true; }

void Util_Time::Measure(void) { gettimeofday(&m_aTimeval, 0); }
float Util_Time::GetElapsedSeconds(void)
{
    timeval now;
    gettimeofday(&now, 0);
    return (float)((now.tv_sec - m_aTimeval.tv_sec) + 1e-6 * (now.tv_usec - m_aTimeval.tv_usec));
}

Mrc::CSaveMrc::CSaveMrc() : m_pSaveMain(0), m_pSaveExt(0), m_pSaveImg(0) {}
Mrc::CSaveMrc::~CSaveMrc() {}

namespace GCTFFind {

CSaveImages::CSaveImages(void) {}
CSaveImages::~CSaveImages(void) {}

// ---------------------------------------------------------------- series input
CInputFolder* CInputFolder::m_pInstance = 0L;

CInputFolder* CInputFolder::GetInstance(void)
{
    if (m_pInstance == 0L) m_pInstance = new CInputFolder;
    return m_pInstance;
}

void CInputFolder::DeleteInstance(void)
{
    delete m_pInstance;
    m_pInstance = 0L;
}

CInputFolder::CInputFolder(void) : m_ppPackages(0L), m_iNumPackages(0), m_iZeroTilt(0), m_bTomo(false)
{
    m_acDirName[0] = m_acPrefix[0] = m_acSuffix[0] = 0;
}

CInputFolder::~CInputFolder(void) { mClean(); }

void CInputFolder::mClean(void)
{
    for (int i = 0; i < m_iNumPackages; i++) delete m_ppPackages[i];
    delete[] m_ppPackages;
    m_ppPackages = 0L;
    m_iNumPackages = 0;
}

// Builds the package list from gref_series (set by the driver) instead of
// scanning the input path.
bool CInputFolder::ReadFiles(void)
{
    mClean();
    const GrefSeries& s = gref_series();
    m_iNumPackages = s.n;
    m_bTomo = s.is_tomo;
    m_iZeroTilt = s.order ? s.order[0] : 0;
    m_ppPackages = new CCtfPackage*[s.n];
    for (int i = 0; i < s.n; i++) {
        CCtfPackage* p = new CCtfPackage;
        p->m_iImgIdx = i;
        p->m_fTilt = s.tilts ? s.tilts[i] : 0.0f;
        p->m_aiImgSize[0] = s.width;
        p->m_aiImgSize[1] = s.height;
        snprintf(p->m_acMrcFileName, sizeof(p->m_acMrcFileName), "%s", s.names ? s.names[i] : "");
        m_ppPackages[i] = p;
    }
    return true;
}

bool CInputFolder::GetFileName(int iPackage, char* pcFileName)
{
    if (iPackage < 0 || iPackage >= m_iNumPackages) return false;
    strcpy(pcFileName, m_ppPackages[iPackage]->m_acMrcFileName);
    return true;
}

CCtfPackage* CInputFolder::GetPackage(int iPackage, bool bClean)
{
    CCtfPackage* p = m_ppPackages[iPackage];
    if (bClean) m_ppPackages[iPackage] = 0L;
    return p;
}

void CInputFolder::SetPackage(int iPackage, CCtfPackage* pPackage) { m_ppPackages[iPackage] = pPackage; }
int CInputFolder::GetNumPackages(void) { return m_iNumPackages; }
int CInputFolder::GetZeroTiltIdx(void) { return m_iZeroTilt; }
bool CInputFolder::IsTomo(void) { return m_bTomo; }

CLoadImages* CLoadImages::m_pInstance = 0L;

CLoadImages* CLoadImages::GetInstance(void)
{
    if (m_pInstance == 0L) m_pInstance = new CLoadImages;
    return m_pInstance;
}

void CLoadImages::DeleteInstance(void)
{
    delete m_pInstance;
    m_pInstance = 0L;
}

CLoadImages::CLoadImages(void) : m_iMode(2), m_iPixels(0) {}
CLoadImages::~CLoadImages(void) { Clean(); }

void CLoadImages::Clean(void)
{
    while (!m_aLoadedQueue.empty()) m_aLoadedQueue.pop();
}

// Queues every package in processing order with a host copy of its image
// (the loader's job in the reference: MrcUtil/CLoadImages.cpp:70-120).
void CLoadImages::AsyncLoad(void)
{
    Clean();
    const GrefSeries& s = gref_series();
    CInputFolder* folder = CInputFolder::GetInstance();
    size_t px = (size_t)s.width * s.height;
    for (int k = 0; k < s.n; k++) {
        int i = s.order ? s.order[k] : k;
        CCtfPackage* p = folder->GetPackage(i, false);
        p->m_pfImage = new float[px];
        memcpy(p->m_pfImage, s.images[i], px * sizeof(float));
        m_aLoadedQueue.push(p);
    }
}

CCtfPackage* CLoadImages::GetPackage(bool bPop)
{
    if (m_aLoadedQueue.empty()) return 0L;
    CCtfPackage* p = m_aLoadedQueue.front();
    if (bPop) m_aLoadedQueue.pop();
    return p;
}

void CLoadImages::ThreadMain(void) {}

CAsyncSaveImages* CAsyncSaveImages::m_pInstance = 0L;

CAsyncSaveImages* CAsyncSaveImages::GetInstance(void)
{
    if (m_pInstance == 0L) m_pInstance = new CAsyncSaveImages;
    return m_pInstance;
}

void CAsyncSaveImages::DeleteInstance(void)
{
    delete m_pInstance;
    m_pInstance = 0L;
}

CAsyncSaveImages::CAsyncSaveImages(void) : m_iNumPackages(0) {}
CAsyncSaveImages::~CAsyncSaveImages(void) {}

// Hands the finished package to the driver's sink (full spectrum copy)
// and frees the image, as the saver does after writing
// (MrcUtil/CAsyncSaveImages.cpp:43-80).
void CAsyncSaveImages::SetPackage(CCtfPackage* pPackage)
{
    const GrefSeries& s = gref_series();
    if (s.full_spectra && pPackage->m_pfFullSpect) {
        size_t n = (size_t)pPackage->m_aiSpectSize[0] * pPackage->m_aiSpectSize[1];
        memcpy(s.full_spectra + (size_t)pPackage->m_iImgIdx * n, pPackage->m_pfFullSpect, n * sizeof(float));
    }
    pPackage->Clean();
    m_iNumPackages += 1;
}

void CAsyncSaveImages::ThreadMain(void) {}

}  // namespace GCTFFind
