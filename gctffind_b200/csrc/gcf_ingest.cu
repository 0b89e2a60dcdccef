// gcf_ingest.cu -- MRC section bytes to float on the GPU, and the copy
// kernel of the context's small uploads.
//
// CLoadImages::mToFloat (MrcUtil/CLoadImages.cpp:146-181) converts each
// section on the host after reading it; here the raw bytes cross PCIe as
// they are in the file (1, 2 or 4 bytes per pixel) and this kernel widens
// them in device memory: mode 0 and 5 unsigned char, 1 short, 6 unsigned
// short, 2 float, optionally byte-swapped (big-endian files).  One thread
// makes four consecutive output pixels from one 4-, 8- or 16-byte load.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gcf_internal.h"

namespace gcf {

namespace {

__device__ __forceinline__ float from_u16(uint32_t v, int sw, bool is_signed)
{
    uint32_t h = v & 0xFFFFu;
    if (sw) h = ((h & 0xFFu) << 8) | (h >> 8);
    return is_signed ? (float)(int16_t)h : (float)h;
}

__device__ __forceinline__ float from_f32(uint32_t v, int sw)
{
    if (sw) v = __byte_perm(v, 0, 0x0123);
    return __uint_as_float(v);
}

// Pixel i of the raw section, any mode (the ragged tail).
__device__ __forceinline__ float pixel(const unsigned char* raw, int mode, int sw, size_t i)
{
    switch (mode) {
    case 1: case 6: {
        const uint32_t v = (uint32_t)raw[2 * i] | ((uint32_t)raw[2 * i + 1] << 8);
        return from_u16(v, sw, mode == 1);
    }
    case 2: {
        const uint32_t v = (uint32_t)raw[4 * i] | ((uint32_t)raw[4 * i + 1] << 8) |
                           ((uint32_t)raw[4 * i + 2] << 16) | ((uint32_t)raw[4 * i + 3] << 24);
        return from_f32(v, sw);
    }
    default: return (float)raw[i];
    }
}

__global__ void k_mrc_to_float(const unsigned char* __restrict__ raw, int mode, int sw, size_t npx,
                               float* __restrict__ out, int vec_out)
{
    const size_t groups = npx / 4;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g <= groups;
         g += (size_t)gridDim.x * blockDim.x) {
        const size_t i0 = 4 * g;
        if (g == groups) {   // the last npx % 4 pixels
            for (size_t i = i0; i < npx; ++i) out[i] = pixel(raw, mode, sw, i);
            continue;
        }
        float4 f;
        if (mode == 1 || mode == 6) {
            const uint2 v = reinterpret_cast<const uint2*>(raw)[g];
            const bool s = mode == 1;
            f = make_float4(from_u16(v.x, sw, s), from_u16(v.x >> 16, sw, s), from_u16(v.y, sw, s),
                            from_u16(v.y >> 16, sw, s));
        } else if (mode == 2) {
            const uint4 v = reinterpret_cast<const uint4*>(raw)[g];
            f = make_float4(from_f32(v.x, sw), from_f32(v.y, sw), from_f32(v.z, sw), from_f32(v.w, sw));
        } else {
            const uint32_t v = reinterpret_cast<const uint32_t*>(raw)[g];
            f = make_float4((float)(v & 0xFFu), (float)((v >> 8) & 0xFFu), (float)((v >> 16) & 0xFFu),
                            (float)(v >> 24));
        }
        if (vec_out) {
            reinterpret_cast<float4*>(out)[g] = f;
        } else {
            out[i0] = f.x;
            out[i0 + 1] = f.y;
            out[i0 + 2] = f.z;
            out[i0 + 3] = f.w;
        }
    }
}

}  // namespace

namespace {

// dst[0, bytes) = src[0, bytes) with src in mapped page-locked host memory:
// 16-byte words where both sides allow, bytes at the ends.
__global__ void k_copy_from_host(unsigned char* __restrict__ dst, const unsigned char* __restrict__ src,
                                 size_t bytes, int vec)
{
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
    size_t done = 0;
    if (vec) {
        const size_t words = bytes / 16;
        for (size_t i = tid; i < words; i += nth)
            reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
        done = words * 16;
    }
    for (size_t i = done + tid; i < bytes; i += nth) dst[i] = src[i];
}

}  // namespace

cudaError_t launch_copy_from_host(void* dst, const void* src_mapped, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) return cudaSuccess;
    const int vec = (((uintptr_t)dst | (uintptr_t)src_mapped) % 16) == 0;
    const int blocks = (int)std::min<size_t>((bytes / 16 + 255) / 256 + 1, 148);
    k_copy_from_host<<<blocks, 256, 0, st>>>(static_cast<unsigned char*>(dst),
                                             static_cast<const unsigned char*>(src_mapped), bytes, vec);
    return cudaGetLastError();
}

cudaError_t launch_mrc_to_float(const void* raw, int mode, int swap, size_t npx, float* out, cudaStream_t st)
{
    const int mb = mrc_mode_bytes(mode);
    if (!raw || !out || mb == 0) return cudaErrorInvalidValue;
    // the vector loads need the raw section aligned to 4 pixels' bytes
    if (((uintptr_t)raw % (size_t)(4 * mb)) != 0) return cudaErrorInvalidValue;
    if (npx == 0) return cudaSuccess;
    const int vec_out = ((uintptr_t)out % 16) == 0;
    const size_t groups = npx / 4 + 1;
    const int blocks = (int)std::min<size_t>((groups + 255) / 256, 148 * 16);
    k_mrc_to_float<<<blocks, 256, 0, st>>>(static_cast<const unsigned char*>(raw), mode, swap, npx, out, vec_out);
    return cudaGetLastError();
}

}  // namespace gcf
