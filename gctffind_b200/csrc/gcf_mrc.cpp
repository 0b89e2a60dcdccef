// gcf_mrc.cpp -- MRC micrograph / tilt-series input and spectrum output.
//
// Reads the subset of the MRC format the reference consumes
// (Include/Mrcfile/CMrcFileInc.h:52-120 header layout; modes converted to
// float as CLoadImages::mToFloat does, MrcUtil/CLoadImages.cpp:146-181:
// 0 and 5 unsigned char, 1 short, 2 float, 6 unsigned short) and writes
// float32 (mode 2) stacks like CAsyncSaveImages (MrcUtil/CAsyncSaveImages.cpp:57-143).
// Tilt angles come from the extended header when it holds more than one
// float per section (CInputFolder::mReadSingle, CInputFolder.cpp:169-180):
// section k's record is (numintegers + numfloats) 4-byte words at offset
// k * record and the tilt is its first float.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/gctf_b200.h"

namespace {

struct Header {
    int32_t nx, ny, nz, mode;
    int32_t nsymbt;
    int16_t nint, nreal;
    float xlen;
    int32_t mx;
    bool swap;
};

inline uint32_t bswap32(uint32_t v)
{
    return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}
inline uint16_t bswap16(uint16_t v) { return (uint16_t)((v >> 8) | (v << 8)); }

template <class T>
T rd(const unsigned char* b, int off, bool sw)
{
    T v;
    std::memcpy(&v, b + off, sizeof(T));
    if (sw) {
        if (sizeof(T) == 4) {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            u = bswap32(u);
            std::memcpy(&v, &u, 4);
        } else if (sizeof(T) == 2) {
            uint16_t u;
            std::memcpy(&u, &v, 2);
            u = bswap16(u);
            std::memcpy(&v, &u, 2);
        }
    }
    return v;
}

bool read_header(FILE* f, Header& h)
{
    unsigned char b[1024];
    if (std::fread(b, 1, 1024, f) != 1024) return false;
    bool sw = false;
    int32_t mode = rd<int32_t>(b, 12, false);
    int32_t nx = rd<int32_t>(b, 0, false);
    if (mode < 0 || mode > 16 || nx <= 0 || nx > (1 << 20)) {
        sw = true;
        mode = rd<int32_t>(b, 12, true);
        nx = rd<int32_t>(b, 0, true);
        if (mode < 0 || mode > 16 || nx <= 0) return false;
    }
    h.swap = sw;
    h.nx = nx;
    h.ny = rd<int32_t>(b, 4, sw);
    h.nz = rd<int32_t>(b, 8, sw);
    h.mode = mode;
    h.mx = rd<int32_t>(b, 28, sw);
    h.xlen = rd<float>(b, 40, sw);
    h.nsymbt = rd<int32_t>(b, 92, sw);
    h.nint = rd<int16_t>(b, 128, sw);
    h.nreal = rd<int16_t>(b, 130, sw);
    if (h.ny <= 0 || h.nz <= 0 || h.nsymbt < 0) return false;
    return true;
}

int mode_bytes(int mode)
{
    switch (mode) {
    case 0: case 5: return 1;
    case 1: case 6: return 2;
    case 2: return 4;
    default: return 0;
    }
}

}  // namespace

namespace gcf {

// Section layout of an MRC file: dims, mode, byte order and the offset of
// section 0 (after the 1024-byte header and the extended header).
bool mrc_layout(const char* path, int dims[3], int* mode, bool* swap, long long* data_off)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    Header h;
    bool ok = read_header(f, h);
    std::fclose(f);
    if (!ok) return false;
    dims[0] = h.nx;
    dims[1] = h.ny;
    dims[2] = h.nz;
    *mode = h.mode;
    *swap = h.swap;
    *data_off = 1024LL + h.nsymbt;
    return true;
}

int mrc_mode_bytes(int mode) { return mode_bytes(mode); }

}  // namespace gcf

extern "C" {

gcf_status gcf_mrc_info(const char* path, int dims[3], int* mode, float* pixel_size,
                        int* ext_floats)
{
    if (!path || !dims) return GCF_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return GCF_ERR_IO;
    Header h;
    bool ok = read_header(f, h);
    std::fclose(f);
    if (!ok) return GCF_ERR_IO;
    dims[0] = h.nx;
    dims[1] = h.ny;
    dims[2] = h.nz;
    if (mode) *mode = h.mode;
    if (pixel_size) *pixel_size = (h.mx > 0 && h.xlen > 0) ? h.xlen / h.mx : 0.0f;
    if (ext_floats) *ext_floats = h.nreal;
    return GCF_OK;
}

gcf_status gcf_mrc_read(const char* path, int z, float* out)
{
    if (!path || !out || z < 0) return GCF_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return GCF_ERR_IO;
    Header h;
    if (!read_header(f, h) || z >= h.nz) {
        std::fclose(f);
        return h.nz > 0 && z >= h.nz ? GCF_ERR_INVALID_ARG : GCF_ERR_IO;
    }
    int mb = mode_bytes(h.mode);
    if (mb == 0) {
        std::fclose(f);
        return GCF_ERR_IO;   // mode 7 / 4-bit / complex not supported
    }
    size_t npx = (size_t)h.nx * h.ny;
    long long off = 1024LL + h.nsymbt + (long long)z * (long long)(npx * mb);
    if (fseeko(f, (off_t)off, SEEK_SET) != 0) {
        std::fclose(f);
        return GCF_ERR_IO;
    }
    std::vector<unsigned char> buf(npx * mb);
    size_t got = std::fread(buf.data(), 1, buf.size(), f);
    std::fclose(f);
    if (got != buf.size()) return GCF_ERR_IO;
    const unsigned char* b = buf.data();
    for (size_t i = 0; i < npx; ++i) {
        switch (h.mode) {
        case 0: case 5: out[i] = (float)b[i]; break;
        case 1: out[i] = (float)rd<int16_t>(b + 2 * i, 0, h.swap); break;
        case 6: out[i] = (float)rd<uint16_t>(b + 2 * i, 0, h.swap); break;
        case 2: out[i] = rd<float>(b + 4 * i, 0, h.swap); break;
        }
    }
    return GCF_OK;
}

gcf_status gcf_mrc_read_tilts(const char* path, float* tilts, int n)
{
    if (!path || !tilts || n <= 0) return GCF_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return GCF_ERR_IO;
    Header h;
    if (!read_header(f, h) || h.nreal <= 1 || h.nint < 0) {
        std::fclose(f);
        return GCF_ERR_IO;
    }
    int rec = (h.nint + h.nreal) * 4;
    std::vector<unsigned char> ext(h.nsymbt);
    if (std::fread(ext.data(), 1, ext.size(), f) != ext.size()) {
        std::fclose(f);
        return GCF_ERR_IO;
    }
    std::fclose(f);
    for (int k = 0; k < n; ++k) {
        long long o = (long long)k * rec + h.nint * 4;
        if (o + 4 > (long long)ext.size()) return GCF_ERR_IO;
        tilts[k] = rd<float>(ext.data(), (int)o, h.swap);
    }
    return GCF_OK;
}

gcf_status gcf_mrc_write(const char* path, const float* data, int nx, int ny, int nz,
                         float pixel_size)
{
    if (!path || !data || nx <= 0 || ny <= 0 || nz <= 0) return GCF_ERR_INVALID_ARG;
    unsigned char b[1024];
    std::memset(b, 0, sizeof(b));
    auto wi = [&](int off, int32_t v) { std::memcpy(b + off, &v, 4); };
    auto wf = [&](int off, float v) { std::memcpy(b + off, &v, 4); };
    wi(0, nx);
    wi(4, ny);
    wi(8, nz);
    wi(12, 2);
    wi(28, nx);
    wi(32, ny);
    wi(36, nz);
    float px = pixel_size > 0 ? pixel_size : 1.0f;
    wf(40, nx * px);
    wf(44, ny * px);
    wf(48, nz * px);
    wf(52, 90.0f);
    wf(56, 90.0f);
    wf(60, 90.0f);
    wi(64, 1);
    wi(68, 2);
    wi(72, 3);
    size_t n = (size_t)nx * ny * nz;
    double s = 0.0;
    float mn = data[0], mx = data[0];
    for (size_t i = 0; i < n; ++i) {
        s += data[i];
        if (data[i] < mn) mn = data[i];
        if (data[i] > mx) mx = data[i];
    }
    wf(76, mn);
    wf(80, mx);
    wf(84, (float)(s / n));
    wi(88, nz > 1 ? 0 : 1);
    std::memcpy(b + 208, "MAP ", 4);
    b[212] = 0x44;
    b[213] = 0x44;
    FILE* f = std::fopen(path, "wb");
    if (!f) return GCF_ERR_IO;
    bool ok = std::fwrite(b, 1, 1024, f) == 1024 && std::fwrite(data, sizeof(float), n, f) == n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GCF_OK : GCF_ERR_IO;
}

}  // extern "C"
