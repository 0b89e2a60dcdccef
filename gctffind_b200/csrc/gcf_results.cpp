// gcf_results.cpp -- result files of CSaveCtfResults (CSaveCtfResults.cpp:34-117).
//
// The CTF text file has one header line and one row per package in image
// order; tilt series additionally get "<stem>_Imod.txt" with defocus in nm.
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/gctf_b200.h"

extern "C" {

gcf_status gcf_write_ctf_file_ex(const char* path, const gcf_result* res, const float* tilts,
                                 const char* const* names, int n, int is_tomo, int flags)
{
    if (!path || !res || n <= 0 || (flags & ~GCF_CTF_COLUMN_RES)) return GCF_ERR_INVALID_ARG;
    const bool col_res = (flags & GCF_CTF_COLUMN_RES) != 0;
    FILE* f = std::fopen(path, "w");
    if (!f) return GCF_ERR_IO;
    // SaveCTF (CSaveCtfResults.cpp:34-66): 0-based image index; the opt-in
    // resolution column goes after the file name, so the reference's columns
    // keep their positions
    std::fprintf(f, col_res ? "# Idx   tilt     dfMin      dfMax   azimuth extPhase  score    fileName  ctfRes\n"
                            : "# Idx   tilt     dfMin      dfMax   azimuth extPhase  score    fileName\n");
    for (int i = 0; i < n; ++i) {
        float tilt = tilts ? tilts[i] : 0.0f;
        const char* nm = (names && names[i]) ? names[i] : "";
        std::fprintf(f, "%4d  %6.2f %10.2f %10.2f %7.2f %7.2f %8.4f  %s", i, tilt, res[i].df_min,
                     res[i].df_max, res[i].azimuth, res[i].ext_phase, res[i].score, nm);
        if (col_res) std::fprintf(f, "  %7.2f", res[i].ctf_res);
        std::fputc('\n', f);
    }
    bool ok = std::fclose(f) == 0;
    if (!ok) return GCF_ERR_IO;
    if (!is_tomo) return GCF_OK;
    // SaveImod (CSaveCtfResults.cpp:68-117): "<path up to the last dot>_Imod.txt"
    std::string imod(path);
    size_t dot = imod.find_last_of('.');
    if (dot == std::string::npos) imod += "_Imod.txt";
    else imod = imod.substr(0, dot) + "_Imod.txt";
    f = std::fopen(imod.c_str(), "w");
    if (!f) return GCF_ERR_IO;
    bool phase = res[0].ext_phase != 0;
    std::fprintf(f, phase ? "5  0  0.0  0.0  0.0  3\n" : "1  0  0.0  0.0  0.0  3\n");
    for (int i = 0; i < n; ++i) {
        float tilt = tilts ? tilts[i] : 0.0f;
        if (!phase)
            std::fprintf(f, "%4d  %4d  %7.2f  %7.2f  %8.2f  %8.2f  %7.2f\n", i + 1, i + 1, tilt, tilt,
                         res[i].df_min * 0.1f, res[i].df_max * 0.1f, res[i].azimuth);
        else
            std::fprintf(f, "%4d  %4d  %7.2f  %7.2f  %8.2f  %8.2f  %7.2f  %8.2f\n", i + 1, i + 1, tilt,
                         tilt, res[i].df_min * 0.1f, res[i].df_max * 0.1f, res[i].azimuth,
                         res[i].ext_phase);
    }
    return std::fclose(f) == 0 ? GCF_OK : GCF_ERR_IO;
}

gcf_status gcf_write_ctf_file(const char* path, const gcf_result* res, const float* tilts,
                              const char* const* names, int n, int is_tomo)
{
    return gcf_write_ctf_file_ex(path, res, tilts, names, n, is_tomo, 0);
}

}  // extern "C"
