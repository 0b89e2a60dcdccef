// gcf_cli.cpp -- the GCtfFind command line on the B200 library.
//
// Same flags, defaults and input discovery as the reference
// (CInput.cpp:25-179, Util/CParseArgs.cpp:25-94, CInputFolder.cpp:131-294,
// CLoadAngFile.cpp:43-71), the same package policy (CFindSeriesCtfs.cpp:50-213:
// the first package gets the full search, every later one is refined around
// the best-scoring earlier one, zero tilt first for tilt series) and the same
// output files (CSaveCtfResults.cpp:34-117, MrcUtil/CAsyncSaveImages.cpp:57-143).
// Tilt series and equal-sized folders run as one batched gcf_run_series call;
// folders of mixed sizes run package by package through the CFindCtf2D facade.
#include <dirent.h>
#include <strings.h>
#include <sys/stat.h>
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gctf_b200.h"
#include "gcf_facade.hpp"

namespace {

double now_s()
{
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

// CParseArgs (Util/CParseArgs.cpp:25-94): case-insensitive tag, followed by
// the run of arguments that parse completely as numbers.
struct Args {
    int argc;
    char** argv;
    bool find(const char* tag, int range[2]) const
    {
        range[0] = -1;
        range[1] = 0;
        for (int i = 1; i < argc; ++i)
            if (strcasecmp(argv[i], tag) == 0) {
                range[0] = i + 1;
                break;
            }
        if (range[0] == -1) return false;
        for (int j = range[0]; j < argc; ++j) {
            char* end = nullptr;
            std::strtod(argv[j], &end);
            if (end != argv[j] && *end == '\0') {
                ++range[1];
                continue;
            }
            std::strtol(argv[j], &end, 0);
            if (end != argv[j] && *end == '\0') {
                ++range[1];
                continue;
            }
            break;
        }
        return true;
    }
    void str(const char* tag, std::string& out) const
    {
        int r[2];
        find(tag, r);
        if (r[0] > 0 && r[0] < argc) out = argv[r[0]];
    }
    void floats(const char* tag, float* v, int maxn) const
    {
        int r[2];
        find(tag, r);
        if (r[0] == -1) return;
        int n = std::min(r[1], maxn);
        for (int i = 0; i < n && r[0] + i < argc; ++i) std::sscanf(argv[r[0] + i], "%f", v + i);
    }
    void ints(const char* tag, int* v) const
    {
        int r[2];
        find(tag, r);
        if (r[0] == -1 || r[1] == 0 || r[0] >= argc) return;
        std::sscanf(argv[r[0]], "%d", v);
    }
};

// CInput (CInput.cpp:43-58 defaults, :113-179 parsing).
struct Input {
    std::string in_mrc, out_mrc, out_ctf, ang_file, in_suffix;
    float kv = 300.0f, cs = 2.7f, ac = 0.07f, px = 1.0f;
    float ext_phase[2] = {0.0f, 0.0f}, tilt_range[2] = {0.0f, 0.0f};
    int tile = 512, log_spect = 0, gpu = 0, serial = 0;
    int ctf_res = 0;   // 1: the CTF file gets the spectral-CC resolution column

    void parse(int argc, char** argv)
    {
        Args a{argc, argv};
        a.str("-InMrc", in_mrc);
        a.str("-OutMrc", out_mrc);
        a.str("-OutCtf", out_ctf);
        a.str("-InSuffix", in_suffix);
        a.str("-AngFile", ang_file);
        a.floats("-kV", &kv, 1);
        a.floats("-Cs", &cs, 1);
        a.floats("-AmpContrast", &ac, 1);
        a.floats("-PixSize", &px, 1);
        a.floats("-ExtPhase", ext_phase, 2);
        if (ext_phase[1] < 0) ext_phase[1] = 0.0f;
        a.floats("-TiltRange", tilt_range, 2);
        tilt_range[0] = std::fmax(tilt_range[0], -70.1f);
        tilt_range[1] = std::fmin(tilt_range[1], 70.1f);
        a.ints("-TileSize", &tile);
        a.ints("-LogSpect", &log_spect);
        a.ints("-Serial", &serial);
        a.ints("-Gpu", &gpu);
        a.ints("-CtfRes", &ctf_res);
    }
    void print() const
    {
        std::printf("\n");
        std::printf("%-15s  %s\n", "-InMrc", in_mrc.c_str());
        std::printf("%-15s  %s\n", "-InSuffix", in_suffix.c_str());
        std::printf("%-15s  %s\n", "-OutMrc", out_mrc.c_str());
        std::printf("%-15s  %s\n", "-OutCtf", out_ctf.c_str());
        std::printf("%-15s  %s\n", "-AngFile", ang_file.c_str());
        std::printf("%-15s  %f\n", "-kV", kv);
        std::printf("%-15s  %f\n", "-Cs", cs);
        std::printf("%-15s  %f\n", "-AmpContrast", ac);
        std::printf("%-15s  %f\n", "-PixSize", px);
        std::printf("%-15s  %f  %f\n", "-ExtPhase", ext_phase[0], ext_phase[1]);
        std::printf("%-15s  %d\n", "-TileSize", tile);
        std::printf("%-15s  %.2f  %.2f\n", "-TiltRange", tilt_range[0], tilt_range[1]);
        std::printf("%-15s  %d\n", "-LogSpect", log_spect);
        std::printf("%-15s  %d\n", "-Serial", serial);
        std::printf("%-15s  %d\n", "-Gpu", gpu);
        if (ctf_res) std::printf("%-15s  %d\n", "-CtfRes", ctf_res);
        std::printf("\n");
    }
};

void show_help()
{
    std::printf(
        "GCtfFind (B200) -- CTF estimation of cryo-EM micrographs and cryo-ET tilt series.\n\n"
        "-InMrc        input MRC: one micrograph, a tilt series stack, or with -Serial 1\n"
        "              the path prefix of the files to process\n"
        "-OutMrc       output MRC of the diagnostic spectra (a stack for a tilt series)\n"
        "-OutCtf       output text file of the estimated CTF, one row per image\n"
        "-AngFile      text file with one tilt angle per line, in stack order (optional)\n"
        "-TiltRange    min and max tilt of a series collected with a fixed step\n"
        "-kV           high tension in keV (300)\n"
        "-Cs           spherical aberration in mm (2.7)\n"
        "-AmpContrast  amplitude contrast (0.07)\n"
        "-PixSize      pixel size in A (1.0)\n"
        "-ExtPhase     extra phase shift and its search range in degrees (0 0)\n"
        "-TileSize     tile size of the averaged spectrum (512)\n"
        "-LogSpect     1: background from the spectrum instead of its square root\n"
        "-InSuffix     with -Serial 1, only files whose names end with this suffix\n"
        "-Serial       1: process every matching file in the folder of -InMrc\n"
        "-Gpu          GPU id (0)\n"
        "-CtfRes       1: add the spectral-CC resolution (A) as a last column of the\n"
        "              CTF file (0: the reference's columns only)\n\n");
}

// CLoadAngFile::DoIt (CLoadAngFile.cpp:43-71)
std::vector<float> load_ang_file(const std::string& path)
{
    std::vector<float> t;
    if (path.empty()) return t;
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return t;
    char line[256];
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#') continue;
        float v;
        if (std::sscanf(line, "%f", &v) == 1 && std::fabs(v) < 85) t.push_back(v);
        if (t.size() >= 1024) break;
    }
    std::fclose(f);
    return t;
}

struct Package {
    std::string file;   // full path as reported in the CTF file
    int section = 0;
    float tilt = 0.0f;
    int w = 0, h = 0;
    std::vector<float> img;
    gcf_result res{};
    std::vector<float> full;
};

// CInputFolder::FindZeroTilt (CInputFolder.cpp:50-69)
int find_zero_tilt(const std::vector<Package>& p)
{
    int n = (int)p.size();
    if (n > 1 && std::fabs(p[0].tilt - p[1].tilt) < 0.0001f) return n / 2;
    float fmin = 10000.0f;
    int z = -1;
    for (int i = 0; i < n; ++i) {
        float a = std::fabs(p[i].tilt);
        if (a >= fmin) continue;
        fmin = a;
        z = i;
    }
    return z;
}

bool read_stack(const Input& in, const std::vector<float>& angs, std::vector<Package>& pk, bool& tomo,
                int& zero)
{
    int dims[3], mode, nf;
    float pxh;
    if (gcf_mrc_info(in.in_mrc.c_str(), dims, &mode, &pxh, &nf) != GCF_OK) return false;
    int n = dims[2];
    pk.assign(n, Package());
    std::vector<float> ext(n, 0.0f);
    bool has_ext = nf > 1 && gcf_mrc_read_tilts(in.in_mrc.c_str(), ext.data(), n) == GCF_OK;
    for (int i = 0; i < n; ++i) {
        pk[i].file = in.in_mrc;
        pk[i].section = i;
        pk[i].w = dims[0];
        pk[i].h = dims[1];
        pk[i].tilt = has_ext ? ext[i] : 0.0f;
    }
    zero = -1;
    tomo = n > 1;
    if (!tomo) return true;
    if ((int)angs.size() == n) {
        for (int i = 0; i < n; ++i) pk[i].tilt = angs[i];
        zero = find_zero_tilt(pk);
    } else {
        float range = in.tilt_range[1] - in.tilt_range[0];
        if (std::fabs(range) >= 10.0f) {
            float step = range / (n - 1);
            for (int i = 0; i < n; ++i) pk[i].tilt = in.tilt_range[0] + i * step;
            zero = find_zero_tilt(pk);
        }
    }
    return true;
}

// CInputFolder::mGetDirName / mReadFolder / mGetSerial (CInputFolder.cpp:231-335)
bool read_folder(const Input& in, std::vector<Package>& pk, std::string& prefix)
{
    std::string dir;
    size_t slash = in.in_mrc.find_last_of('/');
    if (slash == std::string::npos) {
        prefix = in.in_mrc;
        dir = "./";
    } else {
        dir = in.in_mrc.substr(0, slash + 1);
        prefix = in.in_mrc.substr(slash + 1);
    }
    std::printf("Directory: %s\nPrefix:    %s\nSuffix:    %s\n", dir.c_str(), prefix.c_str(),
                in.in_suffix.c_str());
    DIR* d = opendir(dir.c_str());
    if (!d) {
        std::fprintf(stderr, "Error: cannot open folder\n   %s\n\n", dir.c_str());
        return false;
    }
    size_t ip = prefix.size(), is = in.in_suffix.size();
    while (dirent* e = readdir(d)) {
        const char* name = e->d_name;
        if (name[0] == '.') continue;
        if (ip > 0 && !std::strstr(name, prefix.c_str())) continue;
        if (is > 0) {
            if (std::strlen(name) < ip) continue;
            const char* sfx = strcasestr(name + ip, in.in_suffix.c_str());
            if (!sfx || std::strlen(sfx) != is) continue;
        }
        std::string full = dir + name;
        struct stat sb;
        if (stat(full.c_str(), &sb) < 0) continue;
        Package p;
        p.file = full;
        int dims[3], mode, nf;
        float pxh;
        if (gcf_mrc_info(full.c_str(), dims, &mode, &pxh, &nf) != GCF_OK) continue;
        p.w = dims[0];
        p.h = dims[1];
        pk.push_back(p);
        std::printf("added: %s\n", full.c_str());
    }
    closedir(d);
    std::printf("\n");
    return !pk.empty();
}

std::string serial_of(const std::string& file, const std::string& prefix, const std::string& suffix)
{
    std::string name = file.substr(file.find_last_of('/') == std::string::npos ? 0 : file.find_last_of('/') + 1);
    std::string buf = name.size() > prefix.size() ? name.substr(prefix.size()) : std::string();
    const char* cut = suffix.empty() ? strcasestr(buf.c_str(), ".mrc") : strcasestr(buf.c_str(), suffix.c_str());
    if (cut) buf = buf.substr(0, cut - buf.c_str());
    return buf;
}

// CAsyncSaveImages::mEmbedSerial (MrcUtil/CAsyncSaveImages.cpp:113-143)
std::string embed_serial(const std::string& out, const std::string& serial)
{
    size_t pos = out.find(".mrc");
    if (pos == std::string::npos) return out + serial + ".mrc";
    std::string s = out.substr(0, pos) + serial;
    if (s.substr(pos).find("mrc") == std::string::npos) s += ".mrc";
    return s;
}

void display(const Package& p, int idx, int done, int total)
{
    std::string name = p.file.substr(p.file.find_last_of('/') == std::string::npos ? 0 : p.file.find_last_of('/') + 1);
    std::printf("%s: %5d processed, %5d left\n", name.c_str(), done + 1, total - 1 - done);
    std::printf("   Index  dfmin     dfmax    azimuth  phase   score\n");
    std::printf("   %4d  %8.2f  %8.2f  %6.2f %6.2f %9.5f\n\n", idx + 1, p.res.df_min, p.res.df_max,
                p.res.azimuth, p.res.ext_phase, p.res.score);
}

// CSaveCtfResults::SaveCTF + SaveImod (CSaveCtfResults.cpp:34-117): every
// package in image order; packages not processed yet have zero rows.
void save_results(const Input& in, const std::vector<Package>& pk, bool tomo)
{
    if (in.out_ctf.empty()) return;
    const int n = (int)pk.size();
    std::vector<gcf_result> res(n);
    std::vector<float> tilts(n);
    std::vector<const char*> names(n);
    for (int i = 0; i < n; ++i) {
        res[i] = pk[i].res;
        tilts[i] = pk[i].tilt;
        names[i] = pk[i].file.c_str();
    }
    if (gcf_write_ctf_file_ex(in.out_ctf.c_str(), res.data(), tilts.data(), names.data(), n, tomo ? 1 : 0,
                              in.ctf_res ? GCF_CTF_COLUMN_RES : 0) != GCF_OK)
        std::printf("CTF file: %s\n   cannot be opened, CTF results not saved.\n\n", in.out_ctf.c_str());
}

// The crash-safety flush of CFindSeriesCtfs::DoIt (CFindSeriesCtfs.cpp:97-101):
// the result files are rewritten after every 21st package.
constexpr int kFlushEvery = 21;

struct FlushState {
    const Input* in;
    std::vector<Package>* pk;
    bool tomo;
};

void on_package(void* user, int done, int image, const gcf_result* r)
{
    FlushState* f = static_cast<FlushState*>(user);
    (*f->pk)[image].res = *r;
    if (done % kFlushEvery == 0) save_results(*f->in, *f->pk, f->tomo);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc == 1) {
        std::printf("Use GCtfFind --help to get more information.\n");
        return 0;
    }
    if (std::strstr(argv[1], "--help")) {
        show_help();
        return 0;
    }
    if (std::strstr(argv[1], "--version")) {
        std::printf("GCtfFind (B200) 1.1.2-b200\n");
        return 0;
    }
    double t0 = now_s();
    Input in;
    in.parse(argc, argv);
    in.print();
    // mCheckSame (CCtfFindMain.cpp:50-63)
    if (strcasecmp(in.in_mrc.c_str(), in.out_mrc.c_str()) == 0 ||
        strcasecmp(in.in_mrc.c_str(), in.out_ctf.c_str()) == 0) {
        std::fprintf(stderr, "Error: input and output files have the same name.\n\n");
        return 1;
    }
    gcf_ctx* ctx = nullptr;
    gcf_status st = gcf_create(in.gpu, in.tile, in.log_spect, &ctx);
    if (st != GCF_OK) {
        std::printf("Error: GPU (%d) cannot be used: %s\n\n", in.gpu, gcf_strerror(st));
        return 1;
    }
    std::vector<float> angs = load_ang_file(in.ang_file);
    std::vector<Package> pk;
    bool tomo = false;
    int zero = -1;
    std::string prefix;
    bool ok = in.serial == 0 ? read_stack(in, angs, pk, tomo, zero) : read_folder(in, pk, prefix);
    if (!ok || pk.empty()) {
        std::fprintf(stderr, "Error: no input image could be read from %s\n\n", in.in_mrc.c_str());
        gcf_destroy(ctx);
        return 1;
    }
    int n = (int)pk.size();
    // processing order (MrcUtil/CLoadImages.cpp:71-106)
    std::vector<int> order;
    if (tomo) {
        int z = zero < 0 ? n / 2 : zero;
        order.push_back(z);
        for (int i = 0; i < n; ++i)
            if (i != z) order.push_back(i);
    } else {
        for (int i = 0; i < n; ++i) order.push_back(i);
    }
    // a stack goes to the GPU as stored (gcf_mrc_load widens it there);
    // folders are read on the host, file by file
    const bool gpu_load = in.serial == 0;
    for (int i = 0; i < n && !gpu_load; ++i) {
        pk[i].img.resize((size_t)pk[i].w * pk[i].h);
        if (gcf_mrc_read(pk[i].file.c_str(), pk[i].section, pk[i].img.data()) != GCF_OK) {
            std::fprintf(stderr, "Error: cannot read %s (section %d)\n", pk[i].file.c_str(), pk[i].section);
            gcf_destroy(ctx);
            return 1;
        }
    }
    gcf_optics op{in.kv, in.cs, in.ac, in.px, in.ext_phase[0], std::fmax(in.ext_phase[1], 0.0f)};
    bool want_full = !in.out_mrc.empty();
    int T = in.tile;
    bool same = true;
    for (auto& p : pk) same = same && p.w == pk[0].w && p.h == pk[0].h;
    double tp = now_s();
    if (same) {
        std::vector<const float*> ptr(n);
        if (gpu_load) {
            st = gcf_mrc_load(ctx, in.in_mrc.c_str(), 0, n, ptr.data());
            if (st != GCF_OK) {
                std::fprintf(stderr, "Error: cannot load %s: %s\n", in.in_mrc.c_str(), gcf_last_error(ctx));
                gcf_destroy(ctx);
                return 1;
            }
        } else {
            for (int i = 0; i < n; ++i) ptr[i] = pk[i].img.data();
        }
        std::vector<gcf_result> res(n);
        std::vector<float> full(want_full ? (size_t)n * T * T : 0);
        FlushState fs{&in, &pk, tomo};
        gcf_set_package_callback(ctx, on_package, &fs);
        st = gcf_run_series(ctx, ptr.data(), n, pk[0].w, pk[0].h, gpu_load ? 1 : 0, &op, order.data(),
                            tomo ? 1 : 0, res.data(), want_full ? full.data() : nullptr);
        if (st != GCF_OK) {
            std::fprintf(stderr, "Error: %s: %s\n", gcf_strerror(st), gcf_last_error(ctx));
            gcf_destroy(ctx);
            return 1;
        }
        for (int i = 0; i < n; ++i) {
            pk[i].res = res[i];
            if (want_full) pk[i].full.assign(full.begin() + (size_t)i * T * T, full.begin() + (size_t)(i + 1) * T * T);
        }
        for (int k = 0; k < n; ++k) {
            const Package& p = pk[order[k]];
            if (p.res.df_1d > 0) std::printf("1D estimate: %8.2f  %8.2f  %8.2f\n\n", p.res.df_1d, p.res.phase_1d, p.res.score_1d);
            display(p, order[k], k, n);
        }
    } else {
        // mixed sizes: package by package through the facade
        gcf_destroy(ctx);
        ctx = nullptr;
        try {
            GCTFFind::CFindCtf2D find(in.gpu, in.tile, in.log_spect);
            int ref = -1;
            for (int k = 0; k < n; ++k) {
                Package& p = pk[order[k]];
                int nw, nh;
                float pxn;
                gcf_rescale_dims(p.w, p.h, in.px, &nw, &nh, &pxn);
                std::vector<float> scaled((size_t)nw * nh);
                GCTFFind::gcf_check(gcf_rescale(find.GetContext(), p.img.data(), p.w, p.h, in.px, 0, scaled.data()),
                                    find.GetContext());
                GCTFFind::CCTFTheory th;
                th.Setup(in.kv, in.cs, in.ac, pxn, 100.0f, in.ext_phase[0] * 0.017453f);
                find.Setup1(&th);
                int sz[2] = {nw, nh};
                find.Setup2(sz);
                find.GenHalfSpectrum(scaled.data(), nw, false);
                bool full = (k == 0);
                if (!full) {   // mProcessRefine (CFindSeriesCtfs.cpp:168-203)
                    const gcf_result& rp = pk[ref].res;
                    float dfr = 5000.0f * in.px * in.px;
                    float df[2], ast[2] = {0, 0}, ang[2] = {0, 0}, ph[2] = {0, 0};
                    df[0] = 0.5f * (rp.df_min + rp.df_max);
                    df[1] = std::fmax(df[0] * 0.5f, dfr);
                    float diff = (rp.df_max - rp.df_min) * 0.5f, mean = (rp.df_max + rp.df_min) * 0.5f;
                    ast[0] = mean <= 0.0f ? 0.0f : diff / mean;
                    ang[0] = rp.azimuth;
                    ph[0] = rp.ext_phase;
                    ast[1] = 0.04f;
                    ang[1] = 30.0f;
                    if (in.ext_phase[1] > 0) ph[1] = 40.0f;
                    find.Refine(df, ast, ang, ph);
                    p.res = find.GetResult();
                    if (pk[ref].res.score < p.res.score) ref = order[k];
                    if (p.res.score <= 0) full = true;
                }
                if (full) {   // mProcessFull (CFindSeriesCtfs.cpp:154-166)
                    find.SetPhase(in.ext_phase[0], std::fmax(in.ext_phase[1], 0.0f));
                    find.Do2D();
                    p.res = find.GetResult();
                    std::printf("1D estimate: %8.2f  %8.2f  %8.2f\n\n", p.res.df_1d, p.res.phase_1d, p.res.score_1d);
                    ref = order[k];
                }
                display(p, order[k], k, n);
                if ((k + 1) % kFlushEvery == 0) save_results(in, pk, tomo);
                if (want_full) {
                    float* f = find.GenFullSpectrum();
                    p.full.assign(f, f + (size_t)T * T);
                    delete[] f;
                }
            }
        } catch (const std::exception& e) {
            std::fprintf(stderr, "Error: %s\n", e.what());
            return 1;
        }
    }
    std::printf("Processing time: %.2f (s)\n", now_s() - tp);
    // outputs
    if (want_full) {
        if (tomo) {
            std::vector<float> stack((size_t)n * T * T);
            for (int i = 0; i < n; ++i) std::copy(pk[i].full.begin(), pk[i].full.end(), stack.begin() + (size_t)i * T * T);
            if (gcf_mrc_write(in.out_mrc.c_str(), stack.data(), T, T, n, 1.0f) != GCF_OK)
                std::fprintf(stderr, "Error: cannot write %s\n", in.out_mrc.c_str());
        } else {
            for (int i = 0; i < n; ++i) {
                std::string name = in.serial == 0 ? in.out_mrc
                                                  : embed_serial(in.out_mrc, serial_of(pk[i].file, prefix, in.in_suffix));
                if (gcf_mrc_write(name.c_str(), pk[i].full.data(), T, T, 1, 1.0f) != GCF_OK)
                    std::fprintf(stderr, "Error: cannot write %s\n", name.c_str());
            }
        }
    }
    save_results(in, pk, tomo);
    if (ctx) gcf_destroy(ctx);
    std::printf("Total time:  %.3f (s)\n\n", now_s() - t0);
    return 0;
}
