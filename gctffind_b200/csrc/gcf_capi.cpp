// gcf_capi.cpp -- host side of the B200 CTF-estimation library: context,
// host-built tables, device buffers, the C ABI of include/gctf_b200.h and
// the batched series driver.
//
// Compiled with -ffp-contract=off: the float expressions that the
// reference evaluates on the host (search windows, steps, tables) are
// rounded operation by operation here too.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "gcf_internal.h"

using namespace gcf;

namespace gcf {
// Optional: fused spectrum path (gcf_fused.cu).
int fused_tile_supported(int tile);

namespace {
std::atomic<unsigned long long> g_alloc_epoch{0};
thread_local bool t_capturing = false;   // this thread is capturing a batch call
}  // namespace

void note_device_alloc() { g_alloc_epoch.fetch_add(1, std::memory_order_relaxed); }
unsigned long long device_alloc_epoch() { return g_alloc_epoch.load(std::memory_order_relaxed); }
cudaError_t record_timing(cudaEvent_t ev, cudaStream_t st)
{
    return t_capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
}
}  // namespace gcf

namespace {

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t cnt)
    {
        if (cnt <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        gcf::note_device_alloc();
        cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(cnt, 1) * sizeof(T));
        if (e == cudaSuccess) n = cnt;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct BandHost {
    int tile;
    float px, kv, cs, ac;
    int n;
    DBuf<int> idx;
    DBuf<float> a, d, env, c2t, s2t;
    BandDev dev;
};

struct FftPlan {
    cufftHandle h = 0;
    unsigned long long used = 0;   // last use (the context's plan clock)
};

// Mapped page-locked host staging of the small host -> device uploads of
// one call (job tables, work items, descriptors): the copy kernels read
// from here, so the host vectors they came from may go away, and a CUDA
// graph captured from the call keeps valid sources for its copy nodes (a
// graph owns the arena it was captured with).  Blocks never move; reset()
// reuses them once the copies of the previous call are complete.
struct HostArena {
    struct Block {
        char* p;
        size_t cap, used;
        char* dev;   // the block's address on the device (mapped memory)
    };
    std::vector<Block> blocks;
    size_t cur = 0;
    void reset()
    {
        for (Block& b : blocks) b.used = 0;
        cur = 0;
    }
    bool frozen = false;   // no new blocks (inside a stream capture)
    size_t used_bytes() const
    {
        size_t u = 0;
        for (const Block& b : blocks) u += b.used;
        return u;
    }
    // One free block of at least `bytes` (blocks allocated now, not during a
    // capture, where a page-locked allocation would end the capture).
    bool reserve(size_t bytes)
    {
        for (const Block& b : blocks)
            if (b.cap >= bytes) return true;
        release();
        Block b{nullptr, std::max<size_t>(bytes, (size_t)1 << 20), 0, nullptr};
        if (!alloc(b)) return false;
        blocks.push_back(b);
        return true;
    }
    static bool alloc(Block& b)
    {
        if (cudaHostAlloc((void**)&b.p, b.cap, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
            return false;
        if (cudaHostGetDevicePointer((void**)&b.dev, b.p, 0) != cudaSuccess) {
            cudaFreeHost(b.p);
            b.p = nullptr;
            return false;
        }
        return true;
    }
    // Copies src into the arena; returns the copy's device-side address.
    void* put(const void* src, size_t bytes)
    {
        const size_t need = (bytes + 255) & ~(size_t)255;
        while (cur < blocks.size() && blocks[cur].cap - blocks[cur].used < need) ++cur;
        if (cur == blocks.size()) {
            if (frozen) return nullptr;
            Block b{nullptr, std::max<size_t>(need, (size_t)1 << 20), 0, nullptr};
            if (!alloc(b)) return nullptr;
            blocks.push_back(b);
        }
        Block& b = blocks[cur];
        std::memcpy(b.p + b.used, src, bytes);
        void* dev = b.dev + b.used;
        b.used += need;
        return dev;
    }
    void release()
    {
        for (Block& b : blocks) cudaFreeHost(b.p);
        blocks.clear();
        cur = 0;
    }
};

// One captured batch call (gcf_run_batch / gcf_run_batch_mode with CUDA
// graphs on): the graph of its device work, keyed by everything the work
// depends on, and what the host needs to read its results back.
struct BatchGraph {
    unsigned long long key = 0;        // key of the call that `exec` replays
    unsigned long long want = 0;       // key of the latest eager call
    int seen = 0;                      // eager calls in a row with key `want`
    cudaGraphExec_t exec = nullptr;
    unsigned long long epoch = 0;      // device-allocation epoch at capture
    unsigned long long model_version = 0;   // contraction model rows it read
    HostArena arena;                   // sources of the graph's upload nodes
    int kev_used = 0;
    long long launches = 0;            // kernels this library launched in it
    int nodes = 0;                     // graph nodes
    std::vector<float> pxn;            // search pixel size of each slot
    std::vector<int> band;             // band slot of each job
    int nj = 0;
};

}  // namespace

struct gcf_ctx {
    int dev = 0;
    int tile = 512;
    int log_spect = 0;
    int impl = GCF_SPECT_CUFFT;
    cudaStream_t st = nullptr;
    cudaStream_t st_copy = nullptr;   // host -> device uploads
    // Compute work goes to `st`.  A series in device memory runs its tile
    // spectra on the high-priority stream while post-processing and searches
    // of finished chunks run on `st_search` (low priority) in the SMs the
    // cluster kernel leaves free; `st` is swapped with it for those calls.
    cudaStream_t st_search = nullptr;
    // Second high-priority stream: consecutive tile-spectrum chunks of a
    // device series alternate between `st` and `st_tile`, so a chunk's
    // clusters start while the previous chunk's last items finish.
    cudaStream_t st_tile = nullptr;
    std::vector<cudaEvent_t> chunk_ev;
    std::string err;
    long long launches = 0;
    float stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    // candidates evaluated: 2D candidates, 2D (candidate, band pixel) pairs,
    // 1D grid points, 1D (grid point, bin) pairs; reset like stage_ms
    long long search_counts[4] = {0, 0, 0, 0};
    DBuf<int> d_counts;
    cudaEvent_t ev[8] = {};
    std::vector<cudaEvent_t> kev;   // begin/end pairs around fused tile-kernel launches
    int kev_used = 0;

    // per-tile tables
    DBuf<float> taper;
    DBuf<int> rad_off, rad_pix;
    DBuf<int> ring_off, ring_pix;
    DBuf<double2> ring_geo;   // (s^2, polar angle) of each ring pixel

    // bands
    std::vector<BandHost*> bands;
    DBuf<BandDev> d_bands;
    bool bands_dirty = true;

    // buffers
    DBuf<float> images, rescaled, tiles;
    DBuf<float2> cmp, rs_cmp, rs_crop;
    DBuf<float> rs_src;   // an aligned copy of a device image cuFFT cannot read in place
    DBuf<__nv_bfloat16> rsg_bf;   // scratch of the tensor-core rescale (gcf_rsgemm.cu)
    DBuf<float> rsg_f;
    DBuf<int> rsg_err;            // its products' bounded-wait flag, checked when results are read
    DBuf<double> acc, hsum, moments, moments2;
    DBuf<float> lpfull;
    DBuf<float2> lpcmp;
    DBuf<float> raw, ctf0, ctf, radial, band_spec, cc_res, full;
    DBuf<int> lowpassed, spec_off, mic_of;
    DBuf<SearchJob> jobs;
    DBuf<double> sum_ss, ring_sums;
    DBuf<float4> cand;
    DBuf<float2> cval;
    DBuf<double2> part;
    DBuf<int> arrive;
    DBuf<gcf_result> d_res;
    DBuf<PixOptics> d_optics;

    std::map<std::tuple<int, int, int>, FftPlan> plans;   // (kind, a, b)
    unsigned long long plan_clock = 0;
    DBuf<char> fft_work;   // work area shared by the rescale plans (one stream)

    // fused spectrum
    DBuf<float2> tw512;
    DBuf<FusedImageDesc> f_desc;
    DBuf<int4> f_items;
    DBuf<int> f_first;
    DBuf<float> f_inv, f_partial;
    DBuf<unsigned long long> f_next;   // item queues of the tile kernel launches
    // cluster-less tile CTAs beside each cluster launch (SMs the clusters
    // leave free) and their global scratch
    DBuf<double> lp_g;   // lowpass filter per half-spectrum bin, for tile lp_g_tile
    int lp_g_tile = 0;
    int solo_n = -1;
    int n_sms = 0;   // multiprocessors of the device (0 until first asked)
    cudaStream_t st_solo = nullptr;
    cudaEvent_t solo_fork = nullptr, solo_join = nullptr;
    DBuf<float2> solo_col;
    DBuf<float> solo_acc;
    DBuf<double> f_bsum;
    DBuf<double*> f_bsum_ptr;
    std::vector<int> f_first_h;    // host copy of f_first for the current plan
    std::vector<int> f_blocks_h;   // block-sum blocks of each planned micrograph
    int fused_clusters = 0;
    int fused_shape = 0;
    int fused_shape_req = 0;   // 0: pick by SM coverage
    int rescale_impl = GCF_RESCALE_CUFFT;

    // CFindCtf2D call-shape state
    gcf_optics optics{};
    bool have_setup = false;
    bool have_spectrum = false;
    int img_w = 0, img_h = 0;
    float phase_deg = 0.0f, phase_range = 0.0f;
    float held_phase = 0.0f;   // CFindDefocus2D::m_fExtPhase between Do2D / Refine calls
    int cur_lowpassed = 0;

    // GBackground1D
    DBuf<float> bg_spec, bg_curve;
    DBuf<int> bg_start;

    // BF16 candidate contraction (search mode GCF_SEARCH_BF16 / _LEARNED)
    PolarGrid model_grid{};          // grid the model rows were made for
    bool have_model = false;
    DBuf<__nv_bfloat16> cA, cA2, cB, cE;
    DBuf<float> cP, cDz;
    DBuf<double> cSS;
    DBuf<int2> cRows, cTiles;
    DBuf<int> cNtiles, cErr;
    DBuf<float4> cPrior;
    int gemm_bn = 256, gemm_stages = 4;     // tile of the P product (tuned)
    int gemm_persistent = 0;                // P product by the persistent kernel (tuned)
    float contract_dz = 10.0f;              // defocus row step, Angstrom
    int contract_ns = 512, contract_nth = 64;
    // [0] candidates scored on the table, [1] tensor-core multiply-adds,
    // [2] candidates re-scored in FP32, [3] learned searches that fell back
    long long fast_counts[4] = {0, 0, 0, 0};
    // events around the contraction stages: bin | product | table | FP32 finish
    cudaEvent_t fev[7] = {};          // contraction stages [0..4], network [5..6]
    float fast_ms[5] = {0, 0, 0, 0, 0};

    // learned initialiser
    NnNet* nn = nullptr;
    bool nn_ready = false;            // weights set (loaded, trained or given)
    float learned_tau = 0.1f;         // refined CC below which the full search runs
    gcf_package_fn pkg_fn = nullptr;  // per-package completion hook of gcf_run_series
    void* pkg_user = nullptr;
    DBuf<__nv_bfloat16> nx1, nx2;     // network inputs of a chunk of jobs
    DBuf<float> npx, nparams, ntarget, nloss;
    // MRC sections loaded to the device (gcf_mrc_load): float images, the
    // raw section bytes of two in flight, their pinned host staging
    DBuf<float> loaded;
    DBuf<unsigned char> ingest_raw;
    unsigned char* ingest_pin = nullptr;
    size_t ingest_pin_bytes = 0;
    cudaEvent_t ingest_copied[2] = {}, ingest_used[2] = {};
    unsigned long long nn_version = 0;   // bumped whenever the weights change
    unsigned long long model_version = 0;   // bumped whenever the model rows are remade

    // host staging of this call's uploads; CUDA graphs of batch calls
    HostArena arena;
    bool graphs = false;              // gcf_set_graphs
    bool capturing = false;           // inside a stream capture of ctx->st
    BatchGraph bgraph;
    cudaEvent_t fork_ev = nullptr;    // dependency-only fork of st_copy from st
    long long graph_launches = 0;     // graph launches of the last batch call
    int graph_fail = 0;               // why the last capture gave no graph (0: it did)
};

namespace {

// Host -> device upload of `bytes` from a transient host buffer, staged
// through the context's pinned arena and copied by a kernel on `st` (not a
// copy-engine transfer: those queue behind the bulk image uploads of the
// copy stream, which would hold the compute stream until every image had
// landed).  Outside a capture, an arena that has grown past 64 MB is
// recycled once the context's streams are idle.
cudaError_t h2d(gcf_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) return cudaSuccess;
    if (!ctx->capturing) {
        size_t used = 0;
        for (const HostArena::Block& b : ctx->arena.blocks) used += b.used;
        if (used > ((size_t)64 << 20)) {
            for (cudaStream_t s : {ctx->st, ctx->st_copy, ctx->st_search, ctx->st_tile, ctx->st_solo})
                if (s) {
                    cudaError_t e = cudaStreamSynchronize(s);
                    if (e != cudaSuccess) return e;
                }
            ctx->arena.reset();
        }
    }
    void* h = ctx->arena.put(src, bytes);
    if (!h) return cudaErrorMemoryAllocation;
    ctx->launches += 1;
    return launch_copy_from_host(dst, h, bytes, st);
}

gcf_status fail(gcf_ctx* c, gcf_status s, const char* what)
{
    if (c) c->err = what ? what : "";
    return s;
}

gcf_status cuda_fail(gcf_ctx* c, cudaError_t e, const char* where)
{
    if (c) c->err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? GCF_ERR_NO_MEMORY : GCF_ERR_CUDA;
}

#define CK(call)                                                     \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);     \
    } while (0)

#define CKS(call)                                                    \
    do {                                                             \
        gcf_status s_ = (call);                                      \
        if (s_ != GCF_OK) return s_;                                 \
    } while (0)

#define CKL()                                                        \
    do {                                                             \
        cudaError_t e_ = cudaGetLastError();                         \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, "kernel launch"); \
    } while (0)

// CCTFTheory::Setup + GCalcCTF2D::SetParam in pixel units.
PixOptics make_optics(const gcf_optics& op, float px_n)
{
    PixOptics o;
    double wl = 12.26 / std::sqrt((double)op.kv * 1000.0 + 0.9784 * (double)op.kv * op.kv);
    o.wl = (float)wl / px_n;
    o.cs = (float)((double)op.cs_mm * 1e7 / px_n);
    float ac = op.amp_contrast;
    o.amp_phase = (float)atanf(ac / sqrtf(1.0f - ac * ac));
    o.px = px_n;
    return o;
}

void res_range_of(float px, float r[2])
{
    r[0] = 25.0f * px;
    r[1] = (2.0f * px) / 0.8f;
    if (r[1] < 3.5f) r[1] = 3.5f;
}

struct Layout {
    int ntx, nty, offx, offy, ov, stride;
};

Layout tile_layout(int w, int h, int tile)
{
    Layout L;
    int ov = (int)(tile * 0.50f);
    ov = ov / 2 * 2;
    L.ov = ov;
    L.stride = tile - ov;
    L.ntx = (w - ov) / L.stride;
    L.nty = (h - ov) / L.stride;
    L.offx = (w - L.ntx * tile + (L.ntx - 1) * ov) / 2;
    L.offy = (h - L.nty * tile + (L.nty - 1) * ov) / 2;
    return L;
}

gcf_status build_tile_tables(gcf_ctx* ctx)
{
    int T = ctx->tile, cx = T / 2 + 1, cy = T;
    // GRoundEdge taper (FindCTF/GRoundEdge.cu:7-25)
    std::vector<float> tp((size_t)T * T);
    double c = T * 0.5, s = T;
    for (int y = 0; y < T; ++y)
        for (int x = 0; x < T; ++x) {
            double fx = 2.0 * std::fabs(x - c) / s, fy = 2.0 * std::fabs(y - c) / s;
            double r = std::sqrt(fx * fx + fy * fy), v = 0.0;
            if (r < 1.0) {
                double q = 0.5 * (1.0 - std::cos(M_PI * r));
                v = 1.0 - q * q * q;
            }
            tp[(size_t)y * T + x] = (float)v;
        }
    CK(ctx->taper.ensure(tp.size()));
    CK(cudaMemcpy(ctx->taper.p, tp.data(), tp.size() * sizeof(float), cudaMemcpyHostToDevice));
    // GRadialAvg nearest-pixel samples (FindCTF/GRadialAvg.cu:11-33)
    std::vector<int> off(cx + 1), pix;
    for (int r = 0; r < cx; ++r) {
        off[r] = (int)pix.size();
        int np = (int)(3.1415926f * r + 0.5f);
        if (np < 1) np = 1;
        else if (np > 180) np = 180;
        float step = 180.0f / np;
        for (int i = 0; i < np; ++i) {
            float rad = (-90.0f + i * step) * 0.017453f;
            int x = (int)(r * cosf(rad) + 0.5f);
            int y = (int)(r * sinf(rad) + cy / 2 + 0.5f);
            if (y > cy - 1) y = cy - 1;   // the reference reads one row past for r = cx-1
            if (x > cx - 1) x = cx - 1;
            pix.push_back(y * cx + x);
        }
    }
    off[cx] = (int)pix.size();
    CK(ctx->rad_off.ensure(off.size()));
    CK(ctx->rad_pix.ensure(pix.size()));
    CK(cudaMemcpy(ctx->rad_off.p, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->rad_pix.p, pix.data(), pix.size() * sizeof(int), cudaMemcpyHostToDevice));
    // Integer-radius rings of the half spectrum for the spectral-CC
    // resolution (GSpectralCC2D, FindCTF/GSpectralCC2D.cu:27-64): a shell
    // [lo, hi) with integer bounds is exactly the rings lo .. hi-1 of
    // floor(sqrt(x^2 + |y - cy/2|^2)), evaluated in float as the reference does.
    {
        std::vector<std::vector<int>> rings(cx);
        for (int y = 0; y < cy; ++y) {
            float fy = fabsf(y - cy * 0.5f);
            for (int x = 0; x < cx; ++x) {
                float r = sqrtf((float)(x * x) + fy * fy);
                int ri = (int)r;
                if (ri < cx) rings[ri].push_back(y * cx + x);
            }
        }
        std::vector<int> roff(cx + 1), rpix;
        for (int ri = 0; ri < cx; ++ri) {
            roff[ri] = (int)rpix.size();
            rpix.insert(rpix.end(), rings[ri].begin(), rings[ri].end());
        }
        roff[cx] = (int)rpix.size();
        CK(ctx->ring_off.ensure(roff.size()));
        CK(ctx->ring_pix.ensure(rpix.size()));
        CK(cudaMemcpy(ctx->ring_off.p, roff.data(), roff.size() * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->ring_pix.p, rpix.data(), rpix.size() * sizeof(int), cudaMemcpyHostToDevice));
        // s^2 and the polar angle atan(fy / (fx + 1e-30)) of GCalcCTF2D
        // (FindCTF/GCalcCTF2D.cu:20-27) per ring pixel, in double: they
        // depend on the tile size only
        std::vector<double2> geo(rpix.size());
        for (size_t k = 0; k < rpix.size(); ++k) {
            const int y = rpix[k] / cx, x = rpix[k] - y * cx;
            const double fx = x * 0.5 / (cx - 1);
            const double fy = (double)(y - cy / 2) / cy;
            geo[k] = make_double2(fx * fx + fy * fy, std::atan(fy / (fx + 1e-30)));
        }
        CK(ctx->ring_geo.ensure(geo.size()));
        CK(cudaMemcpy(ctx->ring_geo.p, geo.data(), geo.size() * sizeof(double2), cudaMemcpyHostToDevice));
    }
    // exp(-2 pi i t / T), t < T: twiddles of the fused tile FFT
    std::vector<float2> tw(T);
    for (int t = 0; t < T; ++t) {
        double a = -2.0 * M_PI * (double)t / (double)T;
        tw[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    CK(ctx->tw512.ensure(T));
    CK(cudaMemcpy(ctx->tw512.p, tw.data(), T * sizeof(float2), cudaMemcpyHostToDevice));
    // A copy from pageable memory may return before its DMA lands, and the
    // context's streams are non-blocking (not ordered after these copies):
    // wait for the tables once, at creation.
    CK(cudaDeviceSynchronize());
    return GCF_OK;
}

// In-band pixels of the 2D correlation (CFindDefocus2D::Setup2,
// FindCTF/CFindDefocus2D.cpp:86-92; GCC2D band, FindCTF/GCC2D.cu:148-160).
gcf_status get_band(gcf_ctx* ctx, const gcf_optics& op, float px_n, int* slot)
{
    int T = ctx->tile;
    for (size_t i = 0; i < ctx->bands.size(); ++i) {
        BandHost* b = ctx->bands[i];
        if (b->tile == T && b->px == px_n && b->kv == op.kv && b->cs == op.cs_mm &&
            b->ac == op.amp_contrast) {
            *slot = (int)i;
            return GCF_OK;
        }
    }
    int cx = T / 2 + 1, cy = T;
    PixOptics o = make_optics(op, px_n);
    float rr[2];
    res_range_of(px_n, rr);
    float res1 = cy * px_n;
    float lo = res1 / rr[0], hi = res1 / rr[1];
    float l = lo / cy, hh = hi / cy;
    if (hh > 0.75f) hh = 0.75f;
    float lo2 = l * l, hi2 = hh * hh;
    std::vector<int> idx;
    std::vector<float> va, vd, ve, vc, vs;
    for (int y = 0; y < cy; ++y) {
        float fyf = (y - cy * 0.5f) / cy;
        double fy = (double)(y - cy / 2) / cy;
        for (int x = 0; x < cx; ++x) {
            float fxf = (0.5f * x) / (cx - 1);
            float s2f = fxf * fxf + fyf * fyf;
            if (s2f < lo2 || s2f > hi2) continue;
            double fx = x * 0.5 / (cx - 1);
            double s2 = fx * fx + fy * fy;
            double th = std::atan(fy / (fx + 1e-30));
            idx.push_back(y * cx + x);
            va.push_back((float)((double)o.wl * s2));
            vd.push_back((float)(-0.5 * (double)o.wl * o.wl * o.wl * s2 * s2 * o.cs));
            ve.push_back((float)std::exp(-16.0 * s2));
            vc.push_back((float)std::cos(2.0 * th));
            vs.push_back((float)std::sin(2.0 * th));
        }
    }
    BandHost* b = new BandHost();
    b->tile = T;
    b->px = px_n;
    b->kv = op.kv;
    b->cs = op.cs_mm;
    b->ac = op.amp_contrast;
    b->n = (int)idx.size();
    size_t n = idx.size();
    cudaError_t e = cudaSuccess;
    if ((e = b->idx.ensure(n)) != cudaSuccess || (e = b->a.ensure(n)) != cudaSuccess ||
        (e = b->d.ensure(n)) != cudaSuccess || (e = b->env.ensure(n)) != cudaSuccess ||
        (e = b->c2t.ensure(n)) != cudaSuccess || (e = b->s2t.ensure(n)) != cudaSuccess) {
        delete b;
        return cuda_fail(ctx, e, "band alloc");
    }
    // On the compute stream, so the kernels that read the band are ordered
    // after the copies (a pageable source is staged before the call returns).
    CK(h2d(ctx, b->idx.p, idx.data(), n * sizeof(int), ctx->st));
    CK(h2d(ctx, b->a.p, va.data(), n * sizeof(float), ctx->st));
    CK(h2d(ctx, b->d.p, vd.data(), n * sizeof(float), ctx->st));
    CK(h2d(ctx, b->env.p, ve.data(), n * sizeof(float), ctx->st));
    CK(h2d(ctx, b->c2t.p, vc.data(), n * sizeof(float), ctx->st));
    CK(h2d(ctx, b->s2t.p, vs.data(), n * sizeof(float), ctx->st));
    b->dev.n = b->n;
    b->dev.cx = cx;
    b->dev.cy = cy;
    b->dev.pad = 0;
    b->dev.idx = b->idx.p;
    b->dev.a = b->a.p;
    b->dev.d = b->d.p;
    b->dev.env = b->env.p;
    b->dev.c2t = b->c2t.p;
    b->dev.s2t = b->s2t.p;
    ctx->bands.push_back(b);
    ctx->bands_dirty = true;
    *slot = (int)ctx->bands.size() - 1;
    return GCF_OK;
}

gcf_status upload_bands(gcf_ctx* ctx)
{
    if (!ctx->bands_dirty) return GCF_OK;
    std::vector<BandDev> v;
    for (auto* b : ctx->bands) v.push_back(b->dev);
    CK(ctx->d_bands.ensure(v.size()));
    CK(h2d(ctx, ctx->d_bands.p, v.data(), v.size() * sizeof(BandDev), ctx->st));
    ctx->bands_dirty = false;
    return GCF_OK;
}

// Rescale plans (kinds 1, 2) kept at most: a batch of micrographs at
// continuously varying pixel sizes needs a new C2R size per micrograph, so
// the least recently used plans are destroyed beyond this count (more than
// one 256-micrograph batch needs, so a repeated batch finds all its plans).
constexpr size_t kMaxRescalePlans = 640;

gcf_status get_plan(gcf_ctx* ctx, int kind, int a, int b, cufftHandle* out)
{
    auto key = std::make_tuple(kind, a, b);
    auto it = ctx->plans.find(key);
    if (it != ctx->plans.end()) {
        it->second.used = ++ctx->plan_clock;
        *out = it->second.h;
        return GCF_OK;
    }
    cufftHandle h;
    cufftResult r;
    if (kind == 1 || kind == 2) {
        // rescale plans run one after another on ctx->st: they share one
        // work area instead of each holding its own
        size_t n_rescale = 0;
        for (auto& kv : ctx->plans) n_rescale += (std::get<0>(kv.first) == 1 || std::get<0>(kv.first) == 2);
        while (n_rescale >= kMaxRescalePlans) {
            auto lru = ctx->plans.end();
            for (auto q = ctx->plans.begin(); q != ctx->plans.end(); ++q)
                if ((std::get<0>(q->first) == 1 || std::get<0>(q->first) == 2) &&
                    (lru == ctx->plans.end() || q->second.used < lru->second.used))
                    lru = q;
            CK(cudaStreamSynchronize(ctx->st));
            cufftDestroy(lru->second.h);
            ctx->plans.erase(lru);
            note_device_alloc();   // a captured graph may hold the destroyed plan
            --n_rescale;
        }
        size_t ws = 0;
        r = cufftCreate(&h);
        if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(h, 0);
        if (r == CUFFT_SUCCESS) r = cufftMakePlan2d(h, a, b, kind == 1 ? CUFFT_R2C : CUFFT_C2R, &ws);
        if (r == CUFFT_SUCCESS && ws > ctx->fft_work.n) {
            CK(cudaStreamSynchronize(ctx->st));
            CK(ctx->fft_work.ensure(ws));
            for (auto& kv : ctx->plans)
                if (std::get<0>(kv.first) == 1 || std::get<0>(kv.first) == 2)
                    cufftSetWorkArea(kv.second.h, ctx->fft_work.p);
        }
        if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(h, ctx->fft_work.p);
        if (r != CUFFT_SUCCESS) {
            cufftDestroy(h);
            ctx->err = "cufft plan creation failed (" + std::to_string((int)r) + ")";
            return r == CUFFT_ALLOC_FAILED ? GCF_ERR_NO_MEMORY : GCF_ERR_CUFFT;
        }
    }
    if (kind == 0) {   // batched tile R2C: a = tile, b = batch
        int n[2] = {a, a};
        r = cufftPlanMany(&h, 2, n, nullptr, 1, a * a, nullptr, 1, (a / 2 + 1) * a, CUFFT_R2C, b);
    } else if (kind == 3 || kind == 4) {   // batched full-spectrum R2C / C2R: a = tile, b = batch
        int n[2] = {a, a};
        if (kind == 3)
            r = cufftPlanMany(&h, 2, n, nullptr, 1, a * a, nullptr, 1, (a / 2 + 1) * a, CUFFT_R2C, b);
        else
            r = cufftPlanMany(&h, 2, n, nullptr, 1, (a / 2 + 1) * a, nullptr, 1, a * a, CUFFT_C2R, b);
    }   // kinds 1 and 2 (image R2C / C2R: a = height, b = width) above
    if (r != CUFFT_SUCCESS) {
        ctx->err = "cufft plan creation failed (" + std::to_string((int)r) + ")";
        return r == CUFFT_ALLOC_FAILED ? GCF_ERR_NO_MEMORY : GCF_ERR_CUFFT;
    }
    if (cufftSetStream(h, ctx->st) != CUFFT_SUCCESS) {
        cufftDestroy(h);
        return fail(ctx, GCF_ERR_CUFFT, "cufftSetStream failed");
    }
    ctx->plans[key].h = h;
    ctx->plans[key].used = ++ctx->plan_clock;
    *out = h;
    return GCF_OK;
}

// Image description for the spectrum stage.
struct MicImage {
    const float* img;   // device
    int w, h, pitch;
    float px_n;
};

// CGenAvgSpectrum::DoIt for one micrograph, batched-cuFFT variant.
gcf_status spectrum_cufft(gcf_ctx* ctx, const MicImage& m, float* raw_out)
{
    int T = ctx->tile, cx = T / 2 + 1;
    Layout L = tile_layout(m.w, m.h, T);
    int nt = L.ntx * L.nty;
    if (L.ntx <= 0 || L.nty <= 0) return fail(ctx, GCF_ERR_IMAGE_TOO_SMALL, "image holds no tile");
    const int kBatch = 256;
    int batch = std::min(nt, kBatch);
    CK(ctx->tiles.ensure((size_t)batch * T * T));
    CK(ctx->cmp.ensure((size_t)batch * cx * T));
    CK(ctx->acc.ensure((size_t)cx * T));
    CK(cudaMemsetAsync(ctx->acc.p, 0, (size_t)cx * T * sizeof(double), ctx->st));
    for (int t0 = 0; t0 < nt; t0 += batch) {
        int nb = std::min(batch, nt - t0);
        launch_extract_tiles(m.img, m.w, m.h, m.pitch, T, L.ntx, L.offx, L.offy, L.stride, t0, nb,
                             ctx->taper.p, ctx->tiles.p, ctx->st);
        CKL();
        ctx->launches += 1;
        cufftHandle plan;
        CKS(get_plan(ctx, 0, T, nb, &plan));
        if (cufftExecR2C(plan, ctx->tiles.p, (cufftComplex*)ctx->cmp.p) != CUFFT_SUCCESS)
            return fail(ctx, GCF_ERR_CUFFT, "cufftExecR2C (tiles) failed");
        launch_amp_accumulate(ctx->cmp.p, T, nb, ctx->acc.p, ctx->st);
        CKL();
        ctx->launches += 1;
    }
    launch_finalize_raw(ctx->acc.p, cx * T, 1.0 / nt, raw_out, ctx->st);
    CKL();
    ctx->launches += 1;
    return GCF_OK;
}

// Work plan of the fused tile-spectrum kernel (tile 512) for mics: image
// descriptors, block-sum slots and work items, uploaded on ctx->st.  Each
// micrograph's tiles form runs of at most 24 (an item's |F| sums live in
// registers until it ends); the split depends on the micrograph alone, so
// its spectrum does not depend on the batch or chunk it is in.
// The tile kernel's cluster shape and resident cluster count (chosen once,
// again after gcf_set_fused_shape / gcf_autotune).
gcf_status ensure_fused_shape(gcf_ctx* ctx)
{
    if (ctx->fused_clusters > 0) return GCF_OK;
    int n = 0, shape = ctx->fused_shape_req;
    if (shape) CK(fused_clusters_of(shape, &n));
    else CK(fused_max_clusters(&n, &shape));
    if (n <= 0) return fail(ctx, GCF_ERR_CUDA, "fused spectrum kernel cannot be resident");
    ctx->fused_clusters = n;
    ctx->fused_shape = shape;
    return GCF_OK;
}

gcf_status fused_plan(gcf_ctx* ctx, const std::vector<MicImage>& mics)
{
    const int T = ctx->tile, cx = T / 2 + 1, nm = (int)mics.size();
    CKS(ensure_fused_shape(ctx));
    // 24 rather than 32: the cluster-less CTAs then finish their last items
    // sooner and may keep taking items longer (a 41-tilt series step 12.43
    // -> 12.21 ms; the spectra change only in the grouping of the sums)
    const int kItemTiles = 24;
    std::vector<FusedImageDesc> d(nm);
    std::vector<int4> items;
    std::vector<int>& first = ctx->f_first_h;
    first.assign(nm + 1, 0);
    ctx->f_blocks_h.assign(nm, 0);
    std::vector<float> inv(nm);
    std::vector<size_t> boff(nm);
    size_t nblk = 0;
    for (int i = 0; i < nm; ++i) {
        const MicImage& m = mics[i];
        Layout L = tile_layout(m.w, m.h, T);
        int nt = L.ntx * L.nty;
        if (L.ntx <= 0 || L.nty <= 0) return fail(ctx, GCF_ERR_IMAGE_TOO_SMALL, "image holds no tile");
        d[i].img = m.img;
        d[i].bsum = nullptr;   // set below
        d[i].pitch = m.pitch;
        d[i].ntx = L.ntx;
        d[i].nty = L.nty;
        d[i].offx = L.offx;
        d[i].offy = L.offy;
        d[i].stride = L.stride;
        d[i].vec = ((L.offx % 2) == 0 && (L.stride % 2) == 0 && (m.pitch % 2) == 0 &&
                    ((uintptr_t)m.img % 8) == 0) ? 2 : 1;
        d[i].nbx = L.ntx + 1;
        boff[i] = nblk;
        ctx->f_blocks_h[i] = (L.ntx + 1) * (L.nty + 1);
        nblk += (size_t)ctx->f_blocks_h[i];
        inv[i] = 1.0f / nt;
        first[i] = (int)items.size();
        int nch = (nt + kItemTiles - 1) / kItemTiles;
        int chunk = (nt + nch - 1) / nch;
        for (int t0 = 0; t0 < nt; t0 += chunk)
            items.push_back(make_int4(i, t0, std::min(nt, t0 + chunk), (int)items.size()));
    }
    first[nm] = (int)items.size();
    int ni = (int)items.size();
    CK(ctx->f_bsum.ensure(nblk));
    CK(ctx->f_bsum_ptr.ensure(nm));
    std::vector<double*> bptr(nm);
    for (int i = 0; i < nm; ++i) {
        bptr[i] = ctx->f_bsum.p + boff[i];
        d[i].bsum = bptr[i];
    }
    CK(h2d(ctx, ctx->f_bsum_ptr.p, bptr.data(), nm * sizeof(double*), ctx->st));
    CK(ctx->f_desc.ensure(nm));
    CK(ctx->f_items.ensure(ni));
    CK(ctx->f_first.ensure(nm + 1));
    CK(ctx->f_inv.ensure(nm));
    CK(ctx->f_partial.ensure((size_t)ni * cx * T));
    CK(ctx->f_next.ensure(nm));
    CK(h2d(ctx, ctx->f_desc.p, d.data(), nm * sizeof(FusedImageDesc), ctx->st));
    CK(h2d(ctx, ctx->f_items.p, items.data(), ni * sizeof(int4), ctx->st));
    CK(h2d(ctx, ctx->f_first.p, first.data(), (nm + 1) * sizeof(int), ctx->st));
    CK(h2d(ctx, ctx->f_inv.p, inv.data(), nm * sizeof(float), ctx->st));
    return GCF_OK;
}

// Spectra of planned micrographs m0 .. m1-1 into raw_out (the spectrum of
// m0) on stream st.  Launches of disjoint ranges share the plan's buffers
// (each range owns its items, partial spectra and item counter), so they
// may run concurrently once the plan's uploads are done.
// The cluster-less CTAs beside a cluster launch: one per SM that the
// clusters leave free, with their scratch (set up on first use; 1.5 MB of
// global memory per CTA, L2-resident while it works).  Their launches all
// go to st_solo, so launches of two chunks never share the scratch at once.
gcf_status solo_setup(gcf_ctx* ctx, SoloLaunch* sl)
{
    if (ctx->solo_n < 0) {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->dev));
        const int per_cluster = (ctx->fused_shape == 16 || ctx->fused_shape == 168) ? 16 : 8;
        ctx->solo_n = std::max(0, sms - ctx->fused_clusters * per_cluster);
        if (ctx->solo_n > 0 && !ctx->st_solo) {
            int lo = 0, hi = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            CK(cudaStreamCreateWithPriority(&ctx->st_solo, cudaStreamNonBlocking, hi));
            CK(cudaEventCreateWithFlags(&ctx->solo_fork, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->solo_join, cudaEventDisableTiming));
        }
        if (ctx->solo_n > 0) {
            CK(ctx->solo_col.ensure(solo_scratch_float2(ctx->solo_n)));
            CK(ctx->solo_acc.ensure(solo_scratch_floats(ctx->solo_n)));
        }
    }
    sl->n = ctx->solo_n;
    // they stop taking items when <= 6 items per cluster remain (with items
    // of <= 24 tiles; 10 and 14 measured slower)
    sl->reserve_per_cluster = 6;
    sl->st = ctx->st_solo;
    sl->col = ctx->solo_col.p;
    sl->acc = ctx->solo_acc.p;
    sl->fork = ctx->solo_fork;
    sl->join = ctx->solo_join;
    return GCF_OK;
}

gcf_status fused_launch(gcf_ctx* ctx, int m0, int m1, float* raw_out, cudaStream_t st, bool solo = true)
{
    const std::vector<int>& first = ctx->f_first_h;
    if (m0 < 0 || m1 > (int)first.size() - 1 || m0 >= m1) return fail(ctx, GCF_ERR_STATE, "tile-spectrum range outside the plan");
    const int ni = first[m1] - first[m0];
    int max_blocks = 0;
    for (int i = m0; i < m1; ++i) max_blocks = std::max(max_blocks, ctx->f_blocks_h[i]);
    int ncl = std::min(ctx->fused_clusters, ni);
    if (ctx->kev_used > 256) ctx->kev_used = 0;   // calls that never read their stage times
    while ((int)ctx->kev.size() < ctx->kev_used + 2) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ctx->kev.push_back(e);
    }
    cudaEvent_t e0 = ctx->kev[ctx->kev_used], e1 = ctx->kev[ctx->kev_used + 1];
    ctx->kev_used += 2;
    SoloLaunch sl{};
    if (solo) CKS(solo_setup(ctx, &sl));
    CK(launch_fused(ctx->f_desc.p, ctx->f_bsum_ptr.p, max_blocks, ctx->f_items.p + first[m0], ni, ctx->f_first.p,
                    ctx->f_inv.p, m0, m1 - m0, ctx->taper.p, ctx->tw512.p, ctx->f_partial.p, raw_out,
                    ctx->f_next.p + m0, ncl, ctx->fused_shape, st, e0, e1, solo ? &sl : nullptr));
    ctx->launches += (solo && sl.n > 0 && ni > ncl) ? 4 : 3;
    return GCF_OK;
}

// CGenAvgSpectrum::DoIt for all micrographs in one launch of the fused
// tile-spectrum kernel (tile 512).
gcf_status spectrum_fused(gcf_ctx* ctx, const std::vector<MicImage>& mics, float* raw_out)
{
    CKS(fused_plan(ctx, mics));
    return fused_launch(ctx, 0, (int)mics.size(), raw_out, ctx->st);
}

// Buffers of the spectrum stage for nm micrographs.
gcf_status spectra_alloc(gcf_ctx* ctx, int nm)
{
    int T = ctx->tile, cx = T / 2 + 1;
    size_t cmp_n = (size_t)cx * T;
    CK(ctx->raw.ensure(cmp_n * nm));
    CK(ctx->ctf0.ensure(cmp_n * nm));
    CK(ctx->ctf.ensure(cmp_n * nm));
    CK(ctx->hsum.ensure(cmp_n * nm));
    CK(ctx->moments.ensure(2 * (size_t)nm));
    CK(ctx->lowpassed.ensure(nm));
    CK(ctx->radial.ensure((size_t)cx * nm));
    return GCF_OK;
}

// CGenAvgSpectrum::DoIt for micrographs [first, first + count) of mics, into
// their raw-spectrum slots.
gcf_status spectra_chunk(gcf_ctx* ctx, const std::vector<MicImage>& mics, int first, int count)
{
    size_t cmp_n = (size_t)(ctx->tile / 2 + 1) * ctx->tile;
    if (count <= 0) return GCF_OK;
    if (ctx->impl == GCF_SPECT_FUSED) {
        std::vector<MicImage> sub(mics.begin() + first, mics.begin() + first + count);
        CKS(spectrum_fused(ctx, sub, ctx->raw.p + cmp_n * first));
    } else {
        for (int i = first; i < first + count; ++i) CKS(spectrum_cufft(ctx, mics[i], ctx->raw.p + cmp_n * i));
    }
    return GCF_OK;
}

// CFindCtfBase::mRemoveBackground/mLowpass and CFindCtf1D::mCalcRadialAverage
// for slots first .. first + nm - 1.
gcf_status spectra_post(gcf_ctx* ctx, int nm, int first = 0)
{
    int T = ctx->tile, cx = T / 2 + 1;
    size_t cmp_n = (size_t)cx * T;
    if (nm <= 0) return GCF_OK;
    const size_t o = (size_t)first * cmp_n;
    launch_bg_horizontal(ctx->raw.p + o, T, nm, ctx->log_spect, ctx->hsum.p + o, ctx->st);
    CKL();
    launch_bg_vertical(ctx->raw.p + o, ctx->hsum.p + o, T, nm, ctx->log_spect, ctx->ctf0.p + o, ctx->st);
    CKL();
    launch_moments(ctx->ctf0.p + o, (int)cmp_n, nm, ctx->moments.p + 2 * (size_t)first, ctx->st);
    CKL();
    // CFindCtfBase::mLowpass (FindCTF/CFindCtfBase.cpp:191-219): full
    // spectrum, R2C, B-factor 10 (normalised), C2R, half back.  Tile 512
    // with the hand-written spectrum path: the separable filter on the warp
    // FFT (launch_lowpass512); otherwise (and for the cuFFT comparison
    // variant) batched cuFFT.
    CK(ctx->lpfull.ensure((size_t)nm * T * T));
    if (ctx->impl == GCF_SPECT_FUSED && fused_tile_supported(T)) {
        CK(launch_lowpass512(ctx->ctf0.p + o, ctx->tw512.p, 10.0, nm, ctx->moments.p + 2 * (size_t)first,
                             ctx->lpfull.p, ctx->ctf.p + o, ctx->lowpassed.p + first, ctx->st));
        launch_radial(ctx->ctf.p + o, T, nm, ctx->rad_off.p, ctx->rad_pix.p, ctx->radial.p + (size_t)first * cx,
                      ctx->st);
        CKL();
        ctx->launches += 6;
        return GCF_OK;
    }
    CK(ctx->lpcmp.ensure((size_t)nm * cx * T));
    launch_lp_full(ctx->ctf0.p + o, T, nm, ctx->lpfull.p, ctx->st);
    CKL();
    cufftHandle pf, pi;
    CKS(get_plan(ctx, 3, T, nm, &pf));
    CKS(get_plan(ctx, 4, T, nm, &pi));
    if (cufftSetStream(pf, ctx->st) != CUFFT_SUCCESS || cufftSetStream(pi, ctx->st) != CUFFT_SUCCESS)
        return fail(ctx, GCF_ERR_CUFFT, "cufftSetStream (lowpass) failed");
    if (cufftExecR2C(pf, ctx->lpfull.p, (cufftComplex*)ctx->lpcmp.p) != CUFFT_SUCCESS)
        return fail(ctx, GCF_ERR_CUFFT, "cufftExecR2C (lowpass) failed");
    if (ctx->lp_g_tile != T) {   // filter table of this tile size (B-factor 10)
        CK(ctx->lp_g.ensure((size_t)cx * T));
        launch_lp_table(ctx->lp_g.p, T, 10.0, ctx->st);
        CKL();
        ctx->lp_g_tile = T;
    }
    launch_lp_filter(ctx->lpcmp.p, T, nm, ctx->lp_g.p, ctx->st);
    CKL();
    if (cufftExecC2R(pi, (cufftComplex*)ctx->lpcmp.p, ctx->lpfull.p) != CUFFT_SUCCESS)
        return fail(ctx, GCF_ERR_CUFFT, "cufftExecC2R (lowpass) failed");
    launch_lp_extract(ctx->ctf0.p + o, ctx->lpfull.p, T, nm, ctx->moments.p + 2 * (size_t)first,
                      ctx->ctf.p + o, ctx->lowpassed.p + first, ctx->st);
    CKL();
    launch_radial(ctx->ctf.p + o, T, nm, ctx->rad_off.p, ctx->rad_pix.p, ctx->radial.p + (size_t)first * cx,
                  ctx->st);
    CKL();
    ctx->launches += 7;
    return GCF_OK;
}

// CFindCtfBase::GenHalfSpectrum for n micrographs (slots 0..n-1):
// spectrum, background removal, moments, lowpass, radial average.
gcf_status spectra(gcf_ctx* ctx, const std::vector<MicImage>& mics)
{
    int nm = (int)mics.size();
    CKS(spectra_alloc(ctx, nm));
    CK(record_timing(ctx->ev[2], ctx->st));
    CKS(spectra_chunk(ctx, mics, 0, nm));
    CK(record_timing(ctx->ev[3], ctx->st));
    CKS(spectra_post(ctx, nm));
    CK(record_timing(ctx->ev[4], ctx->st));
    return GCF_OK;
}

// Host description of one search job.
struct JobSpec {
    int mic;
    int mode;   // 0 Do2D, 1 Refine
    gcf_optics optics;
    float px_n;
    float phase_deg, phase_range;     // Do2D: CFindCtfBase::m_fExtPhase / m_fPhaseRange
    float rin[8];                     // Refine: {df, df_range, ast, ast_range, ang, ang_range, ph, ph_range}
    float held_phase;                 // extra phase the search object holds on entry (0 after Setup1)
    float r1d_df, r1d_range;          // Refine1D: initial defocus and window (Angstrom)
};

// CFindDefocus2D::Setup3 + Refine (FindCTF/CFindDefocus2D.cpp:98-151) on the host.
void refine_init(SearchJob& J, const float* rin)
{
    J.df_mean = rin[0];
    J.ast_ratio = rin[2];
    J.ast_angle = rin[4];
    J.phase_range[0] = rin[6];
    J.ext_phase = J.held_phase;   // replaced by phase_range[0] after the astigmatism grid
    float h = 0.5f * rin[1];
    J.df_range[0] = fmaxf(J.df_mean - h, 3000.0f);
    J.df_range[1] = J.df_mean + h;
    h = 0.5f * rin[3];
    J.ast_range[0] = fmaxf(J.ast_ratio - h, 0.0f);
    J.ast_range[1] = fminf(J.ast_ratio + h, 0.02f);
    h = 0.5f * rin[5];
    J.ang_range[0] = fmaxf(J.ast_angle - h, -90.0f);
    J.ang_range[1] = fminf(J.ast_angle + h, 90.0f);
    J.phase_range[1] = rin[7];
}

// Runs the 1D + 2D searches of `specs` on the spectra already in their
// slots; results in job order.
// A search whose launches are enqueued on `st` and whose results have not
// been read back yet.
struct SearchPending {
    int nj = 0;
    std::vector<int> band;   // band slot of each job
    cudaStream_t st = nullptr;
};

gcf_status run_search_enqueue(gcf_ctx* ctx, const std::vector<JobSpec>& specs, SearchPending& pend)
{
    int nj = (int)specs.size();
    pend.nj = nj;
    pend.st = ctx->st;
    pend.band.assign(nj, 0);
    if (nj == 0) return GCF_OK;
    int T = ctx->tile, cx = T / 2 + 1;
    size_t cmp_n = (size_t)cx * T;
    std::vector<SearchJob> jh(nj);
    std::vector<int> soff(nj);
    int tot = 0, max_band = 0;
    bool any_full = false, any_grid = false, any_phase = false, any_1d = false;
    for (int j = 0; j < nj; ++j) {
        const JobSpec& s = specs[j];
        SearchJob& J = jh[j];
        std::memset(&J, 0, sizeof(J));
        int slot = -1;
        CKS(get_band(ctx, s.optics, s.px_n, &slot));
        J.mic = s.mic;
        J.band = slot;
        J.mode = s.mode;
        J.o = make_optics(s.optics, s.px_n);
        J.phase_range_in = fmaxf(s.phase_range, 0.0f);
        J.ext_phase_in = s.phase_deg;
        J.held_phase = s.held_phase;
        J.r1d_df = s.r1d_df;
        J.r1d_range = s.r1d_range;
        J.step = STEP_CC0;
        if (s.mode >= 2) {
            any_1d = true;
        } else if (s.mode == 1) {
            refine_init(J, s.rin);
            if (J.ast_range[1] - J.ast_range[0] >= (float)1e-20 ||
                J.ang_range[1] - J.ang_range[0] >= (float)1e-20)
                any_grid = true;
            if (J.phase_range[1] > 0) any_phase = true;
        } else {
            any_full = true;
            any_grid = true;
            if (J.phase_range_in > 0) any_phase = true;
        }
        soff[j] = tot;
        int bn = ctx->bands[slot]->n;
        tot += bn;
        max_band = std::max(max_band, bn);
    }
    CKS(upload_bands(ctx));
    int max_chunks = std::max(1, (max_band + kEvalChunk - 1) / kEvalChunk);
    CK(ctx->jobs.ensure(nj));
    CK(ctx->spec_off.ensure(nj));
    CK(ctx->band_spec.ensure(std::max(tot, 1)));
    CK(ctx->sum_ss.ensure(nj));
    CK(ctx->cand.ensure((size_t)nj * kMaxCand));
    CK(ctx->cval.ensure((size_t)nj * kMaxCand));
    CK(ctx->part.ensure((size_t)nj * kMaxCand * max_chunks));
    CK(ctx->cc_res.ensure((size_t)nj * cx));
    CK(ctx->d_res.ensure(nj));
    CK(ctx->arrive.ensure(nj));
    CK(cudaMemsetAsync(ctx->arrive.p, 0, nj * sizeof(int), ctx->st));
    CK(h2d(ctx, ctx->jobs.p, jh.data(), nj * sizeof(SearchJob), ctx->st));
    CK(h2d(ctx, ctx->spec_off.p, soff.data(), nj * sizeof(int), ctx->st));
    launch_band_gather(ctx->ctf.p, (int)cmp_n, ctx->jobs.p, ctx->d_bands.p, ctx->spec_off.p, nj,
                       ctx->band_spec.p, ctx->sum_ss.p, ctx->st);
    CKL();
    ctx->launches += 1;
    EvalArgs a;
    a.jobs = ctx->jobs.p;
    a.bands = ctx->d_bands.p;
    a.band_spec = ctx->band_spec.p;
    a.sum_ss = ctx->sum_ss.p;
    a.spec_off = ctx->spec_off.p;
    a.cand = ctx->cand.p;
    a.cval = ctx->cval.p;
    a.part = ctx->part.p;
    a.arrive = ctx->arrive.p;
    a.max_chunks = max_chunks;
    a.njobs = nj;
    CK(record_timing(ctx->ev[5], ctx->st));
    if (any_full || any_1d) {
        launch_search1d(ctx->jobs.p, nj, ctx->radial.p, cx, ctx->cand.p, ctx->cval.p, ctx->st);
        CKL();
        ctx->launches += 1;
    }
    launch_init_jobs(a, ctx->st);   // Refine jobs: pending step CC0
    CKL();
    ctx->launches += 1;
    CK(record_timing(ctx->ev[6], ctx->st));
    // Upper bound of non-empty steps: CC0 + astigmatism grid + 19 x 4 refinements.
    bool any_2d = false;
    for (const JobSpec& s : specs) any_2d = any_2d || s.mode <= 1;
    int pairs = any_2d ? 2 + 19 * ((any_grid ? 2 : 0) + 1 + (any_phase ? 1 : 0)) : 0;
    // Candidate blocks per (chunk, job) of the line searches (<= 61
    // candidates, 4 blocks of 16): one block loops over the candidate blocks
    // it is given, reusing its pixels, so with many jobs fewer y-blocks
    // (enough for about two waves of 3 CTAs per SM) do the same work without
    // the blocks that find no candidates and exit.
    if (ctx->n_sms == 0) CK(cudaDeviceGetAttribute(&ctx->n_sms, cudaDevAttrMultiProcessorCount, ctx->dev));
    const long long per_y = (long long)nj * max_chunks;
    const int line_cb = (int)std::min<long long>(4, std::max<long long>(1, (2LL * 3 * ctx->n_sms + per_y - 1) / per_y));
    for (int k = 0; k < pairs; ++k) {
        int cb = (k == 0) ? 1 : (k == 1 && any_grid) ? (kMaxCand / kEvalCB + 3) / 4 : line_cb;
        launch_eval2d(a, cb, max_band, ctx->st);
        CKL();
        ctx->launches += 1;
    }
    if (any_2d) {
        // GSpectralCC2D resolution (FindCTF/CFindDefocus2D.cpp:382-400)
        CK(ctx->ring_sums.ensure((size_t)nj * cx * 6));
        launch_ctf_res(ctx->ctf.p, T, ctx->jobs.p, nj, ctx->ring_off.p, ctx->ring_pix.p, ctx->ring_geo.p,
                       ctx->ring_sums.p, ctx->cc_res.p, ctx->st);
        CKL();
        launch_shell_select(ctx->jobs.p, nj, ctx->cc_res.p, cx, T, ctx->st);
        CKL();
        ctx->launches += 3;
    }
    CK(ctx->d_counts.ensure(3 * (size_t)nj));
    launch_results(ctx->jobs.p, nj, ctx->lowpassed.p, ctx->d_res.p, ctx->d_counts.p, ctx->st);
    CKL();
    ctx->launches += 1;
    CK(record_timing(ctx->ev[7], ctx->st));
    for (int j = 0; j < nj; ++j) pend.band[j] = jh[j].band;
    return GCF_OK;
}

// Reads back the results of an enqueued search (waits for it on the host).
// The tensor-core rescale's flag, read back with a call's results: a
// bounded wait of its products gave up (the flag is cleared for the next
// call).
gcf_status check_rescale_gemm(gcf_ctx* ctx, int flag)
{
    if (!flag) return GCF_OK;
    CK(cudaMemset(ctx->rsg_err.p, 0, sizeof(int)));
    return fail(ctx, GCF_ERR_TIMEOUT, "tensor-core rescale product: a bounded wait gave up");
}

gcf_status run_search_collect(gcf_ctx* ctx, const SearchPending& pend, std::vector<gcf_result>& out)
{
    const int nj = pend.nj;
    out.assign(nj, gcf_result{});
    if (nj == 0) return GCF_OK;
    CK(cudaMemcpyAsync(out.data(), ctx->d_res.p, nj * sizeof(gcf_result), cudaMemcpyDeviceToHost, pend.st));
    std::vector<int> cnt(3 * (size_t)nj);
    CK(cudaMemcpyAsync(cnt.data(), ctx->d_counts.p, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, pend.st));
    int rs_err = 0;
    if (ctx->rsg_err.p)
        CK(cudaMemcpyAsync(&rs_err, ctx->rsg_err.p, sizeof(int), cudaMemcpyDeviceToHost, pend.st));
    CK(cudaStreamSynchronize(pend.st));
    CKS(check_rescale_gemm(ctx, rs_err));
    for (int j = 0; j < nj; ++j) {
        const long long n2 = cnt[3 * j], n1 = cnt[3 * j + 1], p1 = cnt[3 * j + 2];
        ctx->search_counts[0] += n2;
        ctx->search_counts[1] += n2 * (long long)ctx->bands[pend.band[j]]->n;
        ctx->search_counts[2] += n1;
        ctx->search_counts[3] += p1;
    }
    float t1 = 0, t2 = 0;
    cudaEventElapsedTime(&t1, ctx->ev[5], ctx->ev[6]);
    cudaEventElapsedTime(&t2, ctx->ev[6], ctx->ev[7]);
    ctx->stage_ms[4] += t1;
    ctx->stage_ms[5] += t2;
    return GCF_OK;
}

gcf_status run_search(gcf_ctx* ctx, const std::vector<JobSpec>& specs, std::vector<gcf_result>& out)
{
    SearchPending pend;
    CKS(run_search_enqueue(ctx, specs, pend));
    return run_search_collect(ctx, pend, out);
}

// ---------------------------------------------------------------------------
// BF16 contraction search (mode 4 jobs).  Every step is enqueued on ctx->st
// with no host round trip until the results are read back:
//   polar binning of the ctf spectra -> tile plan -> P = A B^T and
//   Dz = E A2^T on the tensor cores -> table search (1D scan + mIterate, or
//   the learned window) -> FP32 re-score of the table's best candidates and
//   kLocalPasses local passes (k_eval2d) -> GSpectralCC2D resolution ->
//   result rows.
// `prior` (device, nullable): per job (mean A, ratio, angle, window scale);
// jobs with prior.x > 0 search the window around it.

// The batch's polar grid: the s^2 band common to all jobs (the 2D band of
// CFindDefocus2D::Setup2, FindCTF/CFindDefocus2D.cpp:86-92, in 1/A), and the
// defocus rows that cover every job's search.
PolarGrid polar_grid(gcf_ctx* ctx, const std::vector<JobSpec>& specs)
{
    double s_lo = 0.0, s_hi = 1e30, z_lo = 1e30, z_hi = 0.0;
    for (const JobSpec& sp : specs) {
        float rr[2];
        res_range_of(sp.px_n, rr);
        s_lo = std::max(s_lo, 1.0 / rr[0]);
        s_hi = std::min(s_hi, 1.0 / rr[1]);
        const double px2 = (double)sp.px_n * sp.px_n;
        z_lo = std::min(z_lo, 3000.0 * px2 * 0.82 * 0.96);
        z_hi = std::max(z_hi, 30000.0 * px2 * 1.2 * 1.04);
    }
    PolarGrid g{};
    g.ns = ctx->contract_ns;
    g.nth = ctx->contract_nth;
    g.s2_lo = (float)(s_lo * s_lo);
    g.ds2 = (float)((s_hi * s_hi - s_lo * s_lo) / g.ns);
    g.dz = ctx->contract_dz;
    g.z0 = (float)(std::floor(z_lo / g.dz) * g.dz);
    g.nz = (int)std::ceil((z_hi - g.z0) / g.dz) + 2;
    g.nz = (g.nz + 127) / 128 * 128;
    const gcf_optics& op = specs[0].optics;
    const double wl = 12.26 / std::sqrt((double)op.kv * 1000.0 + 0.9784 * (double)op.kv * op.kv);
    g.wl = (float)wl;
    g.cs = (float)((double)op.cs_mm * 1e7);
    const float ac = op.amp_contrast;
    g.amp_phase = (float)atanf(ac / sqrtf(1.0f - ac * ac)) + specs[0].phase_deg * 0.01745329f;
    return g;
}

bool same_grid(const PolarGrid& a, const PolarGrid& b)
{
    return a.ns == b.ns && a.nth == b.nth && a.nz == b.nz && a.s2_lo == b.s2_lo && a.ds2 == b.ds2 &&
           a.z0 == b.z0 && a.dz == b.dz && a.wl == b.wl && a.cs == b.cs && a.amp_phase == b.amp_phase;
}

gcf_status run_fast_enqueue(gcf_ctx* ctx, const std::vector<JobSpec>& specs, const float4* prior,
                            SearchPending& pend)
{
    const int nj = (int)specs.size();
    pend.nj = nj;
    pend.st = ctx->st;
    pend.band.assign(nj, 0);
    if (nj == 0) return GCF_OK;
    const int T = ctx->tile, cx = T / 2 + 1;
    const size_t cmp_n = (size_t)cx * T;
    std::vector<SearchJob> jh(nj);
    std::vector<int> soff(nj);
    int tot = 0, max_band = 0;
    for (int j = 0; j < nj; ++j) {
        const JobSpec& sp = specs[j];
        SearchJob& J = jh[j];
        std::memset(&J, 0, sizeof(J));
        int slot = -1;
        CKS(get_band(ctx, sp.optics, sp.px_n, &slot));
        J.mic = sp.mic;
        J.band = slot;
        J.mode = 4;
        J.o = make_optics(sp.optics, sp.px_n);
        J.ext_phase_in = sp.phase_deg;
        J.held_phase = sp.held_phase;
        J.step = STEP_DONE;
        soff[j] = tot;
        const int bn = ctx->bands[slot]->n;
        tot += bn;
        max_band = std::max(max_band, bn);
    }
    CKS(upload_bands(ctx));
    const int max_chunks = std::max(1, (max_band + kEvalChunk - 1) / kEvalChunk);
    CK(ctx->jobs.ensure(nj));
    CK(ctx->spec_off.ensure(nj));
    CK(ctx->band_spec.ensure(std::max(tot, 1)));
    CK(ctx->sum_ss.ensure(nj));
    CK(ctx->cand.ensure((size_t)nj * kMaxCand));
    CK(ctx->cval.ensure((size_t)nj * kMaxCand));
    CK(ctx->part.ensure((size_t)nj * kMaxCand * max_chunks));
    CK(ctx->cc_res.ensure((size_t)nj * cx));
    CK(ctx->d_res.ensure(nj));
    CK(ctx->arrive.ensure(nj));
    CK(cudaMemsetAsync(ctx->arrive.p, 0, nj * sizeof(int), ctx->st));
    CK(h2d(ctx, ctx->jobs.p, jh.data(), nj * sizeof(SearchJob), ctx->st));
    CK(h2d(ctx, ctx->spec_off.p, soff.data(), nj * sizeof(int), ctx->st));
    CK(record_timing(ctx->ev[5], ctx->st));
    launch_band_gather(ctx->ctf.p, (int)cmp_n, ctx->jobs.p, ctx->d_bands.p, ctx->spec_off.p, nj, ctx->band_spec.p,
                       ctx->sum_ss.p, ctx->st);
    CKL();
    // model rows of the grid (kept while the grid and optics stay the same)
    const PolarGrid g = polar_grid(ctx, specs);
    if (!ctx->have_model || !same_grid(g, ctx->model_grid)) {
        CK(ctx->cA.ensure((size_t)g.nz * g.ns));
        CK(ctx->cA2.ensure((size_t)g.nz * g.ns));
        launch_polar_model(g, ctx->cA.p, ctx->cA2.p, ctx->st);
        CKL();
        ctx->launches += 1;
        ctx->model_grid = g;
        ctx->have_model = true;
        ctx->model_version += 1;
    }
    const long long ncols = (long long)nj * g.nth;
    CK(ctx->cB.ensure((size_t)ncols * g.ns));
    CK(ctx->cE.ensure((size_t)nj * g.ns));
    CK(ctx->cSS.ensure(nj));
    CK(ctx->cP.ensure((size_t)g.nz * ncols));
    CK(ctx->cDz.ensure((size_t)nj * g.nz));
    CK(ctx->cRows.ensure(nj));
    const int bn = ctx->gemm_bn;
    if (bn < g.nth || bn % g.nth) return fail(ctx, GCF_ERR_INVALID_ARG, "contraction tile narrower than a job's angle bins");
    const int ncb = (int)((ncols + bn - 1) / bn);
    const int max_tiles = ncb * (g.nz / 128);
    CK(ctx->cTiles.ensure(max_tiles));
    CK(ctx->cNtiles.ensure(1));
    CK(ctx->cErr.ensure(1));
    for (auto& e : ctx->fev)
        if (!e) CK(cudaEventCreate(&e));
    CK(record_timing(ctx->fev[0], ctx->st));
    CK(launch_polar_bin(ctx->ctf.p, T, ctx->jobs.p, nj, g, ctx->cB.p, ctx->cE.p, ctx->cSS.p, ctx->st));
    launch_job_rows(ctx->jobs.p, nj, prior, g, ctx->cRows.p, ctx->st);
    CKL();
    CK(cudaMemsetAsync(ctx->cNtiles.p, 0, sizeof(int), ctx->st));
    CK(cudaMemsetAsync(ctx->cErr.p, 0, sizeof(int), ctx->st));
    CK(record_timing(ctx->fev[1], ctx->st));
    launch_plan_tiles(ctx->cRows.p, nj, g.nth, g.nz, bn, ctx->cTiles.p, ctx->cNtiles.p, max_tiles, ctx->st);
    CKL();
    // P = A B^T over the planned tiles; Dz = E A2^T (every row of every job)
    GemmArgs ga;
    ga.M = g.nz;
    ga.N = (int)ncols;
    ga.K = g.ns;
    ga.D = ctx->cP.p;
    ga.ldd = ncols;
    ga.tiles = ctx->cTiles.p;
    ga.ntiles = ctx->cNtiles.p;
    ga.err = ctx->cErr.p;
    if (ctx->gemm_persistent)
        CK(launch_umma_gemm_persistent(ctx->cA.p, g.ns, ctx->cB.p, g.ns, ga, bn, ctx->gemm_stages, max_tiles,
                                       ctx->st));
    else
        CK(launch_umma_gemm(ctx->cA.p, g.ns, ctx->cB.p, g.ns, ga, bn, ctx->gemm_stages, max_tiles, ctx->st));
    GemmArgs gd;
    gd.M = nj;
    gd.N = g.nz;
    gd.K = g.ns;
    gd.D = ctx->cDz.p;
    gd.ldd = g.nz;
    gd.err = ctx->cErr.p;
    CK(launch_umma_gemm(ctx->cE.p, g.ns, ctx->cA2.p, g.ns, gd, 256, 4, 0, ctx->st));
    ctx->launches += 6;
    CK(record_timing(ctx->fev[2], ctx->st));
    TableArgs ta;
    ta.jobs = ctx->jobs.p;
    ta.njobs = nj;
    ta.P = ctx->cP.p;
    ta.ldp = ncols;
    ta.Dz = ctx->cDz.p;
    ta.ldd = g.nz;
    ta.ss = ctx->cSS.p;
    ta.g = g;
    ta.rows = ctx->cRows.p;
    ta.prior = prior;
    ta.cand = ctx->cand.p;
    ta.cval = ctx->cval.p;
    launch_table_search(ta, ctx->st);
    CKL();
    ctx->launches += 1;
    CK(record_timing(ctx->ev[6], ctx->st));
    CK(record_timing(ctx->fev[3], ctx->st));
    EvalArgs a;
    a.jobs = ctx->jobs.p;
    a.bands = ctx->d_bands.p;
    a.band_spec = ctx->band_spec.p;
    a.sum_ss = ctx->sum_ss.p;
    a.spec_off = ctx->spec_off.p;
    a.cand = ctx->cand.p;
    a.cval = ctx->cval.p;
    a.part = ctx->part.p;
    a.arrive = ctx->arrive.p;
    a.max_chunks = max_chunks;
    a.njobs = nj;
    // FP32 re-score + local passes: candidate blocks of 16 (<= 27 per step)
    for (int k = 0; k < 1 + kLocalPasses; ++k) {
        launch_eval2d(a, 2, max_band, ctx->st);
        CKL();
        ctx->launches += 1;
    }
    CK(record_timing(ctx->fev[4], ctx->st));
    CK(ctx->ring_sums.ensure((size_t)nj * cx * 6));
    launch_ctf_res(ctx->ctf.p, T, ctx->jobs.p, nj, ctx->ring_off.p, ctx->ring_pix.p, ctx->ring_geo.p,
                   ctx->ring_sums.p, ctx->cc_res.p, ctx->st);
    CKL();
    launch_shell_select(ctx->jobs.p, nj, ctx->cc_res.p, cx, T, ctx->st);
    CKL();
    CK(ctx->d_counts.ensure(3 * (size_t)nj));
    launch_results(ctx->jobs.p, nj, ctx->lowpassed.p, ctx->d_res.p, ctx->d_counts.p, ctx->st);
    CKL();
    ctx->launches += 4;
    CK(record_timing(ctx->ev[7], ctx->st));
    for (int j = 0; j < nj; ++j) pend.band[j] = jh[j].band;
    return GCF_OK;
}

// Reads back a contraction search: results, per-job work, the product's
// error flag.
gcf_status run_fast_collect(gcf_ctx* ctx, const SearchPending& pend, std::vector<gcf_result>& out,
                            std::vector<int>* n_table)
{
    CKS(run_search_collect(ctx, pend, out));
    const int nj = pend.nj;
    if (nj == 0) return GCF_OK;
    std::vector<SearchJob> jh(nj);
    int err = 0, nt = 0;
    CK(cudaMemcpyAsync(jh.data(), ctx->jobs.p, nj * sizeof(SearchJob), cudaMemcpyDeviceToHost, pend.st));
    CK(cudaMemcpyAsync(&err, ctx->cErr.p, sizeof(int), cudaMemcpyDeviceToHost, pend.st));
    CK(cudaMemcpyAsync(&nt, ctx->cNtiles.p, sizeof(int), cudaMemcpyDeviceToHost, pend.st));
    CK(cudaStreamSynchronize(pend.st));
    if (err) return fail(ctx, GCF_ERR_TIMEOUT, "tensor-core product: a bounded wait gave up");
    for (int k = 0; k < 4; ++k) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, ctx->fev[k], ctx->fev[k + 1]) == cudaSuccess) ctx->fast_ms[k] += t;
    }
    cudaGetLastError();
    // tensor-core multiply-adds: the planned tiles of P and all of Dz
    const PolarGrid& g = ctx->model_grid;
    ctx->fast_counts[1] += (long long)nt * 128 * ctx->gemm_bn * g.ns + (long long)nj * g.nz * g.ns;
    if (n_table) n_table->assign(nj, 0);
    for (int j = 0; j < nj; ++j) {
        ctx->fast_counts[0] += jh[j].n_table;
        ctx->fast_counts[2] += jh[j].n_cand2d;
        if (n_table) (*n_table)[j] = jh[j].n_table;
    }
    return GCF_OK;
}

// ---------------------------------------------------------------------------
// Searches of the spectra in slots 0 .. n-1 (already post-processed) with
// the chosen method; px_n: pixel size of each slot, optics with the raw
// pixel sizes in px_raw (unused by the searches themselves).
constexpr int kNnChunk = 512;   // network inputs of at most this many jobs at once

gcf_status nn_ensure(gcf_ctx* ctx)
{
    if (ctx->nn) return GCF_OK;
    ctx->nn = nn_create();
    if (!ctx->nn) return fail(ctx, GCF_ERR_NO_MEMORY, "network buffers");
    return GCF_OK;
}

// Learned priors (mean, ratio, angle, window) of slots 0 .. n-1 into cPrior.
gcf_status learned_priors(gcf_ctx* ctx, const std::vector<float>& px_n)
{
    const int n = (int)px_n.size();
    CKS(nn_ensure(ctx));
    if (!ctx->nn_ready) return fail(ctx, GCF_ERR_STATE, "learned search: no network weights (gcf_nn_load / gcf_nn_train)");
    CK(ctx->npx.ensure(n));
    CK(ctx->cPrior.ensure(n));
    CK(ctx->nx1.ensure((size_t)kNnChunk * kNnProfile));
    CK(ctx->nx2.ensure((size_t)kNnChunk * kNnMap * kNnMap));
    for (auto& e : ctx->fev)
        if (!e) CK(cudaEventCreate(&e));
    CK(record_timing(ctx->fev[5], ctx->st));
    CK(h2d(ctx, ctx->npx.p, px_n.data(), n * sizeof(float), ctx->st));
    const size_t cmp_n = (size_t)(ctx->tile / 2 + 1) * ctx->tile;
    for (int c0 = 0; c0 < n; c0 += kNnChunk) {
        const int cn = std::min(kNnChunk, n - c0);
        CK(launch_nn_input(ctx->ctf.p + cmp_n * c0, ctx->tile, ctx->npx.p + c0, 1, cn, ctx->nx1.p, ctx->nx2.p, ctx->st));
        CK(nn_forward(ctx->nn, ctx->nx1.p, ctx->nx2.p, cn, ctx->st));
        launch_prior(nn_pred(ctx->nn), kNnPredPitch, cn, ctx->cPrior.p + c0, ctx->st);
        CKL();
        ctx->launches += 13;   // inputs, first layer, 3 im2col, 6 products, concat, prior
    }
    CK(record_timing(ctx->fev[6], ctx->st));
    return GCF_OK;
}

// Search jobs of slots 0 .. n-1 for a method.  raw_px (nullable): the raw
// pixel size of each slot, kept in its optics as gcf_run_batch does.
std::vector<JobSpec> slot_jobs(const std::vector<float>& px_n, const float* raw_px, const gcf_optics& op, int mode)
{
    const int n = (int)px_n.size();
    std::vector<JobSpec> js(n);
    for (int i = 0; i < n; ++i) {
        std::memset(&js[i], 0, sizeof(JobSpec));
        js[i].mic = i;
        js[i].mode = mode == GCF_SEARCH_PLAIN ? 0 : 4;
        js[i].optics = op;
        if (raw_px) js[i].optics.pixel_size = raw_px[i];
        js[i].px_n = px_n[i];
        js[i].phase_deg = op.ext_phase_deg;
        js[i].phase_range = mode == GCF_SEARCH_PLAIN ? fmaxf(op.ext_phase_range, 0.0f) : 0.0f;
    }
    return js;
}

// Enqueues the searches of slots 0 .. n-1 (already post-processed) with
// the chosen method; nothing is read back.
gcf_status search_enqueue(gcf_ctx* ctx, const std::vector<float>& px_n, const float* raw_px, const gcf_optics& op,
                          int mode, SearchPending& pend)
{
    std::vector<JobSpec> js = slot_jobs(px_n, raw_px, op, mode);
    if (mode == GCF_SEARCH_PLAIN) return run_search_enqueue(ctx, js, pend);
    const float4* prior = nullptr;
    if (mode == GCF_SEARCH_LEARNED) {
        CKS(learned_priors(ctx, px_n));
        prior = ctx->cPrior.p;
    }
    return run_fast_enqueue(ctx, js, prior, pend);
}

// Reads back an enqueued search.  A learned search falls back to the full
// contraction search where the learned window's refined result is not
// trusted: its CC is below the threshold, or its mean defocus ends within
// two final steps of the window's edge (the optimum may lie outside).
gcf_status search_collect(gcf_ctx* ctx, const std::vector<float>& px_n, const float* raw_px, const gcf_optics& op,
                          int mode, const SearchPending& pend, std::vector<gcf_result>& out)
{
    if (mode == GCF_SEARCH_PLAIN) return run_search_collect(ctx, pend, out);
    CKS(run_fast_collect(ctx, pend, out, nullptr));
    if (mode != GCF_SEARCH_LEARNED) return GCF_OK;
    {
        float t = 0.0f;   // the network's inputs and layers (learned_priors)
        if (cudaEventElapsedTime(&t, ctx->fev[5], ctx->fev[6]) == cudaSuccess) ctx->fast_ms[4] += t;
        cudaGetLastError();
    }
    const int n = (int)px_n.size();
    std::vector<SearchJob> jh(n);
    CK(cudaMemcpy(jh.data(), ctx->jobs.p, n * sizeof(SearchJob), cudaMemcpyDeviceToHost));
    std::vector<JobSpec> js = slot_jobs(px_n, raw_px, op, mode), redo;
    std::vector<int> idx;
    for (int i = 0; i < n; ++i) {
        const SearchJob& J = jh[i];
        const float edge = 2.0f * fmaxf(20.0f, 0.105f * J.df_mean / 31.0f);
        const bool at_edge = J.df_mean - J.df_range[0] < edge || J.df_range[1] - J.df_mean < edge;
        if (out[i].score < ctx->learned_tau || at_edge) {
            redo.push_back(js[i]);
            idx.push_back(i);
        }
    }
    ctx->fast_counts[3] += (long long)redo.size();
    if (redo.empty()) return GCF_OK;
    // the fallback's counts and times add to the first pass's
    std::vector<gcf_result> r2;
    SearchPending p2;
    CKS(run_fast_enqueue(ctx, redo, nullptr, p2));
    CKS(run_fast_collect(ctx, p2, r2, nullptr));
    for (size_t k = 0; k < idx.size(); ++k) out[idx[k]] = r2[k];
    return GCF_OK;
}

gcf_status search_slots(gcf_ctx* ctx, const std::vector<float>& px_n, const gcf_optics& op, int mode,
                        std::vector<gcf_result>& out)
{
    SearchPending pend;
    CKS(search_enqueue(ctx, px_n, nullptr, op, mode, pend));
    return search_collect(ctx, px_n, nullptr, op, mode, pend, out);
}

// Synthetic raw spectra of samples first .. first + n - 1 of the generator
// (seed) into slots 0 .. n-1, post-processed like measured ones; their
// pixel sizes to px_n and parameters (8 floats each) to nparams.
gcf_status synth_slots(gcf_ctx* ctx, const gcf_optics& op, unsigned long long seed, unsigned long long first, int n)
{
    CKS(spectra_alloc(ctx, n));
    CK(ctx->nparams.ensure((size_t)n * 8));
    CK(ctx->ntarget.ensure((size_t)n * 3));
    launch_synth_params(seed, first, n, ctx->nparams.p, ctx->ntarget.p, ctx->st);
    launch_synth_raw(seed, first, ctx->nparams.p, n, ctx->tile, make_optics(op, 1.0f), ctx->raw.p, ctx->st);
    CKL();
    CKS(spectra_post(ctx, n));
    ctx->launches += 2;
    return GCF_OK;
}

gcf_status set_device(gcf_ctx* ctx)
{
    CK(cudaSetDevice(ctx->dev));
    return GCF_OK;
}

// The line-transform rescale takes even raw widths and lines of at most
// kResizeMaxLine (raw rows w/2, columns h and nh, new rows nw/2).
bool rescale_lines_supported(int w, int h, int nw, int nh)
{
    return w % 2 == 0 && nw >= 2 && nh >= 2 && resize_line_ok(w / 2) && resize_line_ok(h) && resize_line_ok(nh) &&
           resize_line_ok(nw / 2);
}

// CRescaleImage::DoIt on the device: returns a dense new_w x new_h image
// (FindCTF/CRescaleImage.cpp:68-99), through the line transforms of
// gcf_resize.cu or through cuFFT like the reference.
gcf_status rescale_device(gcf_ctx* ctx, const float* img, int w, int h, float px, float* out,
                          int* nw_out, int* nh_out, float* px_out, bool* copied)
{
    int nw, nh;
    float pxn;
    gcf_rescale_dims(w, h, px, &nw, &nh, &pxn);
    *nw_out = nw;
    *nh_out = nh;
    *px_out = pxn;
    float bin = 1.2f / px;
    if (bin <= 1) bin = 1.0f;
    if (bin == 1.0f) {
        *copied = false;
        return GCF_OK;
    }
    *copied = true;
    int cxi = w / 2 + 1, cxo = nw / 2 + 1;
    if (ctx->rescale_impl == GCF_RESCALE_LINES && rescale_lines_supported(w, h, nw, nh)) {
        ResizeLine La, Lf, Li, Lc;
        const float2 *tA = nullptr, *tC = nullptr;
        CK(resize_line(w / 2, &La));
        CK(resize_line(h, &Lf));
        CK(resize_line(nh, &Li));
        CK(resize_line(nw / 2, &Lc));
        CK(resize_twiddles(w, -1, w / 2 + 1, &tA));
        CK(resize_twiddles(nw, 1, nw / 2, &tC));
        CK(ctx->rs_cmp.ensure((size_t)cxo * h));
        CK(ctx->rs_crop.ensure((size_t)cxo * nh));
        CK(launch_resize(img, w, h, nw, nh, La, tA, Lf, Li, Lc, tC, ctx->rs_cmp.p, ctx->rs_crop.p, out, ctx->st));
        ctx->launches += 3;
        return GCF_OK;
    }
    if (ctx->rescale_impl == GCF_RESCALE_GEMM && rescale_gemm_supported(w, h, nw, nh)) {
        const RescaleGemmLayout L = rescale_gemm_layout(w, h, nw, nh);
        CK(ctx->rsg_bf.ensure((size_t)L.bf16_elems));
        CK(ctx->rsg_f.ensure((size_t)L.f32_elems));
        if (!ctx->rsg_err.p) {
            CK(ctx->rsg_err.ensure(1));
            CK(cudaMemset(ctx->rsg_err.p, 0, sizeof(int)));
        }
        CK(launch_rescale_gemm(img, w, w, h, nw, nh, ctx->rsg_bf.p, ctx->rsg_f.p, ctx->rsg_err.p, out, ctx->st));
        ctx->launches += 5;
        return GCF_OK;
    }
    CK(ctx->rs_cmp.ensure((size_t)cxi * h));
    CK(ctx->rs_crop.ensure((size_t)cxo * nh));
    if (reinterpret_cast<uintptr_t>(img) & 255) {
        // a caller's device view at an offset: cuFFT's R2C wants an aligned
        // input (staged host images are placed 256-byte aligned)
        CK(ctx->rs_src.ensure((size_t)w * h));
        CK(cudaMemcpyAsync(ctx->rs_src.p, img, (size_t)w * h * sizeof(float), cudaMemcpyDeviceToDevice, ctx->st));
        img = ctx->rs_src.p;
    }
    cufftHandle p1, p2;
    CKS(get_plan(ctx, 1, h, w, &p1));
    CKS(get_plan(ctx, 2, nh, nw, &p2));
    if (cufftExecR2C(p1, (cufftReal*)img, (cufftComplex*)ctx->rs_cmp.p) != CUFFT_SUCCESS)
        return fail(ctx, GCF_ERR_CUFFT, "cufftExecR2C (rescale) failed");
    launch_fourier_crop(ctx->rs_cmp.p, cxi, h, ctx->rs_crop.p, cxo, nh, ctx->st);
    CKL();
    ctx->launches += 1;
    if (cufftExecC2R(p2, (cufftComplex*)ctx->rs_crop.p, (cufftReal*)out) != CUFFT_SUCCESS)
        return fail(ctx, GCF_ERR_CUFFT, "cufftExecC2R (rescale) failed");
    return GCF_OK;
}

bool valid_optics(const gcf_optics* o)
{
    return o && o->kv > 0 && o->cs_mm >= 0 && o->amp_contrast >= 0 && o->amp_contrast < 1 &&
           o->pixel_size > 0;
}

// Uploads (if needed), rescales and produces the spectra of n images.
// One image through CRescaleImage (FindCTF/CRescaleImage.cpp:47-99) to the
// MicImage the spectrum stage reads.
gcf_status stage_image(gcf_ctx* ctx, const float* dimg, int w, int h, float px, float* rescale_dst,
                       MicImage& m, size_t* used)
{
    bool copied = false;
    int nw, nh;
    float pn;
    CKS(rescale_device(ctx, dimg, w, h, px, rescale_dst, &nw, &nh, &pn, &copied));
    *used = 0;
    if (copied) {
        m.img = rescale_dst;
        m.pitch = nw;
        *used = (size_t)nw * nh;
    } else {
        m.img = dimg;
        m.pitch = w;
    }
    m.w = nw;
    m.h = nh;
    m.px_n = pn;
    Layout L = tile_layout(m.w, m.h, ctx->tile);
    if (L.ntx <= 0 || L.nty <= 0 || m.w < ctx->tile || m.h < ctx->tile)
        return fail(ctx, GCF_ERR_IMAGE_TOO_SMALL, "image holds no full tile");
    return GCF_OK;
}

// Images packed in one staging buffer start on 256-byte boundaries (cuFFT
// and the vector loads of the tile kernels want aligned rows).
size_t align_floats(size_t n) { return (n + 63) / 64 * 64; }

// Uploads (host inputs), rescales and produces the spectra of n images.
// Host inputs are uploaded in chunks on a copy stream so that the upload of
// chunk c+1 overlaps the rescale and spectrum of chunk c.
gcf_status prepare_images(gcf_ctx* ctx, const float* const* images, const int* ws, const int* hs,
                          const float* pxs, int n, int on_device, std::vector<MicImage>& mics)
{
    mics.assign(n, MicImage{});
    size_t tot_raw = 0, tot_new = 0;
    for (int i = 0; i < n; ++i) {
        int nw, nh;
        float pn;
        gcf_rescale_dims(ws[i], hs[i], pxs[i], &nw, &nh, &pn);
        tot_raw += align_floats((size_t)ws[i] * hs[i]);
        float bin = 1.2f / pxs[i];
        if (bin > 1) tot_new += align_floats((size_t)nw * nh);
    }
    CKS(spectra_alloc(ctx, n));
    if (tot_new) CK(ctx->rescaled.ensure(tot_new));
    if (!on_device) CK(ctx->images.ensure(tot_raw));
    const int kChunk = on_device ? n : 8;
    const int nchunks = (n + kChunk - 1) / kChunk;
    while ((int)ctx->chunk_ev.size() < nchunks) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->chunk_ev.push_back(e);
    }
    CK(record_timing(ctx->ev[0], ctx->st));
    if (!on_device) {
        if (!ctx->fork_ev) CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ctx->fork_ev, ctx->st));
        CK(cudaStreamWaitEvent(ctx->st_copy, ctx->fork_ev, 0));
    }
    CK(record_timing(ctx->ev[2], ctx->st));
    size_t roff = 0, roff_new = 0;
    for (int c = 0; c < nchunks; ++c) {
        int i0 = c * kChunk, i1 = std::min(n, i0 + kChunk);
        std::vector<const float*> dimg(i1 - i0);
        if (!on_device) {
            for (int i = i0; i < i1; ++i) {
                size_t cnt = (size_t)ws[i] * hs[i];
                CK(cudaMemcpyAsync(ctx->images.p + roff, images[i], cnt * sizeof(float),
                                   cudaMemcpyHostToDevice, ctx->st_copy));
                dimg[i - i0] = ctx->images.p + roff;
                roff += align_floats(cnt);
            }
            // the timing record first: in a capture, the chunk event joins
            // everything on the copy stream back into st
            if (c == nchunks - 1) CK(record_timing(ctx->ev[1], ctx->st_copy));
            CK(cudaEventRecord(ctx->chunk_ev[c], ctx->st_copy));
            CK(cudaStreamWaitEvent(ctx->st, ctx->chunk_ev[c], 0));
        } else {
            for (int i = i0; i < i1; ++i) dimg[i - i0] = images[i];
            if (c == 0) CK(record_timing(ctx->ev[1], ctx->st));
        }
        for (int i = i0; i < i1; ++i) {
            size_t used = 0;
            float* dst = tot_new ? ctx->rescaled.p + roff_new : nullptr;
            CKS(stage_image(ctx, dimg[i - i0], ws[i], hs[i], pxs[i], dst, mics[i], &used));
            roff_new += align_floats(used);
        }
        CKS(spectra_chunk(ctx, mics, i0, i1 - i0));
    }
    CK(record_timing(ctx->ev[3], ctx->st));
    CKS(spectra_post(ctx, n));
    CK(record_timing(ctx->ev[4], ctx->st));
    return GCF_OK;
}

// Stage times of the last call.  The tile-kernel time is the union of the
// launches' [begin, end] intervals (launches on two streams may overlap),
// measured from ev[0]; where ev[0] was not recorded, the sum of durations.
void accumulate_stage_times(gcf_ctx* ctx)
{
    float t;
    std::vector<std::pair<float, float>> iv;
    bool rel = true;
    for (int i = 0; i + 1 < ctx->kev_used; i += 2) {
        float a = 0.0f, b = 0.0f;
        if (rel && cudaEventElapsedTime(&a, ctx->ev[0], ctx->kev[i]) == cudaSuccess &&
            cudaEventElapsedTime(&b, ctx->ev[0], ctx->kev[i + 1]) == cudaSuccess) {
            iv.emplace_back(a, b);
        } else {
            rel = false;
        }
    }
    if (rel) {
        std::sort(iv.begin(), iv.end());
        float end = -1e30f;
        for (auto& x : iv) {
            float a = std::max(x.first, end);
            if (x.second > a) ctx->stage_ms[1] += x.second - a;
            end = std::max(end, x.second);
        }
    } else {
        for (int i = 0; i + 1 < ctx->kev_used; i += 2)
            if (cudaEventElapsedTime(&t, ctx->kev[i], ctx->kev[i + 1]) == cudaSuccess) ctx->stage_ms[1] += t;
    }
    cudaGetLastError();   // a failed elapsed-time query leaves no sticky error
    ctx->kev_used = 0;
    if (cudaEventElapsedTime(&t, ctx->ev[0], ctx->ev[1]) == cudaSuccess) ctx->stage_ms[0] += t;
    if (cudaEventElapsedTime(&t, ctx->ev[2], ctx->ev[3]) == cudaSuccess) ctx->stage_ms[2] += t;
    if (cudaEventElapsedTime(&t, ctx->ev[3], ctx->ev[4]) == cudaSuccess) ctx->stage_ms[3] += t;
}

gcf_status full_spectra(gcf_ctx* ctx, const std::vector<int>& mics,
                        const std::vector<gcf_result>& res, const std::vector<float>& pxn,
                        const gcf_optics& op, float* host_out)
{
    int T = ctx->tile, cx = T / 2 + 1, k = (int)mics.size();
    if (k == 0) return GCF_OK;
    int nm = 0;
    for (int m : mics) nm = std::max(nm, m + 1);
    CK(ctx->moments2.ensure(2 * (size_t)nm));
    launch_moments(ctx->ctf.p, cx * T, nm, ctx->moments2.p, ctx->st);
    CKL();
    std::vector<PixOptics> o(k);
    for (int i = 0; i < k; ++i) o[i] = make_optics(op, pxn[i]);
    CK(ctx->d_optics.ensure(k));
    CK(ctx->mic_of.ensure(k));
    CK(ctx->d_res.ensure(std::max<size_t>(k, ctx->d_res.n)));
    CK(ctx->full.ensure((size_t)k * T * T));
    CK(h2d(ctx, ctx->d_optics.p, o.data(), k * sizeof(PixOptics), ctx->st));
    CK(h2d(ctx, ctx->mic_of.p, mics.data(), k * sizeof(int), ctx->st));
    CK(h2d(ctx, ctx->d_res.p, res.data(), k * sizeof(gcf_result), ctx->st));
    launch_full_spectrum(ctx->ctf.p, T, k, ctx->mic_of.p, ctx->d_res.p, ctx->d_optics.p,
                         ctx->moments2.p, 0.0f, ctx->full.p, ctx->st);
    CKL();
    ctx->launches += 2;
    CK(cudaMemcpyAsync(host_out, ctx->full.p, (size_t)k * T * T * sizeof(float),
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GCF_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* gcf_strerror(gcf_status s)
{
    switch (s) {
    case GCF_OK: return "ok";
    case GCF_ERR_INVALID_ARG: return "invalid argument";
    case GCF_ERR_CUDA: return "CUDA error";
    case GCF_ERR_CUFFT: return "cuFFT error";
    case GCF_ERR_NO_MEMORY: return "out of memory";
    case GCF_ERR_IMAGE_TOO_SMALL: return "image smaller than one tile";
    case GCF_ERR_STATE: return "call out of order";
    case GCF_ERR_IO: return "file I/O error";
    case GCF_ERR_TIMEOUT: return "device wait timed out";
    }
    return "unknown status";
}

const char* gcf_last_error(gcf_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : "";
}

gcf_status gcf_create(int gpu, int tile_size, int log_spect, gcf_ctx** out)
{
    if (!out) return GCF_ERR_INVALID_ARG;
    *out = nullptr;
    if (tile_size < 16 || tile_size > 2048 || (tile_size & 1)) return GCF_ERR_INVALID_ARG;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return GCF_ERR_CUDA;
    if (gpu < 0 || gpu >= ndev) return GCF_ERR_INVALID_ARG;
    gcf_ctx* ctx = new gcf_ctx();
    ctx->dev = gpu;
    ctx->tile = tile_size;
    ctx->log_spect = log_spect ? 1 : 0;
    ctx->impl = fused_tile_supported(tile_size) ? GCF_SPECT_FUSED : GCF_SPECT_CUFFT;
    int prio_lo = 0, prio_hi = 0;
    if (cudaSetDevice(gpu) != cudaSuccess ||
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->st, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->st_search, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->st_tile, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->st_copy, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return GCF_ERR_CUDA;
    }
    for (auto& ev : ctx->ev) cudaEventCreate(&ev);
    gcf_status s = build_tile_tables(ctx);
    if (s != GCF_OK) {
        gcf_destroy(ctx);
        return s;
    }
    *out = ctx;
    return GCF_OK;
}

void gcf_destroy(gcf_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->dev);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    if (ctx->st_copy) cudaStreamSynchronize(ctx->st_copy);
    if (ctx->st_search) cudaStreamSynchronize(ctx->st_search);
    if (ctx->st_solo) cudaStreamSynchronize(ctx->st_solo);
    if (ctx->st_tile) cudaStreamSynchronize(ctx->st_tile);
    for (auto& kv : ctx->plans) cufftDestroy(kv.second.h);
    ctx->fft_work.release();
    for (auto* b : ctx->bands) {
        b->idx.release();
        b->a.release();
        b->d.release();
        b->env.release();
        b->c2t.release();
        b->s2t.release();
        delete b;
    }
    ctx->taper.release();
    ctx->rad_off.release();
    ctx->rad_pix.release();
    ctx->ring_off.release();
    ctx->ring_pix.release();
    ctx->ring_geo.release();
    ctx->d_bands.release();
    ctx->images.release();
    ctx->rescaled.release();
    ctx->tiles.release();
    ctx->cmp.release();
    ctx->rs_cmp.release();
    ctx->rs_crop.release();
    ctx->rs_src.release();
    ctx->rsg_bf.release();
    ctx->rsg_f.release();
    ctx->rsg_err.release();
    ctx->acc.release();
    ctx->hsum.release();
    ctx->lpfull.release();
    ctx->lpcmp.release();
    ctx->moments.release();
    ctx->moments2.release();
    ctx->raw.release();
    ctx->ctf0.release();
    ctx->ctf.release();
    ctx->radial.release();
    ctx->band_spec.release();
    ctx->cc_res.release();
    ctx->full.release();
    ctx->lowpassed.release();
    ctx->spec_off.release();
    ctx->mic_of.release();
    ctx->jobs.release();
    ctx->sum_ss.release();
    ctx->ring_sums.release();
    ctx->cand.release();
    ctx->cval.release();
    ctx->part.release();
    ctx->d_res.release();
    ctx->d_optics.release();
    ctx->d_counts.release();
    ctx->tw512.release();
    ctx->f_desc.release();
    ctx->f_items.release();
    ctx->f_first.release();
    ctx->f_inv.release();
    ctx->f_partial.release();
    ctx->f_next.release();
    ctx->solo_col.release();
    ctx->solo_acc.release();
    ctx->f_bsum.release();
    ctx->f_bsum_ptr.release();
    for (auto& ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : ctx->chunk_ev) cudaEventDestroy(ev);
    for (auto& ev : ctx->kev) cudaEventDestroy(ev);
    for (auto& ev : ctx->fev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    for (int k = 0; k < 2; ++k) {
        if (ctx->ingest_copied[k]) cudaEventDestroy(ctx->ingest_copied[k]);
        if (ctx->ingest_used[k]) cudaEventDestroy(ctx->ingest_used[k]);
    }
    if (ctx->ingest_pin) cudaFreeHost(ctx->ingest_pin);
    ctx->loaded.release();
    ctx->ingest_raw.release();
    if (ctx->bgraph.exec) cudaGraphExecDestroy(ctx->bgraph.exec);
    ctx->bgraph.arena.release();
    ctx->arena.release();
    if (ctx->nn) nn_destroy(ctx->nn);
    ctx->nx1.release();
    ctx->nx2.release();
    ctx->npx.release();
    ctx->nparams.release();
    ctx->ntarget.release();
    ctx->nloss.release();
    ctx->cA.release();
    ctx->cA2.release();
    ctx->cB.release();
    ctx->cE.release();
    ctx->cP.release();
    ctx->cDz.release();
    ctx->cSS.release();
    ctx->cRows.release();
    ctx->cTiles.release();
    ctx->cNtiles.release();
    ctx->cErr.release();
    ctx->cPrior.release();
    if (ctx->st_copy) cudaStreamDestroy(ctx->st_copy);
    if (ctx->st_search) cudaStreamDestroy(ctx->st_search);
    if (ctx->st_solo) cudaStreamDestroy(ctx->st_solo);
    if (ctx->solo_fork) cudaEventDestroy(ctx->solo_fork);
    if (ctx->solo_join) cudaEventDestroy(ctx->solo_join);
    if (ctx->st_tile) cudaStreamDestroy(ctx->st_tile);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
}

gcf_status gcf_set_rescale_impl(gcf_ctx* ctx, int impl)
{
    if (!ctx || (impl != GCF_RESCALE_LINES && impl != GCF_RESCALE_CUFFT && impl != GCF_RESCALE_GEMM))
        return GCF_ERR_INVALID_ARG;
    ctx->rescale_impl = impl;
    return GCF_OK;
}

gcf_status gcf_set_spectrum_impl(gcf_ctx* ctx, int impl)
{
    if (!ctx) return GCF_ERR_INVALID_ARG;
    if (impl == GCF_SPECT_CUFFT) {
        ctx->impl = impl;
        return GCF_OK;
    }
    if (impl == GCF_SPECT_FUSED && fused_tile_supported(ctx->tile)) {
        ctx->impl = impl;
        return GCF_OK;
    }
    return fail(ctx, GCF_ERR_INVALID_ARG, "spectrum implementation not available for this tile size");
}

void gcf_rescale_dims(int w, int h, float px, int* nw, int* nh, float* npx)
{
    // CRescaleImage::Setup (FindCTF/CRescaleImage.cpp:47-66)
    float bin = 1.2f / px;
    if (bin <= 1) bin = 1.0f;
    float pxn = px * bin;
    int a = (int)(w / bin + 0.5f), b = (int)(h / bin + 0.5f);
    a = a / 2 * 2;
    b = b / 2 * 2;
    if (nw) *nw = a;
    if (nh) *nh = b;
    if (npx) *npx = pxn;
}

gcf_status gcf_rescale(gcf_ctx* ctx, const float* img, int w, int h, float px, int on_device,
                       float* host_out)
{
    if (!ctx || !img || !host_out || w <= 0 || h <= 0 || !(px > 0)) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    const float* d = img;
    if (!on_device) {
        CK(ctx->images.ensure((size_t)w * h));
        CK(cudaMemcpyAsync(ctx->images.p, img, (size_t)w * h * sizeof(float),
                           cudaMemcpyHostToDevice, ctx->st));
        d = ctx->images.p;
    }
    int nw, nh;
    float pxn;
    bool copied;
    gcf_rescale_dims(w, h, px, &nw, &nh, &pxn);
    CK(ctx->rescaled.ensure((size_t)nw * nh));
    CKS(rescale_device(ctx, d, w, h, px, ctx->rescaled.p, &nw, &nh, &pxn, &copied));
    if (copied) {
        CK(cudaMemcpyAsync(host_out, ctx->rescaled.p, (size_t)nw * nh * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->st));
    } else {
        CK(cudaMemcpy2DAsync(host_out, nw * sizeof(float), d, w * sizeof(float),
                             nw * sizeof(float), nh, cudaMemcpyDeviceToHost, ctx->st));
    }
    int rs_err = 0;
    if (ctx->rsg_err.p)
        CK(cudaMemcpyAsync(&rs_err, ctx->rsg_err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return check_rescale_gemm(ctx, rs_err);
}

gcf_status gcf_set_fused_shape(gcf_ctx* ctx, int shape)
{
    if (!ctx || (shape != 0 && shape != 8 && shape != 816 && shape != 16 && shape != 162 && shape != 168))
        return GCF_ERR_INVALID_ARG;
    ctx->fused_shape_req = shape;
    ctx->fused_clusters = 0;   // recomputed at the next launch
    ctx->solo_n = -1;
    return GCF_OK;
}

gcf_status gcf_setup(gcf_ctx* ctx, const gcf_optics* optics, int width, int height)
{
    if (!ctx || !valid_optics(optics) || width <= 0 || height <= 0) return GCF_ERR_INVALID_ARG;
    ctx->optics = *optics;
    ctx->img_w = width;
    ctx->img_h = height;
    ctx->have_setup = true;
    ctx->have_spectrum = false;
    ctx->phase_deg = 0.0f;
    ctx->phase_range = 0.0f;
    ctx->held_phase = 0.0f;   // Setup1 creates a new CFindDefocus2D
    return GCF_OK;
}

gcf_status gcf_gen_half_spectrum(gcf_ctx* ctx, const float* img, int pitch, int on_device)
{
    if (!ctx || !img || pitch < ctx->img_w) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_setup) return fail(ctx, GCF_ERR_STATE, "gcf_setup first");
    CKS(set_device(ctx));
    const float* d = img;
    if (!on_device) {
        CK(ctx->images.ensure((size_t)pitch * ctx->img_h));
        CK(cudaMemcpyAsync(ctx->images.p, img, (size_t)pitch * ctx->img_h * sizeof(float),
                           cudaMemcpyHostToDevice, ctx->st));
        d = ctx->images.p;
    }
    Layout L = tile_layout(ctx->img_w, ctx->img_h, ctx->tile);
    if (L.ntx <= 0 || L.nty <= 0 || ctx->img_w < ctx->tile || ctx->img_h < ctx->tile)
        return fail(ctx, GCF_ERR_IMAGE_TOO_SMALL, "image holds no full tile");
    std::vector<MicImage> mics(1);
    mics[0] = MicImage{d, ctx->img_w, ctx->img_h, pitch, ctx->optics.pixel_size};
    CKS(spectra(ctx, mics));
    int lp = 0;
    CK(cudaMemcpyAsync(&lp, ctx->lowpassed.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->cur_lowpassed = lp;
    ctx->have_spectrum = true;
    return GCF_OK;
}

gcf_status gcf_set_phase(gcf_ctx* ctx, float phase_deg, float range_deg)
{
    if (!ctx) return GCF_ERR_INVALID_ARG;
    ctx->phase_deg = phase_deg;
    ctx->phase_range = range_deg;
    return GCF_OK;
}

gcf_status gcf_do2d(gcf_ctx* ctx, gcf_result* out)
{
    if (!ctx || !out) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_spectrum) return fail(ctx, GCF_ERR_STATE, "no spectrum: call gcf_gen_half_spectrum");
    CKS(set_device(ctx));
    JobSpec s;
    std::memset(&s, 0, sizeof(s));
    s.mic = 0;
    s.mode = 0;
    s.optics = ctx->optics;
    s.px_n = ctx->optics.pixel_size;
    s.phase_deg = ctx->phase_deg;
    s.phase_range = ctx->phase_range;
    s.held_phase = ctx->held_phase;
    std::vector<gcf_result> r;
    CKS(run_search(ctx, {s}, r));
    *out = r[0];
    ctx->held_phase = r[0].ext_phase;
    ctx->phase_deg = r[0].ext_phase;   // CFindCtf2D::mGetResults sets m_fExtPhase
    return GCF_OK;
}

// CFindCtf1D::Do1D / Refine1D (FindCTF/CFindCtf1D.cpp:49-67): the radial
// average of the current spectrum, then the brute-force defocus (x phase)
// searches; m_fExtPhase takes the found phase.
static gcf_status run_1d(gcf_ctx* ctx, int mode, float init_df, float df_range, gcf_result* out)
{
    if (!ctx || !out) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_spectrum) return fail(ctx, GCF_ERR_STATE, "no spectrum: call gcf_gen_half_spectrum");
    CKS(set_device(ctx));
    JobSpec s;
    std::memset(&s, 0, sizeof(s));
    s.mic = 0;
    s.mode = mode;
    s.optics = ctx->optics;
    s.px_n = ctx->optics.pixel_size;
    s.phase_deg = ctx->phase_deg;
    s.phase_range = ctx->phase_range;
    s.r1d_df = init_df;
    s.r1d_range = df_range;
    std::vector<gcf_result> r;
    CKS(run_search(ctx, {s}, r));
    *out = r[0];
    ctx->phase_deg = r[0].ext_phase;
    return GCF_OK;
}

gcf_status gcf_do1d(gcf_ctx* ctx, gcf_result* out) { return run_1d(ctx, 2, 0.0f, 0.0f, out); }

gcf_status gcf_refine1d(gcf_ctx* ctx, float init_df, float df_range, gcf_result* out)
{
    if (!(df_range >= 0.0f) || !(init_df > 0.0f)) return GCF_ERR_INVALID_ARG;
    return run_1d(ctx, 3, init_df, df_range, out);
}

gcf_status gcf_refine(gcf_ctx* ctx, const float df[2], const float ast[2], const float ang[2],
                      const float ph[2], gcf_result* out)
{
    if (!ctx || !df || !ast || !ang || !ph || !out) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_spectrum) return fail(ctx, GCF_ERR_STATE, "no spectrum: call gcf_gen_half_spectrum");
    CKS(set_device(ctx));
    JobSpec s;
    std::memset(&s, 0, sizeof(s));
    s.mic = 0;
    s.mode = 1;
    s.optics = ctx->optics;
    s.px_n = ctx->optics.pixel_size;
    float rin[8] = {df[0], df[1], ast[0], ast[1], ang[0], ang[1], ph[0], ph[1]};
    std::memcpy(s.rin, rin, sizeof(rin));
    s.held_phase = ctx->held_phase;
    std::vector<gcf_result> r;
    CKS(run_search(ctx, {s}, r));
    *out = r[0];
    ctx->held_phase = r[0].ext_phase;
    ctx->phase_deg = r[0].ext_phase;
    return GCF_OK;
}

// ---------------------------------------------------------------------------
// GBackground1D (FindCTF/GBackground1D.cu:61-169)
// ---------------------------------------------------------------------------
gcf_status gcf_background1d(gcf_ctx* ctx, const float* spectrum, int n, int on_device,
                            float* background, int* start)
{
    if (!ctx || !spectrum || !background || !start || n <= 0 || n > kMaxBackgroundBins)
        return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    const float* d_in = spectrum;
    float* d_out = background;
    if (!on_device) {
        CK(ctx->bg_spec.ensure(n));
        CK(ctx->bg_curve.ensure(n));
        CK(h2d(ctx, ctx->bg_spec.p, spectrum, n * sizeof(float), ctx->st));
        d_in = ctx->bg_spec.p;
        d_out = ctx->bg_curve.p;
    }
    CK(ctx->bg_start.ensure(1));
    CK(launch_background1d(d_in, n, d_out, ctx->bg_start.p, ctx->st));
    ctx->launches += 1;
    if (!on_device)
        CK(cudaMemcpyAsync(background, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(start, ctx->bg_start.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GCF_OK;
}

static gcf_status remove_bg(gcf_ctx* ctx, float* spec, size_t spec_n, int n_or_tile, bool two_d,
                            const float* bg, int bg_n, int start, int on_device)
{
    if (!ctx || !spec || !bg || n_or_tile <= 0 || bg_n <= 0) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    float* d_spec = spec;
    const float* d_bg = bg;
    if (!on_device) {
        CK(ctx->bg_spec.ensure(spec_n));
        CK(ctx->bg_curve.ensure(bg_n));
        CK(h2d(ctx, ctx->bg_spec.p, spec, spec_n * sizeof(float), ctx->st));
        CK(h2d(ctx, ctx->bg_curve.p, bg, bg_n * sizeof(float), ctx->st));
        d_spec = ctx->bg_spec.p;
        d_bg = ctx->bg_curve.p;
    }
    if (two_d) CK(launch_remove_background2d(d_spec, n_or_tile, d_bg, bg_n, start, ctx->st));
    else CK(launch_remove_background1d(d_spec, n_or_tile, d_bg, bg_n, start, ctx->st));
    ctx->launches += 1;
    if (!on_device)
        CK(cudaMemcpyAsync(spec, d_spec, spec_n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GCF_OK;
}

gcf_status gcf_remove_background1d(gcf_ctx* ctx, float* spectrum, int n, const float* background,
                                   int bg_n, int start, int on_device)
{
    return remove_bg(ctx, spectrum, (size_t)std::max(n, 0), n, false, background, bg_n, start, on_device);
}

gcf_status gcf_remove_background2d(gcf_ctx* ctx, float* half_spectrum, int tile,
                                   const float* background, int bg_n, int start, int on_device)
{
    if (tile <= 0 || tile % 2) return GCF_ERR_INVALID_ARG;
    return remove_bg(ctx, half_spectrum, (size_t)(tile / 2 + 1) * tile, tile, true, background, bg_n,
                     start, on_device);
}

gcf_status gcf_get_spect_size(gcf_ctx* ctx, int size[2], int half)
{
    if (!ctx || !size) return GCF_ERR_INVALID_ARG;
    size[0] = ctx->tile / 2 + 1;
    size[1] = ctx->tile;
    if (!half) size[0] = (size[0] - 1) * 2;
    return GCF_OK;
}

gcf_status gcf_get_half_spectrum(gcf_ctx* ctx, int raw, float* host_out)
{
    if (!ctx || !host_out) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_spectrum) return fail(ctx, GCF_ERR_STATE, "no spectrum");
    CKS(set_device(ctx));
    size_t n = (size_t)(ctx->tile / 2 + 1) * ctx->tile;
    CK(cudaMemcpyAsync(host_out, raw ? ctx->raw.p : ctx->ctf.p, n * sizeof(float),
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GCF_OK;
}

gcf_status gcf_get_radial_average(gcf_ctx* ctx, float* host_out)
{
    if (!ctx || !host_out) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_spectrum) return fail(ctx, GCF_ERR_STATE, "no spectrum");
    CKS(set_device(ctx));
    CK(cudaMemcpyAsync(host_out, ctx->radial.p, (ctx->tile / 2 + 1) * sizeof(float),
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GCF_OK;
}

gcf_status gcf_gen_full_spectrum(gcf_ctx* ctx, const gcf_result* res, float* host_out)
{
    if (!ctx || !res || !host_out) return GCF_ERR_INVALID_ARG;
    if (!ctx->have_spectrum) return fail(ctx, GCF_ERR_STATE, "no spectrum");
    CKS(set_device(ctx));
    return full_spectra(ctx, {0}, {*res}, {ctx->optics.pixel_size}, ctx->optics, host_out);
}

namespace {

// The CFindSeriesCtfs package loop (CFindSeriesCtfs.cpp:50-213) over slots
// in processing order: slot 0 gets the full search, every later slot is
// refined around the best-scoring earlier one, a refine with score <= 0
// falls back to the full search.  Refines are issued speculatively as one
// batch over a range of slots around the current best; when the best
// changes, the rest of the range is re-run around the new one, so the
// results equal the sequential loop.
struct SeriesLoop {
    gcf_ctx* ctx;
    gcf_optics op;
    float pxn;
    int is_tomo;
    std::vector<gcf_result> res;
    std::vector<int> ref_used;   // slot whose result seeded this slot's refine
    int cur_ref = -1;
    const int* image_of = nullptr;   // slot -> caller's image index
    int done = 0;

    // Slot k's result is final: report it to the caller's hook.
    void finalize(int k)
    {
        done = k + 1;
        if (ctx->pkg_fn) ctx->pkg_fn(ctx->pkg_user, done, image_of ? image_of[k] : k, &res[k]);
    }

    JobSpec full_job(int slot) const
    {
        JobSpec s;
        std::memset(&s, 0, sizeof(s));
        s.mic = slot;
        s.mode = 0;
        s.optics = op;
        s.px_n = pxn;
        // mProcessFull: SetPhase(extPhase[0], max(extPhase[1], 0)) (CFindSeriesCtfs.cpp:154-157)
        s.phase_deg = op.ext_phase_deg;
        s.phase_range = fmaxf(op.ext_phase_range, 0.0f);
        return s;
    }

    JobSpec refine_job(int slot, const gcf_result& rp) const
    {
        // CFindSeriesCtfs::mProcessRefine (CFindSeriesCtfs.cpp:168-199)
        JobSpec s;
        std::memset(&s, 0, sizeof(s));
        s.mic = slot;
        s.mode = 1;
        s.optics = op;
        s.px_n = pxn;
        float dmin = rp.df_min, dmax = rp.df_max;
        float dfr = 5000.0f * op.pixel_size * op.pixel_size;
        s.rin[0] = 0.5f * (dmin + dmax);
        s.rin[1] = fmaxf(s.rin[0] * 0.5f, dfr);
        float diff = (dmax - dmin) * 0.5f, mean = (dmax + dmin) * 0.5f;
        s.rin[2] = mean <= 0.0f ? 0.0f : (diff / mean);
        s.rin[4] = rp.azimuth;
        s.rin[6] = rp.ext_phase;
        if (!is_tomo) {
            s.rin[3] = 0.04f;
            s.rin[5] = 30.0f;
            if (op.ext_phase_range > 0) s.rin[7] = 40.0f;
        }
        return s;
    }

    // Packages k0 .. k1-1, whose spectra are ready.
    gcf_status run(int k0, int k1)
    {
        std::vector<gcf_result> r;
        int k = k0;
        if (k == 0 && k < k1) {
            CKS(run_search(ctx, {full_job(0)}, r));
            res[0] = r[0];
            cur_ref = 0;
            finalize(0);
            ++k;
        }
        bool batch_valid = false;
        while (k < k1) {
            if (!batch_valid) {
                std::vector<JobSpec> js;
                for (int q = k; q < k1; ++q) js.push_back(refine_job(q, res[cur_ref]));
                CKS(run_search(ctx, js, r));
                for (int q = k; q < k1; ++q) {
                    res[q] = r[q - k];
                    ref_used[q] = cur_ref;
                }
                batch_valid = true;
            }
            if (ref_used[k] != cur_ref) {
                batch_valid = false;
                continue;
            }
            // mProcessPackage / mProcessRefine ref update (CFindSeriesCtfs.cpp:133-146, :200-203)
            int new_ref = cur_ref;
            if (res[cur_ref].score < res[k].score) new_ref = k;
            if (res[k].score <= 0) {
                // same CFindCtf2D object as the refine: its search starts at
                // the phase the refine ended with
                JobSpec fj = full_job(k);
                fj.held_phase = res[k].ext_phase;
                CKS(run_search(ctx, {fj}, r));
                res[k] = r[0];
                new_ref = k;
            }
            if (new_ref != cur_ref) {
                cur_ref = new_ref;
                batch_valid = false;
            }
            finalize(k);
            ++k;
        }
        return GCF_OK;
    }
};

// Chunk bounds of a series of n packages in processing order: the first
// package alone (its full search starts early), then 8 packages, shrinking
// towards the end so that little work follows the last chunk.
std::vector<int> series_chunks(int n)
{
    std::vector<int> bounds{0};
    for (int b = 1; b < n;) {
        bounds.push_back(b);
        int rem = n - b;
        b += rem > 12 ? 8 : rem > 6 ? 4 : rem > 2 ? 2 : 1;
    }
    bounds.push_back(n);
    return bounds;
}

// Host images: uploads in processing order on the copy stream (the first
// package alone, then chunks of 8 shrinking towards the end); each chunk's
// spectra on the high-priority stream as soon as it lands, and its
// post-processing and package searches on the low-priority search stream
// once its spectra are done, so only the last chunk's work follows the last
// copy.
gcf_status series_streamed(gcf_ctx* ctx, const std::vector<const float*>& imgs, int w, int h,
                           float px, std::vector<MicImage>& mics, SeriesLoop& loop)
{
    const int n = (int)imgs.size();
    mics.assign(n, MicImage{});
    int nw, nh;
    float pn;
    gcf_rescale_dims(w, h, px, &nw, &nh, &pn);
    const bool rescaled = (1.2f / px) > 1;
    CKS(spectra_alloc(ctx, n));
    if (rescaled) CK(ctx->rescaled.ensure((size_t)nw * nh * n));
    CK(ctx->images.ensure((size_t)w * h * n));
    std::vector<int> bounds = series_chunks(n);
    const int nchunks = (int)bounds.size() - 1;
    // chunk_ev: [0, nchunks) copies done, [nchunks, 2 nchunks) spectra done,
    // [2 nchunks] searches done
    while ((int)ctx->chunk_ev.size() < 2 * nchunks + 1) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->chunk_ev.push_back(e);
    }
    CK(record_timing(ctx->ev[0], ctx->st));
    CK(cudaStreamWaitEvent(ctx->st_copy, ctx->ev[0], 0));
    const size_t cnt = (size_t)w * h;
    for (int c = 0; c < nchunks; ++c) {
        for (int k = bounds[c]; k < bounds[c + 1]; ++k)
            CK(cudaMemcpyAsync(ctx->images.p + cnt * k, imgs[k], cnt * sizeof(float), cudaMemcpyHostToDevice,
                               ctx->st_copy));
        CK(cudaEventRecord(ctx->chunk_ev[c], ctx->st_copy));
    }
    CK(record_timing(ctx->ev[1], ctx->st_copy));
    CK(record_timing(ctx->ev[2], ctx->st));
    // every chunk's spectra on st as its copy lands ...
    for (int c = 0; c < nchunks; ++c) {
        const int k0 = bounds[c], k1 = bounds[c + 1];
        CK(cudaStreamWaitEvent(ctx->st, ctx->chunk_ev[c], 0));
        for (int k = k0; k < k1; ++k) {
            size_t used = 0;
            float* dst = rescaled ? ctx->rescaled.p + (size_t)nw * nh * k : nullptr;
            CKS(stage_image(ctx, ctx->images.p + cnt * k, w, h, px, dst, mics[k], &used));
        }
        CKS(spectra_chunk(ctx, mics, k0, k1 - k0));
        CK(cudaEventRecord(ctx->chunk_ev[nchunks + c], ctx->st));
    }
    CK(record_timing(ctx->ev[3], ctx->st));
    CK(record_timing(ctx->ev[4], ctx->st));
    // ... and its post-processing and package searches on the low-priority
    // search stream once they are done, so that no chunk's spectra wait for
    // the searches of the chunks before it
    auto search_phase = [&]() -> gcf_status {
        for (int c = 0; c < nchunks; ++c) {
            const int k0 = bounds[c], k1 = bounds[c + 1];
            CK(cudaStreamWaitEvent(ctx->st, ctx->chunk_ev[nchunks + c], 0));
            CKS(spectra_post(ctx, k1 - k0, k0));
            CKS(loop.run(k0, k1));
        }
        return GCF_OK;
    };
    std::swap(ctx->st, ctx->st_search);
    gcf_status st = search_phase();
    cudaError_t e = cudaEventRecord(ctx->chunk_ev[2 * nchunks], ctx->st);
    std::swap(ctx->st, ctx->st_search);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->st, ctx->chunk_ev[2 * nchunks], 0);
    if (st == GCF_OK && e != cudaSuccess) st = fail(ctx, GCF_ERR_CUDA, cudaGetErrorString(e));
    return st;
}

// Device images: the first package alone, then all others.  With fused
// spectra both tile launches are enqueued at once (one plan, one upload of
// the work items) on the two high-priority streams, so the second launch's
// clusters start while the first package's items finish, and each launch
// brings its cluster-less CTAs onto the SMs the clusters leave free.  The
// post-processing and searches of each chunk run on the low-priority search
// stream when its spectra are done: the first package's full search mostly
// in the last part of the big launch, when its cluster-less CTAs have
// stopped, and the other packages' refinements as one batch at the end.
// (Measured alternatives, all slower on a 41-tilt series: the other packages
// in two launches with their searches in between; one launch for all; the
// first package's search started before the big launch's cluster-less CTAs;
// fewer cluster-less CTAs to leave SMs to that search.)
gcf_status series_overlapped(gcf_ctx* ctx, const std::vector<const float*>& imgs, int w, int h,
                             float px, std::vector<MicImage>& mics, SeriesLoop& loop)
{
    const int n = (int)imgs.size();
    const int T = ctx->tile;
    const size_t cmp_n = (size_t)(T / 2 + 1) * T;
    mics.assign(n, MicImage{});
    int nw, nh;
    float pn;
    gcf_rescale_dims(w, h, px, &nw, &nh, &pn);
    const bool rescaled = (1.2f / px) > 1;
    CKS(spectra_alloc(ctx, n));
    if (rescaled) CK(ctx->rescaled.ensure((size_t)nw * nh * n));
    const bool fused = ctx->impl == GCF_SPECT_FUSED;
    std::vector<int> bounds{0, 1};
    if (n > 1) bounds.push_back(n);
    const int nchunks = (int)bounds.size() - 1;
    while ((int)ctx->chunk_ev.size() < nchunks + 2) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->chunk_ev.push_back(e);
    }
    CK(record_timing(ctx->ev[0], ctx->st));
    CK(record_timing(ctx->ev[1], ctx->st));
    CK(record_timing(ctx->ev[2], ctx->st));
    for (int k = 0; k < n; ++k) {
        size_t used = 0;
        float* dst = rescaled ? ctx->rescaled.p + (size_t)nw * nh * k : nullptr;
        CKS(stage_image(ctx, imgs[k], w, h, px, dst, mics[k], &used));
    }
    if (fused) {
        CKS(fused_plan(ctx, mics));
        cudaEvent_t planned = ctx->chunk_ev[nchunks + 1];
        CK(cudaEventRecord(planned, ctx->st));
        CK(cudaStreamWaitEvent(ctx->st_tile, planned, 0));
        for (int c = 0; c < nchunks; ++c) {
            cudaStream_t s = (c & 1) ? ctx->st_tile : ctx->st;
            CKS(fused_launch(ctx, bounds[c], bounds[c + 1], ctx->raw.p + cmp_n * bounds[c], s));
            CK(cudaEventRecord(ctx->chunk_ev[c], s));
        }
        // st joins st_tile (its last chunk) before anything else runs on it
        CK(cudaEventRecord(planned, ctx->st_tile));
        CK(cudaStreamWaitEvent(ctx->st, planned, 0));
    } else {
        for (int c = 0; c < nchunks; ++c) {
            CKS(spectra_chunk(ctx, mics, bounds[c], bounds[c + 1] - bounds[c]));
            CK(cudaEventRecord(ctx->chunk_ev[c], ctx->st));
        }
    }
    CK(record_timing(ctx->ev[3], ctx->st));
    CK(record_timing(ctx->ev[4], ctx->st));
    auto search_phase = [&]() -> gcf_status {
        for (int c = 0; c < nchunks; ++c) {
            CK(cudaStreamWaitEvent(ctx->st, ctx->chunk_ev[c], 0));
            CKS(spectra_post(ctx, bounds[c + 1] - bounds[c], bounds[c]));
            CKS(loop.run(bounds[c], bounds[c + 1]));
        }
        return GCF_OK;
    };
    std::swap(ctx->st, ctx->st_search);
    gcf_status st = search_phase();
    cudaError_t e = cudaEventRecord(ctx->chunk_ev[nchunks], ctx->st);
    std::swap(ctx->st, ctx->st_search);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->st, ctx->chunk_ev[nchunks], 0);
    if (st == GCF_OK && e != cudaSuccess) st = fail(ctx, GCF_ERR_CUDA, cudaGetErrorString(e));
    return st;
}

}  // namespace

gcf_status gcf_run_series(gcf_ctx* ctx, const float* const* images, int n, int w, int h,
                          int on_device, const gcf_optics* optics, const int* order, int is_tomo,
                          gcf_result* results, float* full_out)
{
    if (!ctx || !images || n <= 0 || w <= 0 || h <= 0 || !valid_optics(optics) || !order ||
        !results)
        return GCF_ERR_INVALID_ARG;
    std::vector<int> seen(n, 0), pos(n);
    for (int k = 0; k < n; ++k) {
        if (order[k] < 0 || order[k] >= n || seen[order[k]]) return GCF_ERR_INVALID_ARG;
        seen[order[k]] = 1;
        pos[order[k]] = k;
    }
    for (int i = 0; i < n; ++i)
        if (!images[i]) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    for (float& t : ctx->stage_ms) t = 0.0f;
    for (long long& c : ctx->search_counts) c = 0;
    ctx->kev_used = 0;
    ctx->launches = 0;
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, ctx->st));
    // slot k holds package k of the processing order (image order[k])
    std::vector<const float*> imgs(n);
    for (int k = 0; k < n; ++k) imgs[k] = images[order[k]];
    int nw, nh;
    float pxn;
    gcf_rescale_dims(w, h, optics->pixel_size, &nw, &nh, &pxn);
    SeriesLoop loop{ctx, *optics, pxn, is_tomo, std::vector<gcf_result>(n), std::vector<int>(n, -1)};
    loop.image_of = order;
    std::vector<MicImage> mics;
    gcf_status st;
    if (on_device) {
        st = series_overlapped(ctx, imgs, w, h, optics->pixel_size, mics, loop);
    } else {
        st = series_streamed(ctx, imgs, w, h, optics->pixel_size, mics, loop);
    }
    if (st == GCF_OK && full_out) {
        std::vector<int> mi(n);
        std::vector<gcf_result> ri(n);
        std::vector<float> pv(n, pxn);
        for (int i = 0; i < n; ++i) {
            mi[i] = pos[i];
            ri[i] = loop.res[pos[i]];
        }
        st = full_spectra(ctx, mi, ri, pv, *optics, full_out);
    }
    if (st == GCF_OK)
        for (int i = 0; i < n; ++i) results[i] = loop.res[pos[i]];
    cudaEventRecord(t1, ctx->st);
    cudaEventSynchronize(t1);
    accumulate_stage_times(ctx);
    float tt = 0;
    cudaEventElapsedTime(&tt, t0, t1);
    ctx->stage_ms[6] = tt;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return st;
}

gcf_status gcf_set_package_callback(gcf_ctx* ctx, gcf_package_fn fn, void* user)
{
    if (!ctx) return GCF_ERR_INVALID_ARG;
    ctx->pkg_fn = fn;
    ctx->pkg_user = fn ? user : nullptr;
    return GCF_OK;
}

}  // extern "C"

namespace {

// FNV-1a over everything the device work of a batch call depends on.
struct KeyHash {
    unsigned long long h = 1469598103934665603ull;
    void add(const void* p, size_t n)
    {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    }
    template <class T>
    void v(const T& x)
    {
        add(&x, sizeof(T));
    }
};

unsigned long long batch_key(const gcf_ctx* ctx, const gcf_item* items, int n, int on_device,
                             const gcf_optics& op, int mode)
{
    KeyHash k;
    k.v(mode);
    k.v(n);
    k.v(on_device);
    k.add(items, (size_t)n * sizeof(gcf_item));
    k.v(op);
    k.v(ctx->tile);
    k.v(ctx->impl);
    k.v(ctx->rescale_impl);
    k.v(ctx->log_spect);
    k.v(ctx->fused_shape);
    k.v(ctx->fused_clusters);
    k.v(ctx->gemm_bn);
    k.v(ctx->gemm_stages);
    k.v(ctx->gemm_persistent);
    k.v(ctx->contract_dz);
    k.v(ctx->contract_ns);
    k.v(ctx->contract_nth);
    k.v(ctx->nn_version);
    return k.h;
}

// Host inputs take a graph only from page-locked memory (a graph's copy
// nodes read the same host addresses again on every replay).
bool all_pinned(const float* const* imgs, int n)
{
    for (int i = 0; i < n; ++i) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, imgs[i]) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

// Device work of a batch call: uploads (host inputs), rescale, spectra,
// post-processing, searches enqueued; nothing read back.
gcf_status batch_enqueue(gcf_ctx* ctx, const std::vector<const float*>& imgs, const std::vector<int>& ws,
                         const std::vector<int>& hs, const std::vector<float>& pxs, int on_device,
                         const gcf_optics& op, int mode, SearchPending& pend, std::vector<float>& pxn)
{
    const int n = (int)imgs.size();
    std::vector<MicImage> mics;
    CKS(prepare_images(ctx, imgs.data(), ws.data(), hs.data(), pxs.data(), n, on_device, mics));
    pxn.resize(n);
    for (int i = 0; i < n; ++i) pxn[i] = mics[i].px_n;
    return search_enqueue(ctx, pxn, mode == GCF_SEARCH_PLAIN ? pxs.data() : nullptr, op, mode, pend);
}

// Captures batch_enqueue into ctx->bgraph (the graph then owns the arena
// its upload nodes read).  false: the capture did not produce a graph that
// may be replayed (the caller runs the call eagerly).
bool batch_capture(gcf_ctx* ctx, unsigned long long key, const std::vector<const float*>& imgs,
                   const std::vector<int>& ws, const std::vector<int>& hs, const std::vector<float>& pxs,
                   int on_device, const gcf_optics& op, int mode)
{
    BatchGraph& G = ctx->bgraph;
    // the graph's arena holds all of the call's uploads in one block, sized
    // from the eager call before (with room to spare)
    if (!G.arena.reserve(2 * ctx->arena.used_bytes() + ((size_t)1 << 20))) {
        ctx->graph_fail = 1;
        return false;
    }
    G.arena.reset();
    G.arena.frozen = true;
    std::swap(ctx->arena, G.arena);   // this capture's uploads go to the graph's arena
    const unsigned long long ep0 = device_alloc_epoch();
    const unsigned long long mv0 = ctx->model_version;
    ctx->kev_used = 0;   // only this attempt's timing events and launches count
    ctx->launches = 0;
    const long long launches0 = 0;
    SearchPending pend;
    std::vector<float> pxn;
    cudaGraph_t g = nullptr;
    gcf_status st = GCF_ERR_CUDA;
    ctx->graph_fail = 2;
    cudaError_t ce = cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeRelaxed);
    if (ce == cudaSuccess) {
        ctx->capturing = true;
        t_capturing = true;
        st = batch_enqueue(ctx, imgs, ws, hs, pxs, on_device, op, mode, pend, pxn);
        ctx->capturing = false;
        t_capturing = false;
        ce = cudaStreamEndCapture(ctx->st, &g);
        if (ce != cudaSuccess) g = nullptr;
        ctx->graph_fail = st != GCF_OK ? 3 : (!g ? 4 : 0);
    }
    if (ctx->graph_fail && ce != cudaSuccess) ctx->err = std::string("graph capture: ") + cudaGetErrorString(ce);
    std::swap(ctx->arena, G.arena);
    G.arena.frozen = false;
    cudaGetLastError();
    bool ok = st == GCF_OK && g && device_alloc_epoch() == ep0;
    if (!ctx->graph_fail && !ok) ctx->graph_fail = 5;
    if (ok) {
        cudaGraphExecUpdateResultInfo info;
        if (!(G.exec && cudaGraphExecUpdate(G.exec, g, &info) == cudaSuccess)) {
            cudaGetLastError();
            if (G.exec) cudaGraphExecDestroy(G.exec);
            G.exec = nullptr;
            ce = cudaGraphInstantiate(&G.exec, g, 0);
            ok = ce == cudaSuccess;
            if (!ok) {
                ctx->graph_fail = 6;
                ctx->err = std::string("graph instantiate: ") + cudaGetErrorString(ce);
            }
        }
    }
    if (ok) {
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        G.nodes = (int)nn;
        G.key = key;
        G.epoch = ep0;
        G.model_version = mv0 == ctx->model_version ? mv0 : ctx->model_version;
        G.kev_used = ctx->kev_used;
        G.launches = ctx->launches - launches0;
        G.pxn = pxn;
        G.band = pend.band;
        G.nj = pend.nj;
    } else {
        cudaGetLastError();
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
        G.key = 0;
    }
    if (g) cudaGraphDestroy(g);
    return ok;
}

// gcf_run_batch / gcf_run_batch_mode.  With CUDA graphs on, a call whose
// key repeats an earlier call's is captured once and then replayed as one
// graph launch.
gcf_status batch_run(gcf_ctx* ctx, const gcf_item* items, int n, int on_device, const gcf_optics* optics, int mode,
                     gcf_result* results)
{
    std::vector<const float*> imgs(n);
    std::vector<int> ws(n), hs(n);
    std::vector<float> pxs(n);
    for (int i = 0; i < n; ++i) {
        if (!items[i].image || items[i].width <= 0 || items[i].height <= 0 || !(items[i].pixel_size > 0))
            return GCF_ERR_INVALID_ARG;
        imgs[i] = items[i].image;
        ws[i] = items[i].width;
        hs[i] = items[i].height;
        pxs[i] = items[i].pixel_size;
    }
    CKS(set_device(ctx));
    for (float& t : ctx->stage_ms) t = 0.0f;
    for (long long& c : ctx->search_counts) c = 0;
    for (long long& c : ctx->fast_counts) c = 0;
    for (float& t : ctx->fast_ms) t = 0.0f;
    ctx->kev_used = 0;
    ctx->launches = 0;
    ctx->graph_launches = 0;
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, ctx->st));
    BatchGraph& G = ctx->bgraph;
    const bool graphable = ctx->graphs && (on_device || all_pinned(imgs.data(), n));
    if (graphable && ctx->impl == GCF_SPECT_FUSED && fused_tile_supported(ctx->tile)) {
        gcf_status fs = ensure_fused_shape(ctx);   // part of the key
        if (fs != GCF_OK) {
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
            return fs;
        }
    }
    const unsigned long long key = graphable ? batch_key(ctx, items, n, on_device, *optics, mode) : 0;
    bool replay = graphable && G.exec && G.key == key && G.epoch == device_alloc_epoch() &&
                  G.model_version == ctx->model_version;
    if (!replay && graphable && G.want == key && G.seen >= 1) {
        // a second attempt within the call: a library may initialise
        // something on the first captured use of an object
        for (int attempt = 0; attempt < 2 && !replay; ++attempt)
            replay = batch_capture(ctx, key, imgs, ws, hs, pxs, on_device, *optics, mode);
    }
    SearchPending pend;
    std::vector<float> pxn;
    gcf_status st = GCF_OK;
    if (replay) {
        cudaError_t e = cudaGraphLaunch(G.exec, ctx->st);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "cudaGraphLaunch");
        pend.nj = G.nj;
        pend.st = ctx->st;
        pend.band = G.band;
        pxn = G.pxn;
        ctx->kev_used = G.kev_used;
        ctx->launches = G.launches;
        ctx->graph_launches = 1;
    } else {
        ctx->arena.reset();   // every earlier call has completed
        st = batch_enqueue(ctx, imgs, ws, hs, pxs, on_device, *optics, mode, pend, pxn);
        if (graphable) {
            if (G.want != key) {
                G.want = key;
                G.seen = 0;
            }
            G.seen += 1;
        }
    }
    if (st == GCF_OK) {
        std::vector<gcf_result> r;
        st = search_collect(ctx, pxn, mode == GCF_SEARCH_PLAIN ? pxs.data() : nullptr, *optics, mode, pend, r);
        if (st == GCF_OK)
            for (int i = 0; i < n; ++i) results[i] = r[i];
    }
    cudaEventRecord(t1, ctx->st);
    cudaEventSynchronize(t1);
    if (st == GCF_OK) accumulate_stage_times(ctx);
    float tt = 0;
    cudaEventElapsedTime(&tt, t0, t1);
    ctx->stage_ms[6] = tt;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return st;
}

}  // namespace

extern "C" {

gcf_status gcf_run_batch(gcf_ctx* ctx, const gcf_item* items, int n, int on_device,
                         const gcf_optics* optics, gcf_result* results)
{
    if (!ctx || !items || n <= 0 || !valid_optics(optics) || !results) return GCF_ERR_INVALID_ARG;
    return batch_run(ctx, items, n, on_device, optics, GCF_SEARCH_PLAIN, results);
}

gcf_status gcf_run_batch_mode(gcf_ctx* ctx, const gcf_item* items, int n, int on_device,
                              const gcf_optics* optics, int mode, gcf_result* results)
{
    if (mode == GCF_SEARCH_PLAIN) return gcf_run_batch(ctx, items, n, on_device, optics, results);
    if (!ctx || !items || n <= 0 || !valid_optics(optics) || !results) return GCF_ERR_INVALID_ARG;
    if (mode != GCF_SEARCH_BF16 && mode != GCF_SEARCH_LEARNED) return GCF_ERR_INVALID_ARG;
    if (optics->ext_phase_range > 0) {
        // the table search has no extra-phase dimension: phase-plate data
        // take the plain search
        return gcf_run_batch(ctx, items, n, on_device, optics, results);
    }
    if (mode == GCF_SEARCH_LEARNED && !ctx->nn_ready)
        return fail(ctx, GCF_ERR_STATE, "learned search: no network weights (gcf_nn_load / gcf_nn_train)");
    return batch_run(ctx, items, n, on_device, optics, mode, results);
}

}  // extern "C"

namespace {

// Autotuner results, one per device for the life of the process.
struct TuneCache {
    bool done = false;
    gcf_tuning t{};
};
std::mutex g_tune_mu;
TuneCache g_tune[64];
constexpr int kTuneShapes[5] = {8, 816, 16, 162, 168};
// (tile N, stages, persistent)
constexpr int kTuneGemm[10][3] = {{256, 2, 0}, {256, 3, 0}, {256, 4, 0}, {128, 4, 0}, {128, 6, 0},
                                  {64, 4, 0},  {256, 3, 1}, {256, 4, 1}, {128, 4, 1}, {128, 6, 1}};

// Best of three timed runs after one warm-up of `run` on ctx->st, in ms.
template <class F>
gcf_status time_trial(gcf_ctx* ctx, cudaEvent_t a, cudaEvent_t b, F run, float* ms)
{
    *ms = 1e30f;
    for (int r = 0; r < 4; ++r) {
        CK(cudaEventRecord(a, ctx->st));
        CKS(run());
        CK(cudaEventRecord(b, ctx->st));
        CK(cudaEventSynchronize(b));
        float x = 0.0f;
        CK(cudaEventElapsedTime(&x, a, b));
        if (r > 0) *ms = std::min(*ms, x);
    }
    return GCF_OK;
}

gcf_status tune_device(gcf_ctx* ctx, gcf_tuning& t, cudaEvent_t a, cudaEvent_t b)
{
    // tile kernel: every cluster shape the device can hold, on four
    // synthetic 4096 x 4096 micrographs
    if (ctx->impl == GCF_SPECT_FUSED && fused_tile_supported(ctx->tile)) {
        const int W = 4096, H = 4096, nm = 4;
        DBuf<float> img;
        CK(img.ensure((size_t)W * H * nm));
        launch_fill_f32(img.p, (size_t)W * H * nm, 12345ull, 0.0f, 4.0f, ctx->st);
        CKL();
        std::vector<MicImage> mics(nm);
        for (int i = 0; i < nm; ++i) mics[i] = MicImage{img.p + (size_t)i * W * H, W, H, W, 1.35f};
        CKS(spectra_alloc(ctx, nm));
        float best = 1e30f;
        for (int si = 0; si < 5; ++si) {
            int ncl = 0;
            if (fused_clusters_of(kTuneShapes[si], &ncl) != cudaSuccess || ncl <= 0) {
                cudaGetLastError();
                t.fused_ms[si] = -1.0f;
                continue;
            }
            ctx->fused_clusters = ncl;
            ctx->fused_shape = kTuneShapes[si];
            ctx->solo_n = -1;
            CKS(fused_plan(ctx, mics));
            float ms = 0.0f;
            CKS(time_trial(ctx, a, b, [&] { return fused_launch(ctx, 0, nm, ctx->raw.p, ctx->st); }, &ms));
            t.fused_ms[si] = ms;
            if (ms < best) {
                best = ms;
                t.fused_shape = kTuneShapes[si];
            }
        }
        CK(cudaStreamSynchronize(ctx->st));
        img.release();
    }
    // contraction product: the table of a 128-micrograph batch (1024
    // defocus rows x 128 micrographs' angle bins x the s^2 bins)
    {
        const int M = 1024, K = ctx->contract_ns, N = 128 * ctx->contract_nth;
        DBuf<__nv_bfloat16> A, B;
        DBuf<float> D;
        DBuf<int> err;
        CK(A.ensure((size_t)M * K));
        CK(B.ensure((size_t)N * K));
        CK(D.ensure((size_t)M * N));
        CK(err.ensure(1));
        launch_fill_bf16(A.p, (size_t)M * K, 7ull, ctx->st);
        launch_fill_bf16(B.p, (size_t)N * K, 8ull, ctx->st);
        CKL();
        CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->st));
        float best = 1e30f;
        for (int q = 0; q < 10; ++q) {
            const int bn = kTuneGemm[q][0], stages = kTuneGemm[q][1], pers = kTuneGemm[q][2];
            if (bn < ctx->contract_nth || bn % ctx->contract_nth) {
                t.gemm_ms[q] = -1.0f;
                continue;
            }
            GemmArgs g;
            g.M = M;
            g.N = N;
            g.K = K;
            g.D = D.p;
            g.ldd = N;
            g.err = err.p;
            float ms = 0.0f;
            CKS(time_trial(ctx, a, b, [&]() -> gcf_status {
                if (pers) CK(launch_umma_gemm_persistent(A.p, K, B.p, K, g, bn, stages, 0, ctx->st));
                else CK(launch_umma_gemm(A.p, K, B.p, K, g, bn, stages, 0, ctx->st));
                return GCF_OK;
            }, &ms));
            t.gemm_ms[q] = ms;
            if (ms < best) {
                best = ms;
                t.gemm_tile_n = bn;
                t.gemm_stages = stages;
                t.gemm_persistent = pers;
            }
        }
        int h = 0;
        CK(cudaMemcpy(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) return fail(ctx, GCF_ERR_TIMEOUT, "tensor-core product trial: a bounded wait gave up");
    }
    return GCF_OK;
}

}  // namespace

extern "C" {

gcf_status gcf_autotune(gcf_ctx* ctx, int force, gcf_tuning* out)
{
    if (!ctx) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    if (ctx->dev < 0 || ctx->dev >= 64) return GCF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    TuneCache& C = g_tune[ctx->dev];
    if (!C.done || force) {
        gcf_tuning t{};
        cudaEvent_t a = nullptr, b = nullptr;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        gcf_status st = tune_device(ctx, t, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (st != GCF_OK) return st;
        C.t = t;
        C.done = true;
    }
    // the picks take effect from the next plan of this context
    if (C.t.fused_shape) {
        ctx->fused_shape_req = C.t.fused_shape;
        ctx->fused_clusters = 0;
        ctx->solo_n = -1;
    }
    if (C.t.gemm_tile_n) {
        ctx->gemm_bn = C.t.gemm_tile_n;
        ctx->gemm_stages = C.t.gemm_stages;
        ctx->gemm_persistent = C.t.gemm_persistent;
    }
    if (out) *out = C.t;
    return GCF_OK;
}

gcf_status gcf_mrc_load(gcf_ctx* ctx, const char* path, int z0, int n, const float** dev_images)
{
    if (!ctx || !path || n <= 0 || z0 < 0 || !dev_images) return GCF_ERR_INVALID_ARG;
    int dims[3], mode = 0;
    bool swap = false;
    long long off = 0;
    if (!mrc_layout(path, dims, &mode, &swap, &off)) return fail(ctx, GCF_ERR_IO, "cannot read the MRC header");
    const int mb = mrc_mode_bytes(mode);
    if (mb == 0) return fail(ctx, GCF_ERR_IO, "MRC mode not supported (0, 1, 2, 5, 6 are)");
    if ((long long)z0 + n > dims[2]) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    const size_t npx = (size_t)dims[0] * dims[1], sec = npx * mb;
    const size_t slot = (sec + 255) / 256 * 256;
    CK(ctx->loaded.ensure(npx * n));
    CK(ctx->ingest_raw.ensure(2 * slot));
    if (ctx->ingest_pin_bytes < 2 * slot) {
        if (ctx->ingest_pin) cudaFreeHost(ctx->ingest_pin);
        ctx->ingest_pin = nullptr;
        ctx->ingest_pin_bytes = 0;
        CK(cudaHostAlloc((void**)&ctx->ingest_pin, 2 * slot, cudaHostAllocDefault));
        ctx->ingest_pin_bytes = 2 * slot;
    }
    for (int k = 0; k < 2; ++k) {
        if (!ctx->ingest_copied[k]) CK(cudaEventCreateWithFlags(&ctx->ingest_copied[k], cudaEventDisableTiming));
        if (!ctx->ingest_used[k]) CK(cudaEventCreateWithFlags(&ctx->ingest_used[k], cudaEventDisableTiming));
    }
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ctx, GCF_ERR_IO, "cannot open the MRC file");
    gcf_status st = GCF_OK;
    // section k: wait until its staging pair is free (the copy of section
    // k - 2 is done on the host side, its conversion on the device side),
    // read it from disk while the GPU copies and converts section k - 1
    for (int k = 0; k < n && st == GCF_OK; ++k) {
        const int b = k & 1;
        unsigned char* pin = ctx->ingest_pin + b * slot;
        unsigned char* raw = ctx->ingest_raw.p + b * slot;
        cudaError_t e = cudaSuccess;
        if (k >= 2) e = cudaEventSynchronize(ctx->ingest_copied[b]);
        if (e != cudaSuccess) {
            st = cuda_fail(ctx, e, "mrc load");
            break;
        }
        if (fseeko(f, (off_t)(off + (long long)(z0 + k) * (long long)sec), SEEK_SET) != 0 ||
            std::fread(pin, 1, sec, f) != sec) {
            st = fail(ctx, GCF_ERR_IO, "short MRC section");
            break;
        }
        if ((e = cudaStreamWaitEvent(ctx->st_copy, ctx->ingest_used[b], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(raw, pin, sec, cudaMemcpyHostToDevice, ctx->st_copy)) != cudaSuccess ||
            (e = cudaEventRecord(ctx->ingest_copied[b], ctx->st_copy)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(ctx->st, ctx->ingest_copied[b], 0)) != cudaSuccess ||
            (e = launch_mrc_to_float(raw, mode, swap ? 1 : 0, npx, ctx->loaded.p + (size_t)k * npx, ctx->st)) !=
                cudaSuccess ||
            (e = cudaEventRecord(ctx->ingest_used[b], ctx->st)) != cudaSuccess) {
            st = cuda_fail(ctx, e, "mrc load");
            break;
        }
        dev_images[k] = ctx->loaded.p + (size_t)k * npx;
    }
    std::fclose(f);
    cudaError_t e = cudaStreamSynchronize(ctx->st);
    if (st == GCF_OK && e != cudaSuccess) st = cuda_fail(ctx, e, "mrc load");
    return st;
}

gcf_status gcf_set_graphs(gcf_ctx* ctx, int on)
{
    if (!ctx) return GCF_ERR_INVALID_ARG;
    ctx->graphs = on != 0;
    return GCF_OK;
}

gcf_status gcf_get_graph_info(gcf_ctx* ctx, long long info[4])
{
    if (!ctx || !info) return GCF_ERR_INVALID_ARG;
    info[0] = ctx->graph_launches;
    info[1] = ctx->bgraph.exec ? ctx->bgraph.nodes : 0;
    info[2] = ctx->bgraph.exec ? ctx->bgraph.launches : 0;
    info[3] = ctx->graph_fail;
    return GCF_OK;
}

// ---------------------------------------------------------------------------
// Learned initialiser
// ---------------------------------------------------------------------------
size_t gcf_nn_param_count(void) { return nn_param_count(); }

gcf_status gcf_nn_init(gcf_ctx* ctx, unsigned long long seed)
{
    if (!ctx) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    CKS(nn_ensure(ctx));
    CK(nn_init_random(ctx->nn, seed, ctx->st));
    ctx->nn_ready = true;
    ctx->nn_version += 1;
    return GCF_OK;
}

gcf_status gcf_nn_set_params(gcf_ctx* ctx, const float* params, size_t n)
{
    if (!ctx || !params || n != nn_param_count()) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    CKS(nn_ensure(ctx));
    CK(nn_set_params(ctx->nn, params, ctx->st));
    ctx->nn_ready = true;
    ctx->nn_version += 1;
    return GCF_OK;
}

gcf_status gcf_nn_get_params(gcf_ctx* ctx, float* params, size_t n)
{
    if (!ctx || !params || n != nn_param_count()) return GCF_ERR_INVALID_ARG;
    if (!ctx->nn) return fail(ctx, GCF_ERR_STATE, "no network");
    CKS(set_device(ctx));
    CK(nn_get_params(ctx->nn, params, ctx->st));
    return GCF_OK;
}

static const char kNnMagic[8] = {'G', 'C', 'F', 'N', 'N', '0', '0', '1'};

gcf_status gcf_nn_save(gcf_ctx* ctx, const char* path)
{
    if (!ctx || !path) return GCF_ERR_INVALID_ARG;
    const size_t n = nn_param_count();
    std::vector<float> h(n);
    CKS(gcf_nn_get_params(ctx, h.data(), n));
    FILE* f = fopen(path, "wb");
    if (!f) return fail(ctx, GCF_ERR_IO, "cannot open the weights file for writing");
    unsigned long long cnt = n;
    bool ok = fwrite(kNnMagic, 1, 8, f) == 8 && fwrite(&cnt, sizeof(cnt), 1, f) == 1 &&
              fwrite(h.data(), sizeof(float), n, f) == n;
    ok = (fclose(f) == 0) && ok;
    return ok ? GCF_OK : fail(ctx, GCF_ERR_IO, "weights file write failed");
}

gcf_status gcf_nn_load(gcf_ctx* ctx, const char* path)
{
    if (!ctx || !path) return GCF_ERR_INVALID_ARG;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(ctx, GCF_ERR_IO, "cannot open the weights file");
    char magic[8];
    unsigned long long cnt = 0;
    const size_t n = nn_param_count();
    std::vector<float> h(n);
    bool ok = fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kNnMagic, 8) == 0 &&
              fread(&cnt, sizeof(cnt), 1, f) == 1 && cnt == n && fread(h.data(), sizeof(float), n, f) == n;
    fclose(f);
    if (!ok) return fail(ctx, GCF_ERR_IO, "not a weights file of this network");
    return gcf_nn_set_params(ctx, h.data(), n);
}

gcf_status gcf_set_learned_threshold(gcf_ctx* ctx, float tau)
{
    if (!ctx || !(tau >= -1.0f && tau <= 1.0f)) return GCF_ERR_INVALID_ARG;
    ctx->learned_tau = tau;
    return GCF_OK;
}

gcf_status gcf_nn_train(gcf_ctx* ctx, const gcf_optics* optics, int steps, int batch, unsigned long long seed,
                        unsigned long long first, float lr, float* losses)
{
    if (!ctx || !valid_optics(optics) || steps <= 0 || batch <= 0 || batch > 4096 || !(lr > 0)) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    CKS(nn_ensure(ctx));
    if (!ctx->nn_ready) {
        CK(nn_init_random(ctx->nn, seed ^ 0x9E3779B97F4A7C15ull, ctx->st));
        ctx->nn_ready = true;
        ctx->nn_version += 1;
    }
    CK(ctx->nloss.ensure(steps));
    CK(cudaMemsetAsync(ctx->nloss.p, 0, steps * sizeof(float), ctx->st));
    CK(ctx->nx1.ensure((size_t)batch * kNnProfile));
    CK(ctx->nx2.ensure((size_t)batch * kNnMap * kNnMap));
    CK(cudaMemsetAsync(nn_err_flag(ctx->nn), 0, sizeof(int), ctx->st));
    for (int k = 0; k < steps; ++k) {
        const unsigned long long f0 = first + (unsigned long long)k * batch;
        CKS(synth_slots(ctx, *optics, seed, f0, batch));
        CK(launch_nn_input(ctx->ctf.p, ctx->tile, ctx->nparams.p + 3, 8, batch, ctx->nx1.p, ctx->nx2.p, ctx->st));
        CK(nn_forward(ctx->nn, ctx->nx1.p, ctx->nx2.p, batch, ctx->st));
        CK(nn_backward(ctx->nn, ctx->ntarget.p, batch, ctx->nloss.p + k, ctx->st));
        // cosine decay to 5 % of lr
        const float c = 0.5f * (1.0f + std::cos(3.14159265f * (float)k / (float)steps));
        CK(nn_adam(ctx->nn, lr * (0.05f + 0.95f * c), ctx->st));
    }
    int err = 0;
    CK(cudaMemcpyAsync(&err, nn_err_flag(ctx->nn), sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    if (losses) CK(cudaMemcpyAsync(losses, ctx->nloss.p, steps * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (err) return fail(ctx, GCF_ERR_TIMEOUT, "tensor-core product: a bounded wait gave up");
    return GCF_OK;
}

gcf_status gcf_nn_inputs(gcf_ctx* ctx, const float* spectra, const float* px, int n, float* x1, float* x2)
{
    if (!ctx || !spectra || !px || n <= 0 || n > kNnChunk) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    const size_t cmp_n = (size_t)(ctx->tile / 2 + 1) * ctx->tile;
    DBuf<float> ds, dp;
    DBuf<__nv_bfloat16> d1, d2;
    std::vector<__nv_bfloat16> h1((size_t)n * kNnProfile), h2((size_t)n * kNnMap * kNnMap);
    cudaError_t e = ds.ensure(cmp_n * n);
    if (e == cudaSuccess) e = dp.ensure(n);
    if (e == cudaSuccess) e = d1.ensure(h1.size());
    if (e == cudaSuccess) e = d2.ensure(h2.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds.p, spectra, cmp_n * n * sizeof(float), cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dp.p, px, n * sizeof(float), cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) e = launch_nn_input(ds.p, ctx->tile, dp.p, 1, n, d1.p, d2.p, ctx->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h1.data(), d1.p, h1.size() * 2, cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h2.data(), d2.p, h2.size() * 2, cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    ds.release();
    dp.release();
    d1.release();
    d2.release();
    CK(e);
    if (x1)
        for (size_t i = 0; i < h1.size(); ++i) x1[i] = __bfloat162float(h1[i]);
    if (x2)
        for (size_t i = 0; i < h2.size(); ++i) x2[i] = __bfloat162float(h2[i]);
    return GCF_OK;
}

gcf_status gcf_nn_synth_inputs(gcf_ctx* ctx, const gcf_optics* optics, unsigned long long seed,
                               unsigned long long first, int n, float* x1, float* x2, float* target, float* params)
{
    if (!ctx || !valid_optics(optics) || n <= 0 || n > kNnChunk) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    CKS(synth_slots(ctx, *optics, seed, first, n));
    CK(ctx->nx1.ensure((size_t)n * kNnProfile));
    CK(ctx->nx2.ensure((size_t)n * kNnMap * kNnMap));
    CK(launch_nn_input(ctx->ctf.p, ctx->tile, ctx->nparams.p + 3, 8, n, ctx->nx1.p, ctx->nx2.p, ctx->st));
    std::vector<__nv_bfloat16> h1((size_t)n * kNnProfile), h2((size_t)n * kNnMap * kNnMap);
    CK(cudaMemcpyAsync(h1.data(), ctx->nx1.p, h1.size() * 2, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(h2.data(), ctx->nx2.p, h2.size() * 2, cudaMemcpyDeviceToHost, ctx->st));
    if (target) CK(cudaMemcpyAsync(target, ctx->ntarget.p, (size_t)n * 3 * 4, cudaMemcpyDeviceToHost, ctx->st));
    if (params) CK(cudaMemcpyAsync(params, ctx->nparams.p, (size_t)n * 8 * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (x1)
        for (size_t i = 0; i < h1.size(); ++i) x1[i] = __bfloat162float(h1[i]);
    if (x2)
        for (size_t i = 0; i < h2.size(); ++i) x2[i] = __bfloat162float(h2[i]);
    return GCF_OK;
}

gcf_status gcf_nn_forward_backward(gcf_ctx* ctx, const float* x1, const float* x2, const float* target, int n,
                                   float* loss, float* grads, float* pred)
{
    if (!ctx || !x1 || !x2 || !target || n <= 0 || n > kNnChunk) return GCF_ERR_INVALID_ARG;
    if (!ctx->nn || !ctx->nn_ready) return fail(ctx, GCF_ERR_STATE, "no network weights");
    CKS(set_device(ctx));
    std::vector<__nv_bfloat16> h1((size_t)n * kNnProfile), h2((size_t)n * kNnMap * kNnMap);
    for (size_t i = 0; i < h1.size(); ++i) h1[i] = __float2bfloat16_rn(x1[i]);
    for (size_t i = 0; i < h2.size(); ++i) h2[i] = __float2bfloat16_rn(x2[i]);
    CK(ctx->nx1.ensure(h1.size()));
    CK(ctx->nx2.ensure(h2.size()));
    CK(ctx->ntarget.ensure((size_t)n * 3));
    CK(ctx->nloss.ensure(1));
    CK(h2d(ctx, ctx->nx1.p, h1.data(), h1.size() * 2, ctx->st));
    CK(h2d(ctx, ctx->nx2.p, h2.data(), h2.size() * 2, ctx->st));
    CK(h2d(ctx, ctx->ntarget.p, target, (size_t)n * 3 * 4, ctx->st));
    CK(cudaMemsetAsync(ctx->nloss.p, 0, sizeof(float), ctx->st));
    CK(cudaMemsetAsync(nn_err_flag(ctx->nn), 0, sizeof(int), ctx->st));
    CK(nn_forward(ctx->nn, ctx->nx1.p, ctx->nx2.p, n, ctx->st));
    CK(nn_backward(ctx->nn, ctx->ntarget.p, n, ctx->nloss.p, ctx->st));
    int err = 0;
    CK(cudaMemcpyAsync(&err, nn_err_flag(ctx->nn), sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    if (loss) CK(cudaMemcpyAsync(loss, ctx->nloss.p, sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    if (pred)
        CK(cudaMemcpy2DAsync(pred, 3 * sizeof(float), nn_pred(ctx->nn), kNnPredPitch * sizeof(float),
                             3 * sizeof(float), n, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (err) return fail(ctx, GCF_ERR_TIMEOUT, "tensor-core product: a bounded wait gave up");
    if (grads) CK(nn_get_grads(ctx->nn, grads, ctx->st));
    return GCF_OK;
}

gcf_status gcf_nn_eval_synthetic(gcf_ctx* ctx, const gcf_optics* optics, unsigned long long seed,
                                 unsigned long long first, int n, int mode, gcf_result* results, float* params)
{
    if (!ctx || !valid_optics(optics) || n <= 0 || !results) return GCF_ERR_INVALID_ARG;
    if (mode != GCF_SEARCH_PLAIN && mode != GCF_SEARCH_BF16 && mode != GCF_SEARCH_LEARNED) return GCF_ERR_INVALID_ARG;
    CKS(set_device(ctx));
    for (long long& c : ctx->search_counts) c = 0;
    for (long long& c : ctx->fast_counts) c = 0;
    for (float& t : ctx->fast_ms) t = 0.0f;
    gcf_optics op = *optics;
    op.ext_phase_range = 0.0f;
    for (int c0 = 0; c0 < n; c0 += kNnChunk) {
        const int cn = std::min(kNnChunk, n - c0);
        CKS(synth_slots(ctx, op, seed, first + (unsigned long long)c0, cn));
        std::vector<float> prm((size_t)cn * 8);
        CK(cudaMemcpyAsync(prm.data(), ctx->nparams.p, prm.size() * 4, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        std::vector<float> pxn(cn);
        for (int i = 0; i < cn; ++i) pxn[i] = prm[(size_t)i * 8 + 3];
        std::vector<gcf_result> r;
        CKS(search_slots(ctx, pxn, op, mode, r));
        for (int i = 0; i < cn; ++i) results[c0 + i] = r[i];
        if (params) std::memcpy(params + (size_t)c0 * 8, prm.data(), prm.size() * 4);
    }
    return GCF_OK;
}

gcf_status gcf_get_fast_counts(gcf_ctx* ctx, long long counts[4])
{
    if (!ctx || !counts) return GCF_ERR_INVALID_ARG;
    for (int i = 0; i < 4; ++i) counts[i] = ctx->fast_counts[i];
    return GCF_OK;
}

gcf_status gcf_get_fast_times(gcf_ctx* ctx, float times_ms[5])
{
    if (!ctx || !times_ms) return GCF_ERR_INVALID_ARG;
    for (int i = 0; i < 5; ++i) times_ms[i] = ctx->fast_ms[i];
    return GCF_OK;
}

gcf_status gcf_get_stage_times(gcf_ctx* ctx, float times_ms[7])
{
    if (!ctx || !times_ms) return GCF_ERR_INVALID_ARG;
    for (int i = 0; i < 7; ++i) times_ms[i] = ctx->stage_ms[i];
    return GCF_OK;
}

gcf_status gcf_get_search_counts(gcf_ctx* ctx, long long counts[4])
{
    if (!ctx || !counts) return GCF_ERR_INVALID_ARG;
    for (int i = 0; i < 4; ++i) counts[i] = ctx->search_counts[i];
    return GCF_OK;
}

gcf_status gcf_get_launch_count(gcf_ctx* ctx, long long* count)
{
    if (!ctx || !count) return GCF_ERR_INVALID_ARG;
    *count = ctx->launches;
    return GCF_OK;
}

}  // extern "C"
