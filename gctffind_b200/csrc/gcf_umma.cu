// gcf_umma.cu -- BF16 x BF16 -> FP32 matrix product on the 5th-generation
// tensor cores (tcgen05.mma with the accumulator in tensor memory, operands
// staged by TMA), the building block of the candidate contraction and of the
// learned initialiser's layers.
//
//   D[m][n] = sum_k A[m][k] * B[n][k]          (A: M x K, B: N x K, both
//                                               row-major = K-major)
//
// One CTA computes one 128 x BN tile of D (BN = 32 .. 256) from a list of
// tiles, so a caller can ask for any subset of the output (a band of rows per
// column block).  Four warps: warp 0 lane 0 issues the TMA loads of a
// STAGES-deep ring of 64-wide K slices (SWIZZLE_128B, the layout the MMA
// descriptors below describe), warp 1 lane 0 issues the MMAs (128 x BN x 16
// per instruction) and commits each slice back to the ring, warp 2 owns the
// tensor-memory allocation; after the last MMA all four warps move the
// accumulator out of tensor memory (warp w holds rows 32w .. 32w+31) through
// a swizzled shared-memory stage into coalesced global stores, with an
// optional bias, ReLU, BF16 conversion and transposed copy.
//
// k_umma_gemm_persistent (below) is the same product for many tiles: one CTA
// per SM walks the tile list, with the accumulator double-buffered in tensor
// memory so that each tile's epilogue overlaps the next tile's MMAs.
//
// Every wait is bounded (about one second of global timer): a wait that runs
// out records an error code in *err, the roles stop issuing work, the
// producer waits (bounded) for the loads it has in flight, and the CTA frees
// its tensor memory and returns.  No TMA load here uses cluster multicast;
// every tensor map covers this GPU's own memory.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <mutex>

#include "gcf_internal.h"

namespace gcf {

namespace {

constexpr int kBM = 128;           // rows of a tile (MMA M)
constexpr int kBK = 64;            // K slice per stage: 64 BF16 = one 128-byte swizzle row
constexpr int kUK = 16;            // K per MMA instruction (kind::f16)
constexpr int kThreads = 128;
constexpr uint64_t kWaitNs = 1000000000ull;   // bounded waits: 1 s

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; false after about
// kWaitNs without it.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_test(bar, parity)) return true;
        if ((it & 31) == 0 && global_ns() - t0 > kWaitNs) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major operand tile whose rows are
// 128 bytes (64 BF16) in the 128-byte swizzle that TMA writes: 8-row groups
// of 1024 bytes (stride-dimension offset), descriptor version 1, layout type
// 2 = SWIZZLE_128B.  The leading-dimension offset is unused for a swizzled
// K-major operand whose K slice fits in one swizzle row (set to 1).
__device__ __forceinline__ uint64_t desc_k128(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor: D FP32, A and B BF16, both K-major, M = 128, N = bn.
__host__ __device__ constexpr uint32_t idesc_bf16(int bn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 consecutive accumulator columns of this warp's 32 lanes (one row per
// thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// One warp's 32 rows of a 128 x BN accumulator in tensor memory (columns
// from tacc, the warp's lane quarter q) to global memory: bias, ReLU, and any
// of the FP32 (through a swizzled 4 KB shared-memory stage, 4 rows x 128 B
// per store), BF16 and transposed BF16 outputs.  write = false only drains
// the tensor-memory loads.
template <int BN>
__device__ __forceinline__ void store_accumulator(const GemmArgs& g, uint32_t tacc, int q, int lane, int m0, int n0,
                                                  unsigned char* sb, bool write)
{
    const int row0 = m0 + 32 * q;
#pragma unroll 1
    for (int c = 0; c < BN / 32; ++c) {
        uint32_t v[32];
        tmem_ld32(tacc + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * c), v);
        if (!write) continue;
        const int col0 = n0 + 32 * c;
        float f[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            float x = __uint_as_float(v[i]);
            if (g.bias) {
                const int n = col0 + i;
                x += (n < g.N) ? g.bias[n] : 0.0f;
            }
            if (g.relu) x = fmaxf(x, 0.0f);
            f[i] = x;
        }
        const int myrow = row0 + lane;
        if (g.Dt) {
            // transposed BF16 copy: Dt[n][m]; lanes are consecutive m
            if (myrow < g.M) {
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const int n = col0 + i;
                    if (n < g.N) g.Dt[(size_t)n * g.ldt + myrow] = __float2bfloat16_rn(f[i]);
                }
            }
        }
        if (g.Db) {
            // BF16 row-major copy
            if (myrow < g.M) {
                __nv_bfloat16* dst = g.Db + (size_t)myrow * g.ldd + col0;
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (col0 + i < g.N) dst[i] = __float2bfloat16_rn(f[i]);
            }
        }
        if (g.D) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float4 t = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
                *reinterpret_cast<float4*>(sb + lane * 128 + ((j ^ (lane & 7)) << 4)) = t;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int r = 4 * i + (lane >> 3), j = lane & 7;
                float4 t = *reinterpret_cast<const float4*>(sb + r * 128 + ((j ^ (r & 7)) << 4));
                const int m = row0 + r, n = col0 + 4 * j;
                if (m < g.M) {
                    float* dst = g.D + (size_t)m * g.ldd + n;
                    if (n + 3 < g.N && g.vec4) {
                        if (g.accumulate) {
                            float4 o = *reinterpret_cast<float4*>(dst);
                            t.x += o.x;
                            t.y += o.y;
                            t.z += o.z;
                            t.w += o.w;
                        }
                        *reinterpret_cast<float4*>(dst) = t;
                    } else {
                        const float e[4] = {t.x, t.y, t.z, t.w};
                        for (int u = 0; u < 4; ++u)
                            if (n + u < g.N) dst[u] = g.accumulate ? dst[u] + e[u] : e[u];
                    }
                }
            }
            __syncwarp();
        }
    }
}

template <int BN, int STAGES>
struct GemmSmem {
    static constexpr int kA = kBM * kBK * 2;       // 16 KB per stage
    static constexpr int kB = BN * kBK * 2;
    static constexpr int kStage = kA + kB;
    static constexpr int kBars = 1024;            // barriers + tensor-memory address (one 1 KB block)
    static constexpr int kBytes = 1024 /*alignment slack*/ + STAGES * kStage + kBars;
};

}  // namespace

// ---------------------------------------------------------------------------
template <int BN, int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
k_umma_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g)
{
    using L = GemmSmem<BN, STAGES>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = smem;
    unsigned char* sB = smem + STAGES * L::kA;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * L::kStage);
    // bars[0, STAGES): slice loaded; [STAGES, 2 STAGES): slice consumed; [2 STAGES]: accumulator ready
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 1);
    int* s_abort = reinterpret_cast<int*>(s_taddr + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (g.ntiles && (int)blockIdx.x >= *g.ntiles) return;   // beyond the planned tiles
    int m0, n0;
    if (g.tiles) {
        const int2 t = g.tiles[blockIdx.x];
        m0 = t.x;
        n0 = t.y;
    } else {
        m0 = blockIdx.y * kBM;
        n0 = blockIdx.x * BN;
    }
    const int nkb = (g.K + kBK - 1) / kBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < 2 * STAGES + 1; ++s) mbar_init(smem_u32(bars + s), 1);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_taddr)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_taddr;
    const uint32_t done_bar = smem_u32(bars + 2 * STAGES);

    if (warp == 0 && lane == 0) {
        // producer: TMA loads of the K slices into the ring
        int issued = 0;
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % STAGES;
            if (kb >= STAGES && !mbar_wait(smem_u32(bars + STAGES + s), ((kb / STAGES) & 1) ^ 1)) {
                atomicExch(g.err, 1);
                atomicExch(s_abort, 1);
                break;
            }
            if (*(volatile int*)s_abort) break;
            const uint32_t fb = smem_u32(bars + s);
            mbar_expect_tx(fb, L::kStage);
            tma_load_2d(smem_u32(sA + s * L::kA), &ta, fb, kb * kBK, m0);
            tma_load_2d(smem_u32(sB + s * L::kB), &tb, fb, kb * kBK, n0);
            issued = kb + 1;
        }
        // on an abort, wait (bounded) for the loads still in flight before the
        // CTA's shared memory is released
        if (*(volatile int*)s_abort) {
            for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; ++kb)
                mbar_wait(smem_u32(bars + (kb % STAGES)), (kb / STAGES) & 1);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = idesc_bf16(BN);
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % STAGES;
            if (!mbar_wait(smem_u32(bars + s), (kb / STAGES) & 1)) {
                atomicExch(g.err, 2);
                atomicExch(s_abort, 1);
                break;
            }
            tc_fence_after();
            const uint64_t da = desc_k128(smem_u32(sA + s * L::kA));
            const uint64_t db = desc_k128(smem_u32(sB + s * L::kB));
#pragma unroll
            for (int k = 0; k < kBK / kUK; ++k) {
                // the next 16 K elements start 32 bytes further in every row
                umma(tmem, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, (kb > 0 || k > 0) ? 1u : 0u);
            }
            umma_commit(smem_u32(bars + STAGES + s));   // frees the slot when these MMAs are done
        }
        umma_commit(done_bar);   // accumulator complete (also after an abort: nothing in flight then)
    }
    __syncwarp();

    // epilogue: all four warps (the tensor-memory loads are warp-wide
    // .sync.aligned instructions: every decision before them is made
    // uniform across the warp)
    const bool ok = __all_sync(0xffffffffu, mbar_wait(done_bar, 0));
    if (!ok && lane == 0) atomicExch(g.err, 3);
    tc_fence_after();
    __syncthreads();   // every role is past its loop: the ring's shared memory is free
    const bool write = __all_sync(0xffffffffu, ok && !*(volatile int*)s_abort);
    store_accumulator<BN>(g, tmem, warp, lane, m0, n0, smem + warp * 4096, write);
    tc_fence_before();
    __syncthreads();
    if (warp == 2)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

// ---------------------------------------------------------------------------
// Persistent variant for products of many tiles (the contraction table): one
// CTA per SM walks the tile list with a stride of the grid, and the
// accumulator is double-buffered in tensor memory (2 x BN columns), so the
// epilogue of one tile overlaps the MMAs of the next and the TMA loads of
// the one after.  Six warps: warp 0 lane 0 the TMA producer (one ring of K
// slices across all of the CTA's tiles), warp 1 the tensor-memory
// allocation and lane 0 of it the MMA issuer, warps 2-5 the epilogue (warp w
// reads tensor-memory lanes 32 (w mod 4) .. +31, i.e. those rows of the tile).
// Hand-offs: full/empty per ring slot, acc_full/acc_empty per accumulator
// buffer; every wait bounded as in k_umma_gemm.
constexpr int kPThreads = 192;

template <int BN, int STAGES>
struct PGemmSmem {
    static constexpr int kA = kBM * kBK * 2;
    static constexpr int kB = BN * kBK * 2;
    static constexpr int kStage = kA + kB;
    static constexpr int kEpi = 4 * 4096;          // four epilogue warps' stages
    static constexpr int kBars = 1024;
    static constexpr int kBytes = 1024 + STAGES * kStage + kEpi + kBars;
};

template <int BN, int STAGES>
__global__ void __launch_bounds__(kPThreads, 1)
k_umma_gemm_persistent(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g,
                       int ntiles_grid)
{
    using L = PGemmSmem<BN, STAGES>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = smem;
    unsigned char* sB = smem + STAGES * L::kA;
    unsigned char* sEpi = smem + STAGES * L::kStage;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sEpi + L::kEpi);
    // [0, S): slice loaded; [S, 2S): slice consumed; 2S, 2S+1: accumulator b
    // full; 2S+2, 2S+3: accumulator b drained
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
    int* s_abort = reinterpret_cast<int*>(s_taddr + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = g.ntiles ? *g.ntiles : ntiles_grid;
    const int gn = (g.N + BN - 1) / BN;   // column tiles of the whole grid
    const int nkb = (g.K + kBK - 1) / kBK;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2 * STAGES + 2; ++i) mbar_init(smem_u32(bars + i), 1);
        mbar_init(smem_u32(bars + 2 * STAGES + 2), 4);
        mbar_init(smem_u32(bars + 2 * STAGES + 3), 4);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_taddr)),
                     "r"(2 * BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_taddr;
    volatile int* abort_flag = s_abort;

    if (warp == 0 && lane == 0) {
        // producer
        int it = 0;
        for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
            int m0, n0;
            if (g.tiles) {
                const int2 tt = g.tiles[t];
                m0 = tt.x;
                n0 = tt.y;
            } else {
                m0 = (t / gn) * kBM;
                n0 = (t % gn) * BN;
            }
            for (int kb = 0; kb < nkb; ++kb, ++it) {
                const int s = it % STAGES;
                if (it >= STAGES && !mbar_wait(smem_u32(bars + STAGES + s), ((it / STAGES) & 1) ^ 1)) {
                    atomicExch(g.err, 1);
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                const uint32_t fb = smem_u32(bars + s);
                mbar_expect_tx(fb, L::kStage);
                tma_load_2d(smem_u32(sA + s * L::kA), &ta, fb, kb * kBK, m0);
                tma_load_2d(smem_u32(sB + s * L::kB), &tb, fb, kb * kBK, n0);
            }
        }
        // on an abort, the loads still in flight land before the CTA exits
        if (*abort_flag)
            for (int j = (it > STAGES ? it - STAGES : 0); j < it; ++j)
                mbar_wait(smem_u32(bars + (j % STAGES)), (j / STAGES) & 1);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = idesc_bf16(BN);
        int it = 0, i = 0;
        for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x, ++i) {
            const int b = i & 1, use = i >> 1;
            if (use > 0 && !mbar_wait(smem_u32(bars + 2 * STAGES + 2 + b), (use - 1) & 1)) {
                atomicExch(g.err, 4);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const uint32_t tacc = tmem + (uint32_t)(b * BN);
            bool bad = false;
            for (int kb = 0; kb < nkb; ++kb, ++it) {
                const int s = it % STAGES;
                if (!mbar_wait(smem_u32(bars + s), (it / STAGES) & 1)) {
                    atomicExch(g.err, 2);
                    *abort_flag = 1;
                    bad = true;
                    break;
                }
                tc_fence_after();
                const uint64_t da = desc_k128(smem_u32(sA + s * L::kA));
                const uint64_t db = desc_k128(smem_u32(sB + s * L::kB));
#pragma unroll
                for (int k = 0; k < kBK / kUK; ++k)
                    umma(tacc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, (kb > 0 || k > 0) ? 1u : 0u);
                umma_commit(smem_u32(bars + STAGES + s));
            }
            umma_commit(smem_u32(bars + 2 * STAGES + b));   // accumulator b complete (or abandoned)
            if (bad) break;
        }
    } else if (warp >= 2) {
        // epilogue warps
        const int q = warp & 3;
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
            // warp-uniform decisions: the tensor-memory loads are .sync.aligned
            if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
            const int b = i & 1, use = i >> 1;
            if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(bars + 2 * STAGES + b), use & 1))) {
                if (lane == 0) {
                    atomicExch(g.err, 3);
                    *abort_flag = 1;
                }
                break;
            }
            tc_fence_after();
            int m0, n0;
            if (g.tiles) {
                const int2 tt = g.tiles[t];
                m0 = tt.x;
                n0 = tt.y;
            } else {
                m0 = (t / gn) * kBM;
                n0 = (t % gn) * BN;
            }
            const bool wr = !__any_sync(0xffffffffu, *abort_flag != 0);
            store_accumulator<BN>(g, tmem + (uint32_t)(b * BN), q, lane, m0, n0, sEpi + (warp - 2) * 4096, wr);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bars + 2 * STAGES + 2 + b))
                                        : "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN) : "memory");
}

// ---------------------------------------------------------------------------
// Host side: tensor maps through the driver entry point (no -lcuda), kernel
// attributes, launch.
namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

cudaError_t get_encode()
{
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return g_encode ? cudaSuccess : cudaErrorNotSupported;
}

// K-major BF16 operand: rows x k elements, row pitch ld elements; box 64 x box_rows.
cudaError_t make_map(CUtensorMap* m, const void* base, long long rows, long long k, long long ld, int box_rows)
{
    cudaError_t e = get_encode();
    if (e != cudaSuccess) return e;
    cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int BN, int STAGES>
cudaError_t launch_bn(const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& g, int ntiles, cudaStream_t st)
{
    using L = GemmSmem<BN, STAGES>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(k_umma_gemm<BN, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        L::kBytes);
    });
    if (attr_err != cudaSuccess) return attr_err;
    dim3 grid;
    if (g.tiles) grid = dim3(ntiles, 1, 1);
    else grid = dim3((g.N + BN - 1) / BN, (g.M + kBM - 1) / kBM, 1);
    k_umma_gemm<BN, STAGES><<<grid, kThreads, L::kBytes, st>>>(ta, tb, g);
    return cudaGetLastError();
}

template <int BN, int STAGES>
cudaError_t launch_pbn(const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& g, int ntiles, cudaStream_t st)
{
    using L = PGemmSmem<BN, STAGES>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(k_umma_gemm_persistent<BN, STAGES>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
    });
    if (attr_err != cudaSuccess) return attr_err;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int grid_tiles = ((g.M + kBM - 1) / kBM) * ((g.N + BN - 1) / BN);
    const int total = g.tiles ? ntiles : grid_tiles;   // an upper bound with a device tile count
    const int grid = std::max(1, std::min(total, sms));
    k_umma_gemm_persistent<BN, STAGES><<<grid, kPThreads, L::kBytes, st>>>(ta, tb, g, grid_tiles);
    return cudaGetLastError();
}

}  // namespace

int umma_tile_n_supported(int bn) { return bn == 32 || bn == 64 || bn == 128 || bn == 256; }

cudaError_t launch_umma_gemm_persistent(const __nv_bfloat16* A, long long lda, const __nv_bfloat16* B,
                                        long long ldb, GemmArgs g, int bn, int stages, int ntiles, cudaStream_t st)
{
    if (!umma_tile_n_supported(bn) || g.M <= 0 || g.N <= 0 || g.K <= 0 || !g.err) return cudaErrorInvalidValue;
    if (((uintptr_t)A & 15) || ((uintptr_t)B & 15) || (lda * 2) % 16 || (ldb * 2) % 16 || lda < g.K || ldb < g.K)
        return cudaErrorInvalidValue;
    if (g.tiles && ntiles <= 0) return cudaSuccess;
    g.vec4 = (g.D && ((uintptr_t)g.D & 15) == 0 && g.ldd % 4 == 0) ? 1 : 0;
    CUtensorMap ta, tb;
    cudaError_t e;
    if ((e = make_map(&ta, A, g.M, g.K, lda, kBM)) != cudaSuccess) return e;
    if ((e = make_map(&tb, B, g.N, g.K, ldb, bn)) != cudaSuccess) return e;
    switch (bn * 10 + stages) {
    case 2563: return launch_pbn<256, 3>(ta, tb, g, ntiles, st);
    case 2564: return launch_pbn<256, 4>(ta, tb, g, ntiles, st);
    case 1284: return launch_pbn<128, 4>(ta, tb, g, ntiles, st);
    case 1286: return launch_pbn<128, 6>(ta, tb, g, ntiles, st);
    case 644: return launch_pbn<64, 4>(ta, tb, g, ntiles, st);
    case 324: return launch_pbn<32, 4>(ta, tb, g, ntiles, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_umma_gemm(const __nv_bfloat16* A, long long lda, const __nv_bfloat16* B, long long ldb,
                             GemmArgs g, int bn, int stages, int ntiles, cudaStream_t st)
{
    if (!umma_tile_n_supported(bn) || g.M <= 0 || g.N <= 0 || g.K <= 0 || !g.err) return cudaErrorInvalidValue;
    // TMA: 16-byte aligned bases and row pitches
    if (((uintptr_t)A & 15) || ((uintptr_t)B & 15) || (lda * 2) % 16 || (ldb * 2) % 16 || lda < g.K || ldb < g.K)
        return cudaErrorInvalidValue;
    if (g.tiles && ntiles <= 0) return cudaSuccess;
    g.vec4 = (g.D && ((uintptr_t)g.D & 15) == 0 && g.ldd % 4 == 0) ? 1 : 0;
    CUtensorMap ta, tb;
    cudaError_t e;
    if ((e = make_map(&ta, A, g.M, g.K, lda, kBM)) != cudaSuccess) return e;
    if ((e = make_map(&tb, B, g.N, g.K, ldb, bn)) != cudaSuccess) return e;
    switch (bn * 10 + stages) {
    case 2562: return launch_bn<256, 2>(ta, tb, g, ntiles, st);
    case 2563: return launch_bn<256, 3>(ta, tb, g, ntiles, st);
    case 2564: return launch_bn<256, 4>(ta, tb, g, ntiles, st);
    case 1282: return launch_bn<128, 2>(ta, tb, g, ntiles, st);
    case 1284: return launch_bn<128, 4>(ta, tb, g, ntiles, st);
    case 1286: return launch_bn<128, 6>(ta, tb, g, ntiles, st);
    case 642: return launch_bn<64, 2>(ta, tb, g, ntiles, st);
    case 644: return launch_bn<64, 4>(ta, tb, g, ntiles, st);
    case 322: return launch_bn<32, 2>(ta, tb, g, ntiles, st);
    case 324: return launch_bn<32, 4>(ta, tb, g, ntiles, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace gcf

// ---------------------------------------------------------------------------
// C ABI: the product on caller-owned device buffers (tests, tuning).
namespace {
__device__ int g_umma_err_flag;
}

extern "C" gcf_status gcf_gemm_bf16_ex(const void* a, long long lda, const void* b, long long ldb, int m, int n,
                                       int k, float* d, long long ldd, int tile_n, int stages, int persistent,
                                       void* cuda_stream)
{
    using namespace gcf;
    if (!a || !b || !d || m <= 0 || n <= 0 || k <= 0 || ldd < n) return GCF_ERR_INVALID_ARG;
    int* flag = nullptr;
    if (cudaGetSymbolAddress((void**)&flag, g_umma_err_flag) != cudaSuccess || !flag) return GCF_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    if (cudaMemsetAsync(flag, 0, sizeof(int), st) != cudaSuccess) return GCF_ERR_CUDA;
    GemmArgs g;
    g.M = m;
    g.N = n;
    g.K = k;
    g.D = d;
    g.ldd = ldd;
    g.err = flag;
    cudaError_t e = persistent ? launch_umma_gemm_persistent(static_cast<const __nv_bfloat16*>(a), lda,
                                                             static_cast<const __nv_bfloat16*>(b), ldb, g, tile_n,
                                                             stages, 0, st)
                               : launch_umma_gemm(static_cast<const __nv_bfloat16*>(a), lda,
                                                  static_cast<const __nv_bfloat16*>(b), ldb, g, tile_n, stages, 0, st);
    if (e == cudaErrorInvalidValue) return GCF_ERR_INVALID_ARG;
    if (e != cudaSuccess) return GCF_ERR_CUDA;
    int hflag = 0;
    if (cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return GCF_ERR_CUDA;
    return hflag ? GCF_ERR_TIMEOUT : GCF_OK;
}

extern "C" gcf_status gcf_gemm_bf16(const void* a, long long lda, const void* b, long long ldb, int m, int n,
                                    int k, float* d, long long ldd, int tile_n, int stages, void* cuda_stream)
{
    return gcf_gemm_bf16_ex(a, lda, b, ldb, m, n, k, d, ldd, tile_n, stages, 0, cuda_stream);
}
