// Learned k-step corrector: BF16 tcgen05 GEMMs (FP32 accumulation in TMEM), message passing over
// the mesh adjacency, SiLU, MSE loss and Adam -- forward, backward and optimiser all hand-written.
//
// GEMM form used throughout:  D[M][N] = epilogue(A[M][K] . B[N][K]^T)
//   A, B: bf16, row-major, K contiguous ("K-major" for both UMMA operands); M any (128-row tiles,
//   rows past M read as zero and are not stored); N in {32, 64, 128, 256}; K a multiple of 64.
// One CTA of 128 threads computes one 128 x N tile:
//   * the K loop stages 64-wide slices of A and B in shared memory in the canonical no-swizzle
//     K-major core-matrix layout (8 rows x 16 bytes per core matrix; the two 16-byte K halves of an
//     MMA step LBO = 128 B apart; 8-row groups SBO = 256 B apart);
//   * one elected thread issues tcgen05.mma.cta_group::1.kind::f16 (M = 128, N, K = 16) four times
//     per slice and tcgen05.commit's completion to an mbarrier, which all threads wait on with an
//     iteration limit (a timeout sets the error flag instead of hanging);
//   * the accumulator lives in tensor memory (N fp32 columns x 128 lanes, allocated per CTA); the
//     epilogue reads it back with tcgen05.ld (warp w owns lanes 32w..32w+31 = rows of the tile),
//     adds the bias, stores the pre-activation if asked, applies SiLU, adds a residual, and writes
//     fp32 and/or bf16.
// Split-K (for weight gradients, K = number of cells): `k_splits` > 1 makes each CTA handle one
// K range and atomically add its fp32 tile into D (no epilogue other than the add).
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>

#include "fvm_common.cuh"

namespace fvm {
namespace corr {

constexpr int TM = 128;          // tile rows (UMMA M)
constexpr int TK = 64;           // K slice staged per iteration
constexpr int kGemmThreads = 128;
constexpr long long kWaitLimit = 1LL << 22;   // mbarrier polls before a wait gives up

struct GemmArgs {
    const __nv_bfloat16* A;
    int64_t lda;
    const __nv_bfloat16* B;
    int64_t ldb;
    int M, N, K;
    int k_splits;                 // > 1: split-K with atomic accumulation into Df
    const float* bias;            // [N] or null
    const float* resid;           // [M][ldr] fp32 added after the activation, or null
    int64_t ldr;
    float* Df;                    // [M][ldd] fp32 output (or accumulation target), or null
    __nv_bfloat16* Db;            // [M][ldd] bf16 output, or null
    int64_t ldd;
    float* preact;                // [M][ldd] fp32 pre-activation, or null
    int act;                      // 0 none, 1 SiLU
    int* err;                     // device error flag (set to 1 on an mbarrier timeout)
    int vec;                      // every epilogue row chunk is 32-byte aligned: 256-bit accesses
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory matrix descriptor: no swizzle, K-major, version 1 (sm100).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;       // descriptor version for tcgen05
    return d;                      // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: D fp32, A and B bf16, both K-major, M = 128.
__host__ __device__ constexpr uint32_t make_idesc(int N) {
    return (1u << 4)                      // D format: F32
           | (1u << 7)                    // A format: BF16
           | (1u << 10)                   // B format: BF16
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(TM >> 4) << 24); // M / 16
}

// Stage rows [r0, r0 + nrows) x K columns [k0, k0 + 64) of a row-major bf16 matrix into the
// core-matrix layout: 16-byte unit (row r, unit u of 8 K elements) -> slice u/2, half u%2.
__device__ __forceinline__ void stage_tile(uint8_t* smem, const __nv_bfloat16* src, int64_t ld, int r0, int rows_valid,
                                           int nrows, int k0, int kmax) {
    const int units = nrows * (TK / 8);
    const int slice_bytes = (nrows / 8) * 256;
    for (int t = threadIdx.x; t < units; t += blockDim.x) {
        const int r = t >> 3, u = t & 7;
        const int k = k0 + 8 * u;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (r < rows_valid && k < kmax) v = *reinterpret_cast<const uint4*>(src + (int64_t)(r0 + r) * ld + k);
        const int off = (u >> 1) * slice_bytes + (r >> 3) * 256 + (u & 1) * 128 + (r & 7) * 16;
        *reinterpret_cast<uint4*>(smem + off) = v;
    }
}

// Same layout as stage_tile, copied global -> shared by cp.async (no registers; rows past
// rows_valid and columns past kmax are zero-filled).  Thread -> (row, unit) mapping: the 32 lanes
// of a warp take 8 consecutive rows x 4 units, so their 16-byte stores cover all 32 banks once per
// 8 lanes (conflict-free) and each row's 4 units are 64 contiguous global bytes.
__device__ __forceinline__ void stage_tile_async(uint8_t* smem, const __nv_bfloat16* src, int64_t ld, int r0,
                                                 int rows_valid, int nrows, int k0, int kmax) {
    const int units = nrows * (TK / 8);
    const int slice_bytes = (nrows / 8) * 256;
    const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    for (int t = threadIdx.x; t < units; t += blockDim.x) {
        const int r = (t & 7) + 8 * (t >> 6), u = (t >> 3) & 7;
        const int k = k0 + 8 * u;
        const bool valid = r < rows_valid && k < kmax;
        const __nv_bfloat16* gp = valid ? src + (int64_t)(r0 + r) * ld + k : src;
        const uint32_t off = (uint32_t)((u >> 1) * slice_bytes + (r >> 3) * 256 + (u & 1) * 128 + (r & 7) * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(base + off), "l"(gp),
                     "r"(valid ? 16 : 0)
                     : "memory");
    }
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done = 0;
    for (long long it = 0; it < kWaitLimit && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(bar))), "r"(parity));
    }
    return done != 0;
}

// z sigmoid(z) with the fast-division intrinsic: the denominator is >= 1, so the intrinsic's range
// limit only matters where exp overflows and the quotient is 0 anyway (within 2 ulp elsewhere).
// Every residual added to it goes through __fadd_rn, so no kernel fuses the quotient's multiply
// with that add and all kernels round alike (the fused layer equals GEMM + epilogue bitwise).
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.f + __expf(-z)); }

// 8 consecutive floats (32-byte aligned) with one 256-bit access.
__device__ __forceinline__ void ld8(const float* p, float* v) {
    asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}
__device__ __forceinline__ void st8(float* p, const float* v) {
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
                 "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
}

// Epilogue of 32 consecutive accumulator columns [c0, c0 + 32) of one row with 256-bit accesses:
// each thread reads and writes whole 32-byte sectors of its own row (no partial-sector traffic).
__device__ __forceinline__ void epilogue_vec(const GemmArgs& g, int64_t row, int c0, const uint32_t (&r)[32]) {
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
    if (g.bias) {
        float b[32];
#pragma unroll
        for (int q = 0; q < 4; ++q) ld8(g.bias + c0 + 8 * q, b + 8 * q);
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += b[j];
    }
    if (g.preact)
#pragma unroll
        for (int q = 0; q < 4; ++q) st8(g.preact + row * g.ldd + c0 + 8 * q, v + 8 * q);
    if (g.act == 1)
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = silu(v[j]);
    if (g.resid) {
        float x[32];
#pragma unroll
        for (int q = 0; q < 4; ++q) ld8(g.resid + row * g.ldr + c0 + 8 * q, x + 8 * q);
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = __fadd_rn(v[j], x[j]);
    }
    if (g.Df)
#pragma unroll
        for (int q = 0; q < 4; ++q) st8(g.Df + row * g.ldd + c0 + 8 * q, v + 8 * q);
    if (g.Db) {
        float pk[16];   // bf16 pairs, bit patterns carried in float registers
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            pk[j] = __uint_as_float(*reinterpret_cast<const uint32_t*>(&h));
        }
        float* dst = reinterpret_cast<float*>(g.Db + row * g.ldd + c0);
        st8(dst, pk);
        st8(dst + 8, pk + 8);
    }
}

template <int N>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(GemmArgs g) {
    // Two staging buffers of one K slice each (A: TM x TK, B: N x TK, bf16): slice j + 1 is copied
    // (cp.async) while the tensor cores work on slice j; a buffer is refilled only after the MMAs
    // that read it have completed (their commit's mbarrier).
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int kStageBytes = TM * TK * 2 + N * TK * 2;
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t s_taddr;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TM;
    const int split = blockIdx.y;
    const int kchunks = g.K / TK;
    const int per = (kchunks + g.k_splits - 1) / g.k_splits;
    const int kc0 = split * per, kc1 = min(kchunks, kc0 + per);
    const int nk = max(0, kc1 - kc0);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"((uint32_t)(N < 32 ? 32 : N)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t taddr = s_taddr;
    const uint32_t idesc = make_idesc(N);
    const int rows_a = min(TM, g.M - m0);
    // The epilogue's residual rows (one contiguous block of the tile's rows) go to L2 while the
    // tile is loaded and multiplied: the bulk-copy unit prefetches them, so the epilogue's loads
    // see L2 latency instead of DRAM latency.
    if (threadIdx.x == 0 && g.resid && g.k_splits == 1 && g.vec && rows_a > 0) {
        const uint32_t bytes = (uint32_t)((int64_t)rows_a * g.ldr * 4) & ~15u;
        if (bytes) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g.resid + (int64_t)m0 * g.ldr),
                                "r"(bytes) : "memory");
    }
    auto stage = [&](int buf, int kc) {
        uint8_t* sA = smem + buf * kStageBytes;
        stage_tile_async(sA, g.A, g.lda, m0, rows_a, TM, kc * TK, g.K);
        stage_tile_async(sA + TM * TK * 2, g.B, g.ldb, 0, g.N, N, kc * TK, g.K);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    bool ok = true;
    for (int j = 0; j < min(2, nk); ++j) stage(j, kc0 + j);
    for (int j = 0; j < nk && ok; ++j) {
        const int buf = j & 1;
        if (j + 1 < nk) asm volatile("cp.async.wait_group 1;" ::: "memory");
        else asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t sa = smem_u32(smem + buf * kStageBytes), sb = sa + TM * TK * 2;
#pragma unroll
            for (int s = 0; s < TK / 16; ++s) {
                const uint64_t ad = make_desc(sa + s * (TM / 8) * 256, 128, 256);
                const uint64_t bd = make_desc(sb + s * (N / 8) * 256, 128, 256);
                const uint32_t acc = (j > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(taddr),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar[buf]))
                         : "memory");
        }
        // Refill this buffer with slice j + 2 once its MMAs are done; after the last slice, wait
        // for the last commit (the MMAs of one thread complete in order).
        const bool refill = j + 2 < nk, last = j + 1 == nk;
        if (refill || last) {                              // uniform across the block
            bool done = mbar_wait(&mbar[buf], (uint32_t)((j >> 1) & 1));
            if (!done) {
                // Give the MMAs in flight a second bounded chance to finish before the tensor memory
                // they write is released; the timeout is reported below.
                done = mbar_wait(&mbar[buf], (uint32_t)((j >> 1) & 1)) && false;
            }
            // one verdict for the whole block (also the barrier before the buffer is refilled)
            ok = __syncthreads_and(done) != 0;
            if (!ok) {
                if (threadIdx.x == 0 && g.err) atomicExch(g.err, 1);
            } else if (refill) {
                stage(buf, kc0 + j + 2);
            }
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("tcgen05.fence::after_thread_sync;");
    const bool have = ok && kc1 > kc0;
    // Epilogue: warp w owns tile rows 32w .. 32w + 31 (TMEM lanes).
    const int row = m0 + warp * 32 + lane;
    if (have) {
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 32) {
            uint32_t r[32];
            const uint32_t a = taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(a));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (row < g.M && g.vec && g.k_splits == 1) {
                epilogue_vec(g, row, c0, r);
            } else if (row < g.M) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = c0 + j;
                    if (col >= g.N) break;
                    float v = __uint_as_float(r[j]);
                    if (g.k_splits > 1) {
                        atomicAdd(g.Df + (int64_t)row * g.ldd + col, v);
                        continue;
                    }
                    if (g.bias) v += g.bias[col];
                    if (g.preact) g.preact[(int64_t)row * g.ldd + col] = v;
                    if (g.act == 1) v = silu(v);
                    if (g.resid) v = __fadd_rn(v, g.resid[(int64_t)row * g.ldr + col]);
                    if (g.Df) g.Df[(int64_t)row * g.ldd + col] = v;
                    if (g.Db) g.Db[(int64_t)row * g.ldd + col] = __float2bfloat16(v);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                     "r"((uint32_t)(N < 32 ? 32 : N)));
}

template <int N>
static int launch_gemm(const GemmArgs& g, cudaStream_t s) {
    // one staging buffer per K slice a CTA handles, at most two (fewer bytes: more CTAs per SM)
    const int kchunks = g.K / TK, per = (kchunks + g.k_splits - 1) / g.k_splits;
    const size_t smem = (size_t)(per >= 2 ? 2 : 1) * ((size_t)TM * TK * 2 + (size_t)N * TK * 2);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * ((size_t)TM * TK * 2 + (size_t)N * TK * 2)));
        attr = true;
    }
    dim3 grid((unsigned)((g.M + TM - 1) / TM), (unsigned)g.k_splits);
    FVM_LAUNCH(KID_CORRECTOR, s, k_gemm<N><<<grid, kGemmThreads, smem, s>>>(g));
    return launch_status();
}

}  // namespace corr
}  // namespace fvm

using namespace fvm;

extern "C" int fvm_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                             int32_t k_splits, const float* bias, const float* resid, int64_t ldr, float* Df,
                             void* Db, int64_t ldd, float* preact, int32_t act, int32_t* err, void* stream) {
    if (!A || !B || M <= 0 || K <= 0 || K % corr::TK != 0 || k_splits < 1 || (!Df && !Db) || !err) return FVM_E_ARG;
    if (N != 32 && N != 64 && N != 128 && N != 256) return FVM_E_UNSUPPORTED;
    if ((uintptr_t)A % 16 || (uintptr_t)B % 16 || lda % 8 || ldb % 8) return FVM_E_ARG;
    if (k_splits > 1 && (!Df || bias || resid || preact || Db || act)) return FVM_E_ARG;
    // 256-bit epilogue when every row chunk of 32 columns starts on a 32-byte boundary.
    auto a32 = [](const void* p) { return ((uintptr_t)p & 31u) == 0; };
    const int vec = a32(bias) && a32(resid) && a32(Df) && a32(Db) && a32(preact) && (!resid || ldr % 8 == 0) &&
                    ((!Df && !preact) || ldd % 8 == 0) && (!Db || ldd % 16 == 0);
    corr::GemmArgs g{static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B), ldb, M, N, K,
                     k_splits, bias, resid, ldr, Df, static_cast<__nv_bfloat16*>(Db), ldd, preact, act, err, vec};
    cudaStream_t s = (cudaStream_t)stream;
    switch (N) {
        case 32: return corr::launch_gemm<32>(g, s);
        case 64: return corr::launch_gemm<64>(g, s);
        case 128: return corr::launch_gemm<128>(g, s);
        default: return corr::launch_gemm<256>(g, s);
    }
}

// ------------------------------------------------------------------------------------------
// Message passing, activations, loss and optimiser kernels of the corrector.
// Activations h: bf16 [N][W] (W = 64); neighbour table nbr: int32 [N][KN] (-1 = none).
// ------------------------------------------------------------------------------------------
namespace fvm {
namespace corr {

// dh_out[i] = dh_in[i] + dA[i][:W] + sum_{j in nbr(i)} dA[j][W:] / deg(j)   (adjacency symmetric).
__global__ void k_mp_scatter_back(const float* __restrict__ dA, const int32_t* __restrict__ nbr, int N, int W, int KN,
                                  const float* __restrict__ dh_in, float* __restrict__ dh_out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * W) return;
    const int i = (int)(t / W), c = (int)(t % W);
    float v = dA[(int64_t)i * 2 * W + c] + (dh_in ? dh_in[t] : 0.f);
    for (int k = 0; k < KN; ++k) {
        const int j = __ldg(nbr + (int64_t)i * KN + k);
        if (j < 0) continue;
        int deg = 0;
        for (int q = 0; q < KN; ++q) deg += __ldg(nbr + (int64_t)j * KN + q) >= 0;
        v += dA[(int64_t)j * 2 * W + W + c] / (float)deg;
    }
    dh_out[t] = v;
}

// dZ = dh * silu'(Z); writes dZ as bf16 [N][W] and transposed bf16 [W][ldT] (columns >= N zero),
// and accumulates the bias gradient sum_i dZ[i].
__global__ void k_silu_back(const float* __restrict__ dh, const float* __restrict__ Z, int N, int W,
                            __nv_bfloat16* __restrict__ dZ, __nv_bfloat16* __restrict__ dZT, int64_t ldT,
                            float* __restrict__ db) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * W) return;
    const int i = (int)(t / W), c = (int)(t % W);
    const float z = Z[t];
    const float s = 1.f / (1.f + __expf(-z));
    const float g = dh[t] * s * (1.f + z * (1.f - s));
    dZ[t] = __float2bfloat16(g);
    if (dZT) dZT[(int64_t)c * ldT + i] = __float2bfloat16(g);
    if (db) atomicAdd(db + c, g);
}

// dst[c][r] = src[r][c] for a bf16 [R][Cc] matrix (32 x 32 tiles through shared memory).
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ src, int R, int Cc, int64_t lds,
                                 __nv_bfloat16* __restrict__ dst, int64_t ldd) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;   // rows on x: R may exceed 65535 * 32
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < R && c < Cc) ? src[(int64_t)r * lds + c] : __float2bfloat16(0.f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < Cc && r < R) dst[(int64_t)c * ldd + r] = tile[threadIdx.x][k];
    }
}

__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ tgt, int64_t n_elem, float inv_n,
                      double* __restrict__ loss, float* __restrict__ dpred) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    __shared__ double red[32];
    double v[1] = {0.0};
    if (t < n_elem) {
        const float d = pred[t] - tgt[t];
        dpred[t] = 2.f * d * inv_n;
        v[0] = (double)d * d * inv_n;
    }
    block_sum<1>(v, red);
    if (threadIdx.x == 0) atomicAdd(loss, v[0]);
}

// Adam (decoupled bias correction) on fp32 master weights; refreshes the bf16 copy [rows][cols]
// and, if requested, its transpose [cols][rows] used by the backward GEMMs.  Zeroes the gradient.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ pb, __nv_bfloat16* __restrict__ pbT, int rows, int cols) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gr = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gr;
    const float vt = b2 * v[t] + (1.f - b2) * gr * gr;
    m[t] = mt;
    v[t] = vt;
    const float w = p[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    p[t] = w;
    g[t] = 0.f;
    if (pb) pb[t] = __float2bfloat16(w);
    if (pbT) {
        const int r = (int)(t / cols), c = (int)(t % cols);
        pbT[(int64_t)c * rows + r] = __float2bfloat16(w);
    }
}

// Network input: X[i] = [(U_i - mean) * inv_std (C values), geometry (G values), zeros] bf16 [N][64].
__global__ void k_features(const float* __restrict__ state, int N, int C, const float* __restrict__ mean,
                           const float* __restrict__ inv_std, const float* __restrict__ geo, int G,
                           __nv_bfloat16* __restrict__ X, int XW) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * XW) return;
    const int i = (int)(t / XW), c = (int)(t % XW);
    float v = 0.f;
    if (c < C) v = (state[(int64_t)i * C + c] - mean[c]) * inv_std[c];
    else if (c < C + G) v = geo[(int64_t)i * G + (c - C)];
    X[t] = __float2bfloat16(v);
}

// U_new = U + scale * out (out: normalised increment, fp32 [N][C]).
__global__ void k_apply_increment(const float* __restrict__ state, const float* __restrict__ out,
                                  const float* __restrict__ scale, int N, int C, float* __restrict__ new_state) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * C) return;
    new_state[t] = state[t] + scale[t % C] * out[t];
}

// Corrector inputs, one thread per cell: base = k dt(case) * r0 and the bf16 feature row
// [(U - mean) * inv_std, (base - mean) * inv_std, geometry, zeros] (XW entries).
template <int C>
__global__ void k_corrector_inputs(const float* __restrict__ state, const float* __restrict__ r0,
                                   const float* __restrict__ kdt_case, const int32_t* __restrict__ cell_case, int N,
                                   const float* __restrict__ mean, const float* __restrict__ inv_std,
                                   const float* __restrict__ geo, int G, float* __restrict__ base,
                                   __nv_bfloat16* __restrict__ X, int XW) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float h = kdt_case[cell_case ? __ldg(cell_case + i) : 0];
    float u[C], b[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        u[c] = __ldg(state + (int64_t)i * C + c);
        b[c] = h * __ldg(r0 + (int64_t)i * C + c);
        base[(int64_t)i * C + c] = b[c];
    }
    __nv_bfloat16* row = X + (int64_t)i * XW;
    // entries 0..15 hold the 2C <= 10 state / baseline features (indices known at compile time)
#pragma unroll
    for (int q = 0; q < 16; q += 8) {
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int c = q + e;
            float x = 0.f;
            if (c < C) x = (u[c < C ? c : 0] - __ldg(mean + c)) * __ldg(inv_std + c);
            else if (c < 2 * C) x = (b[(c >= C && c < 2 * C) ? c - C : 0] - __ldg(mean + c)) * __ldg(inv_std + c);
            else if (c < 2 * C + G) x = __ldg(geo + (int64_t)i * G + (c - 2 * C));
            v[e] = __float2bfloat16(x);
        }
        *reinterpret_cast<uint4*>(row + q) = *reinterpret_cast<const uint4*>(v);
    }
    for (int q = 16; q < XW; q += 8) {
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int c = q + e;
            v[e] = __float2bfloat16(c < 2 * C + G ? __ldg(geo + (int64_t)i * G + (c - 2 * C)) : 0.f);
        }
        *reinterpret_cast<uint4*>(row + q) = *reinterpret_cast<const uint4*>(v);
    }
}

// prop = state + base + scale * out - shift(case)  (shift: per-case [C] offsets, or null).
__global__ void k_corrector_combine(const float* __restrict__ state, const float* __restrict__ base,
                                    const float* __restrict__ out, const float* __restrict__ scale,
                                    const float* __restrict__ shift, const int32_t* __restrict__ cell_case, int N,
                                    int C, float* __restrict__ prop) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * C) return;
    const int i = (int)(t / C), c = (int)(t % C);
    float v = state[t] + base[t] + __ldg(scale + c) * out[t];
    if (shift) v -= __ldg(shift + (int64_t)(cell_case ? __ldg(cell_case + i) : 0) * C + c);
    prop[t] = v;
}

static inline unsigned nblk(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace corr
}  // namespace fvm

extern "C" int fvm_mp_scatter_back(const float* dA, const int32_t* nbr, int32_t N, int32_t W, int32_t KN,
                                   const float* dh_in, float* dh_out, void* stream) {
    if (!dA || !nbr || !dh_out || N <= 0 || W <= 0 || KN <= 0) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_mp_scatter_back<<<corr::nblk((int64_t)N * W, 256), 256, 0, s>>>(
                                     dA, nbr, N, W, KN, dh_in, dh_out));
    return launch_status();
}

extern "C" int fvm_silu_back(const float* dh, const float* Z, int32_t N, int32_t W, void* dZ, void* dZT, int64_t ldT,
                             float* db, void* stream) {
    if (!dh || !Z || !dZ || N <= 0 || W <= 0 || (dZT && ldT < N)) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_silu_back<<<corr::nblk((int64_t)N * W, 256), 256, 0, s>>>(
                                     dh, Z, N, W, static_cast<__nv_bfloat16*>(dZ), static_cast<__nv_bfloat16*>(dZT),
                                     ldT, db));
    return launch_status();
}

extern "C" int fvm_transpose_bf16(const void* src, int32_t R, int32_t Cc, int64_t lds, void* dst, int64_t ldd,
                                  void* stream) {
    if (!src || !dst || R <= 0 || Cc <= 0 || ldd < R || lds < Cc || (Cc + 31) / 32 > 65535) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid((unsigned)((R + 31) / 32), (unsigned)((Cc + 31) / 32));
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_transpose_bf16<<<grid, dim3(32, 8), 0, s>>>(
                                     static_cast<const __nv_bfloat16*>(src), R, Cc, lds,
                                     static_cast<__nv_bfloat16*>(dst), ldd));
    return launch_status();
}

extern "C" int fvm_mse(const float* pred, const float* tgt, int64_t n_elem, double* loss, float* dpred,
                       void* stream) {
    if (!pred || !tgt || !loss || !dpred || n_elem <= 0) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_mse<<<corr::nblk(n_elem, 256), 256, 0, s>>>(
                                     pred, tgt, n_elem, 1.f / (float)n_elem, loss, dpred));
    return launch_status();
}

extern "C" int fvm_adam(float* p, float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                        float eps, int32_t step, void* pb, void* pbT, int32_t rows, int32_t cols, void* stream) {
    if (!p || !g || !m || !v || n <= 0 || step < 1 || (pbT && (int64_t)rows * cols != n)) return FVM_E_ARG;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_adam<<<corr::nblk(n, 256), 256, 0, s>>>(
                                     p, g, m, v, n, lr, beta1, beta2, eps, c1, c2, static_cast<__nv_bfloat16*>(pb),
                                     static_cast<__nv_bfloat16*>(pbT), rows, cols));
    return launch_status();
}

extern "C" int fvm_corrector_features(const float* state, int32_t N, int32_t C, const float* mean,
                                      const float* inv_std, const float* geo, int32_t G, void* X, int32_t XW,
                                      void* stream) {
    if (!state || !mean || !inv_std || !X || N <= 0 || C + G > XW || (G > 0 && !geo)) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_features<<<corr::nblk((int64_t)N * XW, 256), 256, 0, s>>>(
                                     state, N, C, mean, inv_std, geo, G, static_cast<__nv_bfloat16*>(X), XW));
    return launch_status();
}

extern "C" int fvm_apply_increment(const float* state, const float* out, const float* scale, int32_t N, int32_t C,
                                   float* new_state, void* stream) {
    if (!state || !out || !scale || !new_state || N <= 0 || C <= 0) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_apply_increment<<<corr::nblk((int64_t)N * C, 256), 256, 0, s>>>(
                                     state, out, scale, N, C, new_state));
    return launch_status();
}

extern "C" int fvm_corrector_inputs(const float* state, const float* r0, const float* kdt_case,
                                    const int32_t* cell_case, int32_t N, int32_t C, const float* mean,
                                    const float* inv_std, const float* geo, int32_t G, float* base, void* X,
                                    int32_t XW, void* stream) {
    if (!state || !r0 || !kdt_case || !mean || !inv_std || (G > 0 && !geo) || !base || !X || N <= 0 || G < 0 ||
        XW % 8 != 0 || XW < 16 || 2 * C + G > XW || ((uintptr_t)X & 15u) != 0)
        return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (C == 4)
        FVM_LAUNCH(KID_CORRECTOR, s, corr::k_corrector_inputs<4><<<corr::nblk(N, 128), 128, 0, s>>>(
                                         state, r0, kdt_case, cell_case, N, mean, inv_std, geo, G, base,
                                         static_cast<__nv_bfloat16*>(X), XW));
    else if (C == 5)
        FVM_LAUNCH(KID_CORRECTOR, s, corr::k_corrector_inputs<5><<<corr::nblk(N, 128), 128, 0, s>>>(
                                         state, r0, kdt_case, cell_case, N, mean, inv_std, geo, G, base,
                                         static_cast<__nv_bfloat16*>(X), XW));
    else
        return FVM_E_UNSUPPORTED;
    return launch_status();
}

extern "C" int fvm_corrector_combine(const float* state, const float* base, const float* out, const float* scale,
                                     const float* shift, const int32_t* cell_case, int32_t N, int32_t C, float* prop,
                                     void* stream) {
    if (!state || !base || !out || !scale || !prop || N <= 0 || C <= 0) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_corrector_combine<<<corr::nblk((int64_t)N * C, 256), 256, 0, s>>>(
                                     state, base, out, scale, shift, cell_case, N, C, prop));
    return launch_status();
}


// ------------------------------------------------------------------------------------------
// Persistent message-passing layer on an fp32 residual stream (fvm_mp_layer).
//
//   h'_i = h_i + SiLU([bf16(h_i), bf16(mean_{j in nbr(i)} h_j)] . W^T + b)       (W: bf16 [64][128])
//   and, for the last layer, out_i = W_out h'_i + b_out instead of storing h'.
//
// One CTA per SM slot runs a grid-stride loop over 128-row tiles with three roles:
//   * warps 0-7 (loaders): stage tile k's A operand (128 x 128 bf16, canonical no-swizzle K-major
//     core-matrix layout, two K slices: own row, neighbour mean) into shared-memory stage k % 2;
//     the neighbour mean is an fp32 sum over the valid neighbours in table order times 1 / count
//     (the gathers are latency-bound: eight warps, each thread with two rows' loads in flight);
//   * thread 0 (a loader) issues the tile's eight tcgen05.mma (M 128, N 64, K 16) into tensor-memory
//     accumulator k % 2 and commits to two mbarriers: "stage free" and "accumulator full";
//   * warps 8-11 (epilogue): read accumulator k % 2 (warp 8 + w owns TMEM lanes 32w..32w+31 = tile
//     rows), free it for tile k + 2 (an mbarrier), add bias, SiLU, the fp32 residual and store h'
//     (or the decoder's outputs) with 256-bit accesses.
// So the gathers of tile k + 1, the MMAs of tile k and the epilogue of tile k - 1 overlap.  The
// weights stay in shared memory for the whole launch.  Every mbarrier wait is bounded; a wait that
// gives up sets *err and ends the role's loop, and the final MMA wait is bounded too, so the kernel
// always returns and frees its tensor memory.
// ------------------------------------------------------------------------------------------
namespace fvm {
namespace corr {

constexpr int kLayerLoaders = 256;                       // warps 0-7: gathers (+ the MMA issuer)
constexpr int kLayerThreads = kLayerLoaders + 128;       // warps 8-11: epilogue
constexpr int kLayerW = 64;                              // channels
constexpr int kLayerStageBytes = 2 * TM * TK * 2;        // two K slices of 128 x 64 bf16
constexpr int kLayerWBytes = kLayerW * 2 * kLayerW * 2;  // W: 64 x 128 bf16
constexpr int kLayerSmem = kLayerWBytes + 2 * kLayerStageBytes + 1024;

struct LayerArgs {
    const float* h;              // [M][64] fp32 residual stream (input)
    const int32_t* nbr;          // [M][KN]
    int M, KN;
    const __nv_bfloat16* Wt;     // [64][128]
    const float* bias;           // [64]
    float* h_out;                // [M][64] or null (decoder only)
    const float* Wo;             // [O][64] decoder weights or null
    const float* bo;             // [O]
    int O;
    float* out;                  // [M][O] decoder outputs or null
    int* err;
};

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void loader_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
// Named barrier of the 256 loader threads that also returns whether any of them passed v != 0,
// so every loader takes the same branch afterwards.
__device__ __forceinline__ int loader_sync_or(int v) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 256, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"(v)
        : "memory");
    return r;
}

// 32 accumulator columns [c0, c0 + 32) of this warp's TMEM lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Stage rows [m0, m0 + 128) of tile into the two K slices at sA (own row, neighbour mean), bf16.
// Loader thread lt (0..255) handles the 8-channel unit u = (lt >> 3) & 7 of rows
// (lt & 7) + 8 * (lt >> 6) + 32 q, q = 0..3: a warp covers 8 rows x 4 units per q, so its 16-byte
// shared-memory stores hit all 32 banks once per 8 lanes and its global reads are 128-byte row
// segments.  With at most KM <= 4 neighbours the loads of two rows (own + KM neighbours each) are
// all issued before any is used -- a missing neighbour reads the row itself and contributes +0,
// which leaves the sum unchanged (the sum starts at +0 and is never -0) -- so a thread keeps ten
// 32-byte loads in flight instead of one; wider neighbour lists take the row-by-row loop.
__device__ __forceinline__ void stage_store(uint8_t* sA, int r, int u, const float (&own)[8], const float (&acc)[8],
                                            float inv) {
    const int slice_bytes = (TM / 8) * 256;
    __align__(16) __nv_bfloat16 a[8], b[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        a[e] = __float2bfloat16(own[e]);
        b[e] = __float2bfloat16(acc[e] * inv);
    }
    const int off = (u >> 1) * slice_bytes + (r >> 3) * 256 + (u & 1) * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(sA + off) = *reinterpret_cast<const uint4*>(a);
    *reinterpret_cast<uint4*>(sA + TM * TK * 2 + off) = *reinterpret_cast<const uint4*>(b);
}

template <int KM>
__device__ __forceinline__ void stage_layer_tile_batched(uint8_t* sA, const LayerArgs& g, int m0, const int* s_nb,
                                                         const float* s_inv, int lt) {
    const int u = (lt >> 3) & 7;
#pragma unroll 1
    for (int q0 = 0; q0 < 4; q0 += 2) {
        float own[2][8], nb[2][KM][8];
        bool use[2][KM];
        int rs[2];
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int r = (lt & 7) + 8 * (lt >> 6) + 32 * (q0 + b);
            rs[b] = r;
            const int64_t row = (int64_t)m0 + r;
            const bool valid = row < g.M;
            const int64_t self = valid ? row : 0;
            ld8(g.h + self * kLayerW + 8 * u, own[b]);
#pragma unroll
            for (int k = 0; k < KM; ++k) {
                const int j = k < g.KN ? s_nb[r * 8 + k] : -1;
                use[b][k] = valid && j >= 0;
                ld8(g.h + (use[b][k] ? (int64_t)j : self) * kLayerW + 8 * u, nb[b][k]);
            }
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const bool valid = (int64_t)m0 + rs[b] < g.M;
            float o[8], acc[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                o[e] = valid ? own[b][e] : 0.f;
                acc[e] = 0.f;
            }
#pragma unroll
            for (int k = 0; k < KM; ++k)
#pragma unroll
                for (int e = 0; e < 8; ++e) acc[e] += use[b][k] ? nb[b][k][e] : 0.f;
            stage_store(sA, rs[b], u, o, acc, s_inv[rs[b]]);
        }
    }
}

__device__ __forceinline__ void stage_layer_tile(uint8_t* sA, const LayerArgs& g, int m0, const int* s_nb,
                                                 const float* s_inv, int lt) {
    if (g.KN <= 4) {
        stage_layer_tile_batched<4>(sA, g, m0, s_nb, s_inv, lt);
        return;
    }
    const int u = (lt >> 3) & 7;
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        const int r = (lt & 7) + 8 * (lt >> 6) + 32 * q;
        const int64_t row = (int64_t)m0 + r;
        const bool valid = row < g.M;
        float own[8], acc[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) own[e] = acc[e] = 0.f;
        if (valid) {
            ld8(g.h + row * kLayerW + 8 * u, own);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (k >= g.KN) break;
                const int j = s_nb[r * 8 + k];
                if (j < 0) continue;
                float v[8];
                ld8(g.h + (int64_t)j * kLayerW + 8 * u, v);
#pragma unroll
                for (int e = 0; e < 8; ++e) acc[e] += v[e];
            }
        }
        stage_store(sA, r, u, own, acc, s_inv[r]);
    }
}

__global__ void __launch_bounds__(kLayerThreads, 1) k_mp_layer(LayerArgs g) {
    extern __shared__ __align__(1024) uint8_t dsmem[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)dsmem + 1023) & ~(uintptr_t)1023);
    uint8_t* sW = smem;                                   // B operand, both K slices
    uint8_t* sStage = smem + kLayerWBytes;                // two stages of A
    __shared__ __align__(8) uint64_t bar_free[2], bar_full[2], bar_empty[2];
    __shared__ uint32_t s_taddr;
    __shared__ int s_nb[TM * 8];
    __shared__ float s_inv[TM];
    __shared__ float s_bias[kLayerW];
    __shared__ float s_wo[8 * kLayerW];
    __shared__ int s_fail;
    __shared__ int s_last;                                // last local tile whose MMAs were issued
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (g.M + TM - 1) / TM;
    const int nlocal = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"(128u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(&bar_free[b], 1);
            mbar_init(&bar_full[b], 1);
            mbar_init(&bar_empty[b], 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
        s_fail = 0;
        s_last = -1;
    }
    // weights into the B-operand layout (both K slices), bias and decoder weights
    for (int t = threadIdx.x; t < 2 * kLayerW * 8; t += blockDim.x) {
        const int c = t / (kLayerW * 8), rem = t % (kLayerW * 8);
        const int r = rem >> 3, u = rem & 7;
        const uint4 v = *reinterpret_cast<const uint4*>(g.Wt + (int64_t)r * 2 * kLayerW + c * TK + 8 * u);
        const int off = c * (kLayerW * TK * 2) + (u >> 1) * ((kLayerW / 8) * 256) + (r >> 3) * 256 + (u & 1) * 128 +
                        (r & 7) * 16;
        *reinterpret_cast<uint4*>(sW + off) = v;
    }
    for (int t = threadIdx.x; t < kLayerW; t += blockDim.x) s_bias[t] = g.bias[t];
    if (g.out)
        for (int t = threadIdx.x; t < g.O * kLayerW; t += blockDim.x) s_wo[t] = g.Wo[t];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t taddr = s_taddr;
    const uint32_t idesc = make_idesc(kLayerW);

    if (warp < kLayerLoaders / 32) {
        // ---- loaders (and, thread 0, the MMA issuer) ----
        // Every decision to stop is taken together (loader_sync_or), so no loader is left waiting
        // at a named barrier: a loader's own bounded wait that gave up, or thread 0's, counts.
        const int lt = threadIdx.x;
        int fail = 0;
        // neighbour lists are fetched one tile ahead (the gathers of a tile then wait for one
        // memory round trip, not two)
        int nxt[8];
        auto fetch_nbr = [&](int tile) {
            const int64_t row = (int64_t)tile * TM + lt;
#pragma unroll
            for (int q = 0; q < 8; ++q)
                nxt[q] = (lt < TM && row < g.M && q < g.KN) ? __ldg(g.nbr + row * g.KN + q) : -1;
        };
        if (nlocal > 0) fetch_nbr((int)blockIdx.x);
        for (int k = 0; k < nlocal; ++k) {
            const int tile = (int)blockIdx.x + k * (int)gridDim.x;
            const int m0 = tile * TM, s = k & 1;
            uint8_t* sA = sStage + s * kLayerStageBytes;
            if (k >= 2 && !fail)   // the MMAs of tile k - 2 read this stage
                fail = !mbar_wait(&bar_free[s], (uint32_t)(((k >> 1) - 1) & 1));
            // this tile's neighbour lists (every loader finished reading the last ones before the
            // previous loader_sync)
            if (lt < TM) {
                int cnt = 0;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    s_nb[lt * 8 + q] = nxt[q];
                    cnt += nxt[q] >= 0;
                }
                s_inv[lt] = cnt > 0 ? 1.f / (float)cnt : 0.f;
            }
            if (k + 1 < nlocal) fetch_nbr(tile + (int)gridDim.x);
            fail = loader_sync_or(fail);
            if (fail) break;
            stage_layer_tile(sA, g, m0, s_nb, s_inv, lt);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            loader_sync();
            if (lt == 0) {
                const int a = k & 1;
                if (k >= 2) fail = !mbar_wait(&bar_empty[a], (uint32_t)(((k >> 1) - 1) & 1));
                if (!fail) {
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t d = taddr + (uint32_t)(a * kLayerW);
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const uint32_t sa = smem_u32(sA + c * TM * TK * 2);
                        const uint32_t sb = smem_u32(sW + c * kLayerW * TK * 2);
#pragma unroll
                        for (int q = 0; q < TK / 16; ++q) {
                            const uint64_t ad = make_desc(sa + q * (TM / 8) * 256, 128, 256);
                            const uint64_t bd = make_desc(sb + q * (kLayerW / 8) * 256, 128, 256);
                            const uint32_t acc = (c > 0 || q > 0) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                    d),
                                "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                        }
                    }
                    tc_commit(&bar_free[s]);
                    tc_commit(&bar_full[a]);
                    s_last = k;
                }
            }
        }
        if (fail) atomicExch(&s_fail, 1);
    } else {
        // ---- epilogue ----
        const int we = warp - kLayerLoaders / 32;         // TMEM lane quarter = warp % 4
        for (int k = 0; k < nlocal; ++k) {
            const int tile = (int)blockIdx.x + k * (int)gridDim.x;
            const int a = k & 1;
            {   // the residual row is read after the accumulator: ask for it into L1 now
                const int64_t prow = (int64_t)tile * TM + 32 * we + lane;
                if (prow < g.M) {
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(g.h + prow * kLayerW));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(g.h + prow * kLayerW + 32));
                }
            }
            bool ok = mbar_wait(&bar_full[a], (uint32_t)((k >> 1) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) atomicExch(&s_fail, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int64_t row = (int64_t)tile * TM + 32 * we + lane;
            const uint32_t base = taddr + ((uint32_t)(32 * we) << 16) + (uint32_t)(a * kLayerW);
            uint32_t r0[32], r1[32];
            tmem_ld32(base, r0);
            tmem_ld32(base + 32, r1);
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_empty[a]);   // accumulator a may take tile k + 2
            if (row < g.M) {
                float dec[8];
#pragma unroll
                for (int o = 0; o < 8; ++o) dec[o] = (g.out && o < g.O) ? __ldg(g.bo + o) : 0.f;
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const uint32_t* r = half ? r1 : r0;
                    const int c0 = 32 * half;
                    float v[32], x[32];
#pragma unroll
                    for (int q = 0; q < 4; ++q) ld8(g.h + row * kLayerW + c0 + 8 * q, x + 8 * q);
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = __fadd_rn(silu(__uint_as_float(r[j]) + s_bias[c0 + j]), x[j]);
                    if (g.h_out)
#pragma unroll
                        for (int q = 0; q < 4; ++q) st8(g.h_out + row * kLayerW + c0 + 8 * q, v + 8 * q);
                    if (g.out) {
#pragma unroll
                        for (int o = 0; o < 8; ++o) {
                            if (o < g.O) {
#pragma unroll
                                for (int j = 0; j < 32; ++j)
                                    dec[o] = fmaf(v[j], s_wo[o * kLayerW + c0 + j], dec[o]);
                            }
                        }
                    }
                }
                if (g.out)
#pragma unroll
                    for (int o = 0; o < 8; ++o)
                        if (o < g.O) g.out[row * g.O + o] = dec[o];
            }
        }
    }
    // All MMAs of this CTA have completed once the last accumulator was read.  If a role gave up,
    // wait (bounded) for the commit of the last tile whose MMAs were issued (one thread issued them
    // in order, so they complete in order) before the tensor memory is released.
    __syncthreads();
    if (s_fail && threadIdx.x == 0) {
        const int k = s_last;
        if (k >= 0) mbar_wait(&bar_full[k & 1], (uint32_t)((k >> 1) & 1));
        if (g.err) atomicExch(g.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(128u));
}

// Training-path gather with the fused layer's arithmetic: out[i] = [bf16(h_i), bf16(mean_j h_j)]
// from the fp32 residual stream (mean = fp32 sum over the valid neighbours in table order times
// 1 / count); bf16 [N][128].  One thread per (cell, 8-channel unit).
__global__ void k_mp_gather_f32(const float* __restrict__ h, const int32_t* __restrict__ nbr, int N, int KN,
                                __nv_bfloat16* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * 8) return;
    const int i = (int)(t >> 3), u = (int)(t & 7);
    float own[8], acc[8];
    ld8(h + (int64_t)i * kLayerW + 8 * u, own);
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] = 0.f;
    int cnt = 0;
    for (int k = 0; k < KN; ++k) {
        const int j = __ldg(nbr + (int64_t)i * KN + k);
        cnt += j >= 0;
    }
    const float inv = cnt > 0 ? 1.f / (float)cnt : 0.f;
    for (int k = 0; k < KN && k < 8; ++k) {
        const int j = __ldg(nbr + (int64_t)i * KN + k);
        if (j < 0) continue;
        float v[8];
        ld8(h + (int64_t)j * kLayerW + 8 * u, v);
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[e] += v[e];
    }
    __align__(16) __nv_bfloat16 a[8], b[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        a[e] = __float2bfloat16(own[e]);
        b[e] = __float2bfloat16(acc[e] * inv);
    }
    *reinterpret_cast<uint4*>(out + (int64_t)i * 2 * kLayerW + 8 * u) = *reinterpret_cast<const uint4*>(a);
    *reinterpret_cast<uint4*>(out + (int64_t)i * 2 * kLayerW + kLayerW + 8 * u) = *reinterpret_cast<const uint4*>(b);
}

// Decoder on the fp32 stream with the fused layer's order: out[i][o] = b[o] + sum_c h[i][c] Wo[o][c]
// (fp32 fma over c ascending).
__global__ void k_decoder_f32(const float* __restrict__ h, const float* __restrict__ Wo, const float* __restrict__ bo,
                              int N, int O, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float acc[8];
#pragma unroll
    for (int o = 0; o < 8; ++o) acc[o] = o < O ? bo[o] : 0.f;
    for (int c0 = 0; c0 < kLayerW; c0 += 8) {
        float x[8];
        ld8(h + (int64_t)i * kLayerW + c0, x);
#pragma unroll
        for (int e = 0; e < 8; ++e)
#pragma unroll
            for (int o = 0; o < 8; ++o)
                if (o < O) acc[o] = fmaf(x[e], Wo[o * kLayerW + c0 + e], acc[o]);
    }
    for (int o = 0; o < O; ++o) out[(int64_t)i * O + o] = acc[o];
}

// Decoder backward on the fp32 stream: dh[i][c] = sum_o dOut[i][o] Wo[o][c];
// dWo[o][c] += sum_i dOut[i][o] h[i][c]; dbo[o] += sum_i dOut[i][o].
__global__ void k_decoder_back_f32(const float* __restrict__ h, const float* __restrict__ Wo,
                                   const float* __restrict__ dOut, int N, int O, float* __restrict__ dh,
                                   float* __restrict__ dWo, float* __restrict__ dbo) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * kLayerW) return;
    const int i = (int)(t / kLayerW), c = (int)(t % kLayerW);
    const float x = h[t];
    float v = 0.f;
    for (int o = 0; o < O; ++o) {
        const float d = dOut[(int64_t)i * O + o];
        v = fmaf(d, Wo[o * kLayerW + c], v);
        atomicAdd(dWo + o * kLayerW + c, d * x);
        if (c == 0) atomicAdd(dbo + o, d);
    }
    dh[t] = v;
}

}  // namespace corr
}  // namespace fvm

extern "C" int fvm_mp_layer(const float* h, const int32_t* nbr, int32_t M, int32_t KN, const void* Wt,
                            const float* bias, float* h_out, const float* Wo, const float* bo, int32_t O, float* out,
                            int32_t* err, void* stream) {
    if (!h || !nbr || !Wt || !bias || M <= 0 || KN <= 0 || KN > 8 || !err) return FVM_E_ARG;
    if (!h_out && !out) return FVM_E_ARG;
    if (out && (!Wo || !bo || O < 1 || O > 8)) return FVM_E_ARG;
    auto a32 = [](const void* p) { return ((uintptr_t)p & 31u) == 0; };
    if (!a32(h) || !a32(h_out) || (uintptr_t)Wt % 16) return FVM_E_ARG;
    if (h_out == h) return FVM_E_ARG;                    // the neighbours of later tiles read h
    static int sms = 0;
    static bool attr = false;
    if (!attr) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaFuncSetAttribute(corr::k_mp_layer, cudaFuncAttributeMaxDynamicSharedMemorySize, corr::kLayerSmem) !=
                cudaSuccess) {
            launch_status();
            return FVM_E_CUDA;
        }
        attr = true;
    }
    const int ntiles = (M + corr::TM - 1) / corr::TM;
    const unsigned grid = (unsigned)std::min(ntiles, sms);
    corr::LayerArgs g{h, nbr, M, KN, static_cast<const __nv_bfloat16*>(Wt), bias, h_out, Wo, bo, O, out, err};
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_mp_layer<<<grid, corr::kLayerThreads, corr::kLayerSmem, s>>>(g));
    return launch_status();
}

extern "C" int fvm_mp_gather_f32(const float* h, const int32_t* nbr, int32_t N, int32_t KN, void* out, void* stream) {
    if (!h || !nbr || !out || N <= 0 || KN <= 0 || KN > 8 || ((uintptr_t)h & 31u) || ((uintptr_t)out & 15u))
        return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_mp_gather_f32<<<corr::nblk((int64_t)N * 8, 256), 256, 0, s>>>(
                                     h, nbr, N, KN, static_cast<__nv_bfloat16*>(out)));
    return launch_status();
}

extern "C" int fvm_decoder_f32(const float* h, const float* Wo, const float* bo, int32_t N, int32_t O, float* out,
                               void* stream) {
    if (!h || !Wo || !bo || !out || N <= 0 || O < 1 || O > 8 || ((uintptr_t)h & 31u)) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_decoder_f32<<<corr::nblk(N, 256), 256, 0, s>>>(h, Wo, bo, N, O, out));
    return launch_status();
}

extern "C" int fvm_decoder_back_f32(const float* h, const float* Wo, const float* dOut, int32_t N, int32_t O,
                                    float* dh, float* dWo, float* dbo, void* stream) {
    if (!h || !Wo || !dOut || !dh || !dWo || !dbo || N <= 0 || O < 1 || O > 8) return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_decoder_back_f32<<<corr::nblk((int64_t)N * corr::kLayerW, 256), 256, 0, s>>>(
                                     h, Wo, dOut, N, O, dh, dWo, dbo));
    return launch_status();
}

// ------------------------------------------------------------------------------------------
// Acceptance checks of a corrector proposal, per case, in two launches (fvm_corrector_checks).
//   sums[c] (FP64, 3C + 4 slots): sum vol U, sum vol P, sum vol r0 (C each), sum vol |r0|^2,
//   sum vol |r1|^2, number of inadmissible cells of P (rho <= 0, internal energy <= 0 or not finite),
//   sum vol |P - U - k dt_c (r0 + r1) / 2|^2 (the proposal against the trapezoidal rule over the
//   window).  ok[c] = drift <= tol && |r1|^2 <= ratio^2 |r0|^2 && drift finite && no inadmissible
//   cell [&& trapezoid distance <= consistency * k dt_c |r0| when consistency > 0], with drift =
//   max over mass and energy of |sum vol P - (sum vol U + k dt_c sum vol r0)| / |sum vol U|.
// The reduction walks one contiguous chunk of cells per warp and flushes per case change (cells of
// a case are contiguous), as the conservation sums do; the verdict kernel clears the sums after
// reading them, so the pair can be replayed from a CUDA graph.
// ------------------------------------------------------------------------------------------
namespace fvm {
namespace corr {

template <int C>
__global__ void k_checks_reduce(const float* __restrict__ U, const float* __restrict__ P,
                                const float* __restrict__ r0, const float* __restrict__ r1,
                                const float* __restrict__ vol, const int32_t* __restrict__ cell_case, int N,
                                const float* __restrict__ dt, int k, double* __restrict__ sums) {
    constexpr int DIM = C - 2, NS = 3 * C + 4;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t chunk = (((int64_t)N + warps - 1) / warps + 31) & ~(int64_t)31;
    const int64_t beg = w * chunk, end = beg + chunk < N ? beg + chunk : (int64_t)N;
    int cur = -1;
    double acc[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) acc[q] = 0.0;
    auto flush = [&]() {
        if (cur < 0) return;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            double v = acc[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
            if (lane == 0) atomicAdd(sums + (int64_t)cur * NS + q, v);
            acc[q] = 0.0;
        }
    };
    for (int64_t i0 = beg; i0 < end; i0 += 32) {
        const int64_t i = i0 + lane;
        const bool live = i < end;
        const int cse = live ? __ldg(cell_case + i) : -1;
        double v[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) v[q] = 0.0;
        if (live) {
            const double vo = (double)__ldg(vol + i);
            float u[C], pp[C], a[C], b[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                u[c] = __ldg(U + i * C + c);
                pp[c] = __ldg(P + i * C + c);
                a[c] = __ldg(r0 + i * C + c);
                b[c] = __ldg(r1 + i * C + c);
            }
            const double half_kdt = 0.5 * (double)k * (double)__ldg(dt + cse);
            double n0 = 0.0, n1 = 0.0, e2 = 0.0;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                v[c] = vo * (double)u[c];
                v[C + c] = vo * (double)pp[c];
                v[2 * C + c] = vo * (double)a[c];
                n0 += vo * (double)(a[c] * a[c]);
                n1 += vo * (double)(b[c] * b[c]);
                const double e = ((double)pp[c] - (double)u[c]) - half_kdt * ((double)a[c] + (double)b[c]);
                e2 += vo * (e * e);
            }
            v[3 * C + 3] = e2;
            v[3 * C] = n0;
            v[3 * C + 1] = n1;
            const float rho = pp[DIM];
            float k2 = 0.f;
#pragma unroll
            for (int d = 0; d < DIM; ++d) k2 += pp[d] * pp[d];
            const float e_int = pp[DIM + 1] - 0.5f * k2 / rho;
            v[3 * C + 2] = (rho <= 0.f || e_int <= 0.f || !isfinite(e_int)) ? 1.0 : 0.0;
        }
        unsigned pending = __ballot_sync(full, live);
        while (pending) {
            const int lc = __shfl_sync(full, cse, __ffs(pending) - 1);
            if (lc != cur) {
                flush();
                cur = lc;
            }
            const bool mine = live && cse == lc;
            if (mine)
#pragma unroll
                for (int q = 0; q < NS; ++q) acc[q] += v[q];
            pending &= ~__ballot_sync(full, mine);
        }
    }
    flush();
}

__global__ void k_checks_verdict(double* __restrict__ sums, int n_cases, int C, const float* __restrict__ dt, int k,
                                 double tol, double ratio2, double consistency, uint8_t* __restrict__ ok,
                                 double* __restrict__ keep) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cases) return;
    const int NS = 3 * C + 4, DIM = C - 2;
    double* s = sums + (int64_t)c * NS;
    const double kdt = (double)k * (double)dt[c];
    double drift = 0.0;
    for (int q = DIM; q < DIM + 2; ++q) {
        const double m0 = s[q], mp = s[C + q], r = s[2 * C + q];
        const double d = fabs(mp - (m0 + kdt * r)) / fabs(m0);
        drift = (d > drift || isnan(d)) ? d : drift;
    }
    const bool near_trapezoid = consistency <= 0.0 || s[3 * C + 3] <= consistency * consistency * kdt * kdt * s[3 * C];
    ok[c] = (drift <= tol && s[3 * C + 1] <= ratio2 * s[3 * C] && isfinite(drift) && s[3 * C + 2] == 0.0 &&
             near_trapezoid) ? 1 : 0;
    for (int q = 0; q < NS; ++q) {
        if (keep) keep[(int64_t)c * NS + q] = s[q];
        s[q] = 0.0;
    }
}

}  // namespace corr
}  // namespace fvm

extern "C" int fvm_corrector_checks(const float* U, const float* P, const float* r0, const float* r1,
                                    const float* volumes, const int32_t* cell_case, int32_t N, int32_t C,
                                    int32_t n_cases, const float* dt, int32_t k, double drift_tol, double ratio,
                                    double consistency, double* sums, uint8_t* ok, double* keep, void* stream) {
    if (!U || !P || !r0 || !r1 || !volumes || !cell_case || !dt || !sums || !ok || N <= 0 || n_cases <= 0 ||
        (C != 4 && C != 5) || k < 1)
        return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess) {
            launch_status();
            return FVM_E_CUDA;
        }
    }
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(4LL * sms, ((int64_t)N + 255) / 256));
    if (C == 4)
        FVM_LAUNCH(KID_CORRECTOR, s, corr::k_checks_reduce<4><<<grid, 256, 0, s>>>(U, P, r0, r1, volumes, cell_case, N,
                                                                                    dt, k, sums));
    else
        FVM_LAUNCH(KID_CORRECTOR, s, corr::k_checks_reduce<5><<<grid, 256, 0, s>>>(U, P, r0, r1, volumes, cell_case, N,
                                                                                    dt, k, sums));
    int rc = launch_status();
    if (rc) return rc;
    FVM_LAUNCH(KID_CORRECTOR, s, corr::k_checks_verdict<<<(n_cases + 127) / 128, 128, 0, s>>>(
                                     sums, n_cases, C, dt, k, drift_tol, ratio * ratio, consistency, ok, keep));
    return launch_status();
}
