// ELL sparse operators: y = A x (+ b), Y = A X (+ b).
//
// Replaces the Triton kernels of the reference (time_fvm/utils/ell_kernel.py:25-80 ell_spmm_kernel,
// :100-132 _ell_spmv_kernel) and their wrappers (:135-210).  Differences by design:
//  * ELL is slot-major (vals[k][row]) with int32 columns: a warp reading slot k of 32 consecutive
//    rows issues one 128-byte transaction for the values and one for the columns, where the
//    reference's row-major layout strides K * 4 (8 for int64) bytes between lanes;
//  * SpMM with few columns (B = 4 or 5 conserved variables) gives each thread a whole row and up to
//    8 columns, so no lanes are masked (the reference's BLOCK_B >= 16 masks >= 69 % of them);
//  * SpMV of a multi-column x is one launch, not one launch per column (ell_kernel.py:157-165);
//  * the bias is added in-kernel after the K-slot accumulation (same order as the reference);
//  * the slot loop is unrolled to a compile-time bound (K <= FVM_MAX_ELL_K = 16), so a row's
//    gathers are issued together instead of one dependent load chain per slot.
#include "fvm_common.cuh"

namespace fvm {

// Every kernel is templated on an upper bound KT of the slot count (4, 8 or 16) and unrolls the
// slot loop, so the values, columns and gathers of all slots of a row are in flight together (one
// dependent round trip per row instead of K); slots are summed in order k = 0, 1, ... as before.
template <int KT>
__global__ void __launch_bounds__(kBlock) k_ell_spmv(const float* __restrict__ vals,
                                                      const int32_t* __restrict__ cols, int64_t M,
                                                      int K, const float* __restrict__ x,
                                                      int64_t incx, const float* __restrict__ bias,
                                                      float* __restrict__ y, int64_t incy) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= M) return;
    float v[KT], xv[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        v[k] = 0.f;
        xv[k] = 0.f;
        if (k < K) {
            v[k] = __ldg(vals + k * M + r);
            xv[k] = __ldg(x + (int64_t)__ldg(cols + k * M + r) * incx);
        }
    }
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < KT; ++k)
        if (k < K) acc = fmaf(v[k], xv[k], acc);
    if (bias) acc += __ldg(bias + r);
    y[r * incy] = acc;
}

// One thread per (row, group of CB columns).
template <int KT, int CB>
__global__ void __launch_bounds__(kBlock) k_ell_spmm(const float* __restrict__ vals,
                                                      const int32_t* __restrict__ cols, int64_t M,
                                                      int K, const float* __restrict__ X,
                                                      int64_t ldx, int B,
                                                      const float* __restrict__ bias,
                                                      float* __restrict__ Y, int64_t ldy) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= M) return;
    const int c0 = blockIdx.y * CB;
    const int nb = min(CB, B - c0);
    float v[KT];
    int64_t xo[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        v[k] = k < K ? __ldg(vals + k * M + r) : 0.f;
        xo[k] = k < K ? (int64_t)__ldg(cols + k * M + r) * ldx + c0 : 0;
    }
    float acc[CB];
#pragma unroll
    for (int j = 0; j < CB; ++j) acc[j] = 0.f;
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        if (k >= K) break;
        float xr[CB];
#pragma unroll
        for (int j = 0; j < CB; ++j) xr[j] = j < nb ? __ldg(X + xo[k] + j) : 0.f;
#pragma unroll
        for (int j = 0; j < CB; ++j)
            if (j < nb) acc[j] = fmaf(v[k], xr[j], acc[j]);
    }
    float b = bias ? __ldg(bias + r) : 0.f;
    float* yr = Y + r * ldy + c0;
#pragma unroll
    for (int j = 0; j < CB; ++j)
        if (j < nb) yr[j] = bias ? acc[j] + b : acc[j];
}

// Specialisation for 4 contiguous, 16-byte aligned columns: one float4 gather per slot.
template <int KT>
__global__ void __launch_bounds__(kBlock) k_ell_spmm4(const float* __restrict__ vals,
                                                       const int32_t* __restrict__ cols, int64_t M,
                                                       int K, const float* __restrict__ X,
                                                       const float* __restrict__ bias,
                                                       float* __restrict__ Y) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= M) return;
    float v[KT], x[KT][4];
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        v[k] = 0.f;
#pragma unroll
        for (int j = 0; j < 4; ++j) x[k][j] = 0.f;
        if (k < K) {
            v[k] = __ldg(vals + k * M + r);
            load_row<4>(X + 4 * (int64_t)__ldg(cols + k * M + r), x[k]);
        }
    }
    float a[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < KT; ++k)
        if (k < K)
#pragma unroll
            for (int j = 0; j < 4; ++j) a[j] = fmaf(v[k], x[k][j], a[j]);
    if (bias) {
        const float b = __ldg(bias + r);
#pragma unroll
        for (int j = 0; j < 4; ++j) a[j] += b;
    }
    store_row<4>(Y + 4 * r, a);
}

}  // namespace fvm

#include <vector>

namespace fvm {
static thread_local int g_last_cuda_error = 0;

struct ProfState {
    bool on = false;
    int cap = 0, n = 0;
    bool overflow = false;
    std::vector<cudaEvent_t> ev;   // 2 per launch
    std::vector<int> ids;
};
static ProfState g_prof;

void prof_begin(int kid, cudaStream_t s) {
    if (!g_prof.on) return;
    if (g_prof.n >= g_prof.cap) {
        g_prof.overflow = true;
        return;
    }
    g_prof.ids[g_prof.n] = kid;
    cudaEventRecord(g_prof.ev[2 * g_prof.n], s);
}

void prof_end(cudaStream_t s) {
    if (!g_prof.on || g_prof.n >= g_prof.cap) return;
    cudaEventRecord(g_prof.ev[2 * g_prof.n + 1], s);
    ++g_prof.n;
}

int g_launch_overlap = 1;
static thread_local cudaError_t g_pending_launch_error = cudaSuccess;

void note_launch_error(cudaError_t e) {
    if (g_pending_launch_error == cudaSuccess) g_pending_launch_error = e;
}

int launch_status() {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = g_pending_launch_error;
    g_pending_launch_error = cudaSuccess;
    if (e != cudaSuccess) {
        g_last_cuda_error = (int)e;
        return FVM_E_CUDA;
    }
    return FVM_OK;
}
}  // namespace fvm

extern "C" int fvm_set_launch_overlap(int32_t on) {
    if (on != 0 && on != 1) return FVM_E_ARG;
    fvm::g_launch_overlap = on;
    return FVM_OK;
}

extern "C" int fvm_last_cuda_error(void) { return fvm::g_last_cuda_error; }

extern "C" int fvm_profile_start(int32_t capacity) {
    using fvm::g_prof;
    if (capacity <= 0 || g_prof.on) return FVM_E_ARG;
    if ((int)g_prof.ids.size() < capacity) {
        const size_t have = g_prof.ev.size();
        g_prof.ev.resize(2 * (size_t)capacity);
        for (size_t i = have; i < g_prof.ev.size(); ++i)
            if (cudaEventCreate(&g_prof.ev[i]) != cudaSuccess) return fvm::launch_status();
        g_prof.ids.resize(capacity);
    }
    g_prof.cap = capacity;
    g_prof.n = 0;
    g_prof.overflow = false;
    g_prof.on = true;
    return FVM_OK;
}

extern "C" int fvm_profile_stop(void) {
    using fvm::g_prof;
    g_prof.on = false;
    return g_prof.overflow ? FVM_E_ARG : g_prof.n;
}

extern "C" int fvm_profile_read(int32_t n, int32_t* ids, float* ms) {
    using fvm::g_prof;
    if (n < 0 || n > g_prof.n || !ids || !ms) return FVM_E_ARG;
    for (int i = 0; i < n; ++i) {
        ids[i] = g_prof.ids[i];
        if (cudaEventSynchronize(g_prof.ev[2 * i + 1]) != cudaSuccess ||
            cudaEventElapsedTime(&ms[i], g_prof.ev[2 * i], g_prof.ev[2 * i + 1]) != cudaSuccess) {
            fvm::launch_status();
            return FVM_E_CUDA;
        }
    }
    return n;
}

extern "C" const char* fvm_version(void) { return "fvm_b200 1.0 sm_100a"; }

using fvm::launch_status;

extern "C" int fvm_ell_spmv(const float* vals, const int32_t* cols, int64_t M, int32_t K,
                            const float* x, int64_t incx, const float* bias, float* y, int64_t incy,
                            void* stream) {
    if (M < 0 || K < 0 || (M > 0 && (!vals && K > 0)) || (M > 0 && (!x || !y))) return FVM_E_ARG;
    if (M == 0) return FVM_OK;
    if (K > FVM_MAX_ELL_K) return FVM_E_UNSUPPORTED;
    const int64_t grid = (M + fvm::kBlock - 1) / fvm::kBlock;
    cudaStream_t s = (cudaStream_t)stream;
#define FVM_SPMV(KT) FVM_LAUNCH(fvm::KID_ELL_SPMV, s, fvm::k_ell_spmv<KT><<<(unsigned)grid, fvm::kBlock, 0, s>>>( \
                                    vals, cols, M, K, x, incx, bias, y, incy))
    if (K <= 4) FVM_SPMV(4);
    else if (K <= 8) FVM_SPMV(8);
    else FVM_SPMV(16);
#undef FVM_SPMV
    return launch_status();
}

extern "C" int fvm_ell_spmm(const float* vals, const int32_t* cols, int64_t M, int32_t K,
                            const float* X, int64_t ldx, int32_t B, const float* bias, float* Y,
                            int64_t ldy, void* stream) {
    if (M < 0 || K < 0 || B < 0 || (M > 0 && B > 0 && (!X || !Y || (K > 0 && !vals))))
        return FVM_E_ARG;
    if (M == 0 || B == 0) return FVM_OK;
    const int64_t gx = (M + fvm::kBlock - 1) / fvm::kBlock;
    cudaStream_t s = (cudaStream_t)stream;
    if (K > FVM_MAX_ELL_K) return FVM_E_UNSUPPORTED;
    const bool aligned = ((uintptr_t)X % 16 == 0) && ((uintptr_t)Y % 16 == 0);
    if (B == 4 && ldx == 4 && ldy == 4 && aligned) {
#define FVM_SPMM4(KT) FVM_LAUNCH(fvm::KID_ELL_SPMM, s, fvm::k_ell_spmm4<KT><<<(unsigned)gx, fvm::kBlock, 0, s>>>( \
                                     vals, cols, M, K, X, bias, Y))
        if (K <= 4) FVM_SPMM4(4);
        else if (K <= 8) FVM_SPMM4(8);
        else FVM_SPMM4(16);
#undef FVM_SPMM4
    } else {
        const unsigned gy = (unsigned)((B + 7) / 8);
#define FVM_SPMM(KT) FVM_LAUNCH(fvm::KID_ELL_SPMM, s, fvm::k_ell_spmm<KT, 8><<<dim3((unsigned)gx, gy), fvm::kBlock, 0, s>>>( \
                                    vals, cols, M, K, X, ldx, B, bias, Y, ldy))
        if (K <= 4) FVM_SPMM(4);
        else if (K <= 8) FVM_SPMM(8);
        else FVM_SPMM(16);
#undef FVM_SPMM
    }
    return launch_status();
}
