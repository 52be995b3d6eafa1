// Shared device helpers for the fvm_b200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fvm_b200.h"

namespace fvm {

constexpr int kBlock = 256;

// Returns FVM_OK or FVM_E_CUDA after a launch (records the CUDA error code).
int launch_status();

// Kernel identifiers reported by the profiling hooks (fvm_profile_*).
enum KernelId {
    KID_ELL_SPMV = 0, KID_ELL_SPMM = 1, KID_BC = 2, KID_CELL = 3, KID_FACE = 4, KID_DIV_STAGE = 5,
    KID_FINALIZE = 6, KID_STATE_TO_PRIMS = 7, KID_REDUCE_STATE = 8, KID_BATCH = 9, KID_CORRECTOR = 10,
    KID_FUSED = 11,
};

// When profiling is on, prof_begin/prof_end bracket a launch with CUDA events on its stream.
void prof_begin(int kid, cudaStream_t s);
void prof_end(cudaStream_t s);

// Launches of the stage kernels (boundary, cell, facet, divergence, finalisation) go through
// `launch`: with launch overlap on (fvm_set_launch_overlap, default on) each carries the
// programmatic-stream-serialisation attribute, so the next kernel of a stream (or of a CUDA graph)
// is launched while the previous one drains; every such kernel starts with `dependency_wait`
// (griddepcontrol.wait), which returns once the previous kernel has completed and its writes are
// visible, so results are unchanged.  A launch error is kept for launch_status().
extern int g_launch_overlap;
void note_launch_error(cudaError_t e);

__device__ __forceinline__ void dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_launch_overlap ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
    if (e != cudaSuccess) note_launch_error(e);
}

#define FVM_LAUNCH(kid, stream, ...)          \
    do {                                      \
        ::fvm::prof_begin((kid), (stream));   \
        __VA_ARGS__;                          \
        ::fvm::prof_end((stream));            \
    } while (0)

// Row loads/stores of C consecutive floats.  Rows of C = 4 floats are 16-byte aligned (all
// buffers come from cudaMalloc / torch and rows start at multiples of 16 bytes), so they use one
// vector access; C = 5 rows use scalar accesses, which a warp still coalesces into contiguous
// 32-byte sectors.
template <int C>
__device__ __forceinline__ void load_row(const float* __restrict__ p, float (&v)[C]) {
    if constexpr (C == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = __ldg(p + c);
    }
}

template <int C>
__device__ __forceinline__ void store_row(float* p, const float (&v)[C]) {
    if constexpr (C == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int c = 0; c < C; ++c) p[c] = v[c];
    }
}

// Block-wide sum of NV doubles; the result is valid in thread 0.  blockDim.x <= 1024.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* [32 * NV] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[warp * NV + k] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? smem[lane * NV + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
}

__device__ __forceinline__ double block_max(double v, double* smem /* [32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? smem[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    return v;
}

// Positive doubles order like their bit patterns, so an unsigned 64-bit atomicMax is a max.
__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace fvm
