// Fused finite-volume residual and explicit time-stepping kernels.
//
// One residual evaluation (FVMEquation.forward, time_fvm/fvm_equation.py:406-435) is three
// kernels (four with boundaries) instead of the reference's ~60 eager PyTorch ops:
//
//   k_bc        boundary facets: A_bc U + b_bc + A_corr grads_prev, then the characteristic BC
//               (facet_boundary.py:124-168, 418-512).  Each block recomputes the group mean of the
//               interior sound speed in the same order, so no grid-wide synchronisation is needed.
//   k_cell      per cell: LSQ gradient (G_mats spMM, facet_process.py:409-418), slope limiter
//               (facet_process.py:387-407, limiter.py) and the limited gradient
//               (FacetCalc.cell_grads, facet_process.py:345-346).
//   k_face      per facet: limited facet values of both sides, rebuilt from each cell's primitives
//               and limited gradient (U + grad_lim . r, the reference's addcmul(U, dU, phi) of
//               facet_process.py:405 with the limiter applied to the gradient), averaged gradients,
//               normal gradient (A_face_grad spMV) and non-orthogonal correction
//               (facet_process.py:362-385), EOS and stress (fvm_equation.py:62-187), advection +
//               pressure + viscous + heating + Kurganov-Tadmor fluxes (fvm_equation.py:199-368).
//   k_div_stage per cell: divergence (flux_mat spMM, fvm_equation.py:428-435) fused with the
//               Runge-Kutta / Adams stage combination, the conserved -> primitive conversion of
//               the next stage input (fvm_equation.py:35-44) and, on the last stage, the FP64
//               reductions for the adaptive step size (integrators.py:42-62), the CFL time step and
//               the conservation sums.
//
// All kernels are memory-bound gathers.  Every per-cell and per-facet table is one contiguous
// record, and every gathered row (primitives, limited gradients, fluxes) is padded to a 32-byte
// multiple (16 bytes for the 4-float rows of 2D), so a record or a gather is a few aligned 256-bit
// loads and never straddles more 32-byte sectors than it must.  k_cell, k_face and k_div_stage are
// persistent grid-stride loops over one wave of resident blocks that load the next item's gather
// indices one iteration ahead: a cell's or facet's gathers then leave together with its record,
// one dependent memory round trip per item instead of two.  Optionally (autotuned) each block also
// has the bulk-copy unit prefetch the record tile it will read a wave later into L2.  Rebuilding the
// facet values in k_face removes the reference's [F, 2, C] facet table (a scattered write plus a
// read per facet side).
#include <math.h>

#include <algorithm>

#include "fvm_common.cuh"

namespace fvm {

constexpr int kMaxBlock = 512;   // largest block size the autotuner may pick

struct Phys {
    float T_0, mu, mu_b, S, C_v, gamma, kappa, v_factor;
    float R, gR, inv_Cv, T0pS, T0sq;  // derived, rounded to float as the reference's scalars are
    float inv_T0, inv_T0sq;           // 1 / T_0 and 1 / T_0^2, for the facet kernel's transport terms
    int lim_p;
};

// Stage descriptor built on the host from a tableau.
struct StageArgs {
    int s;          // index of the increment computed by this stage (k[s] = dt * f)
    int store_k;    // write k[s] to memory (needed by a later combination)
    int final_;     // 1: combination is the new state (written to state); 0: next stage input
    int n_terms;    // combination U0 + sum_t coef[t] * k[idx[t]]
    int idx[FVM_MAX_STAGES];
    float coef[FVM_MAX_STAGES];
    int n_lo;       // embedded low-order combination (adaptive error estimate)
    int idx_lo[FVM_MAX_STAGES];
    float coef_lo[FVM_MAX_STAGES];
    int adaptive, cfl, cons;
};

// Compile-time layout of one dimension.
template <int DIM>
struct L {
    static constexpr int C = DIM + 2, K = DIM + 1, KG = DIM + 2;
    static constexpr int RS = FVM_ROW(DIM), GS = FVM_GROW(DIM);
    static constexpr int CR = FVM_CELL_REC(DIM), FR = FVM_FACE_REC(DIM), DR = FVM_DIV_REC;
    // compact cell record offsets: neighbour columns [KG - 1] (padded to 4, one 128-bit load),
    // weights [DIM][KG], displacements [K][DIM], eps
    static constexpr int GC = 0, GV = 4, DISP = GV + DIM * KG, EPS = DISP + K * DIM;
    static constexpr int SELF_SHIFT = 28;                 // own slot: bits 28..30 of the first column
    // face record offsets
    static constexpr int FA = 0, FB = 1, INVD = 2, SIZE = 3, NRM = 4, XO = 4 + DIM, RA = 4 + 2 * DIM,
                         RB = 4 + 3 * DIM;
    // limited-gradient row index of (spatial direction d, component comp)
    static __host__ __device__ __forceinline__ constexpr int gi(int d, int comp) {
        return comp == DIM ? DIM * (DIM + 1) + d : d * (DIM + 1) + (comp < DIM ? comp : DIM);
    }
    static_assert(EPS + 1 <= CR && RB + DIM <= FR && 2 * K <= DR, "record layout");
};

// N consecutive floats -> registers.  Rows whose width is a multiple of 8 floats start on 32-byte
// boundaries and move with 256-bit accesses (one L1 wavefront per lane-row instead of two); the
// others (4-float rows) with 128-bit accesses.
__device__ __forceinline__ void ld8_nc(const float* p, float* v) {
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}
__device__ __forceinline__ void ld8_cg(const float* p, float* v) {
    asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}
__device__ __forceinline__ void st8(float* p, const float* v) {
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
                 "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
}

template <int N>
__device__ __forceinline__ void ld_vec(const float* __restrict__ p, float (&v)[N]) {
    static_assert(N % 4 == 0, "row width");
    if constexpr (N % 8 == 0) {
#pragma unroll
        for (int q = 0; q < N / 8; ++q) ld8_nc(p + 8 * q, v + 8 * q);
    } else {
#pragma unroll
        for (int q = 0; q < N / 4; ++q) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(p) + q);
            v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
        }
    }
}
// Same, for data written by an earlier kernel of the same sequence (no read-only cache).
template <int N>
__device__ __forceinline__ void ld_vec_cg(const float* p, float (&v)[N]) {
    static_assert(N % 4 == 0, "row width");
    if constexpr (N % 8 == 0) {
#pragma unroll
        for (int q = 0; q < N / 8; ++q) ld8_cg(p + 8 * q, v + 8 * q);
    } else {
#pragma unroll
        for (int q = 0; q < N / 4; ++q) {
            const float4 t = __ldcg(reinterpret_cast<const float4*>(p) + q);
            v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
        }
    }
}
// Loads of arrays the same launch may have written (COH = true: the fused step kernel, whose
// phases read what other blocks wrote before a grid barrier) go through L2 (.cg); in the one-phase
// kernels those arrays are read-only for the launch and use the read-only path.
template <bool COH, int N>
__device__ __forceinline__ void ld_mut(const float* p, float (&v)[N]) {
    if constexpr (COH) ld_vec_cg<N>(p, v);
    else ld_vec<N>(p, v);
}
template <bool COH>
__device__ __forceinline__ float ld1_mut(const float* p) {
    if constexpr (COH) return __ldcg(p);
    else return __ldg(p);
}
template <int N>
__device__ __forceinline__ void st_vec(float* p, const float (&v)[N]) {
    static_assert(N % 4 == 0, "row width");
    if constexpr (N % 8 == 0) {
#pragma unroll
        for (int q = 0; q < N / 8; ++q) st8(p + 8 * q, v + 8 * q);
    } else {
#pragma unroll
        for (int q = 0; q < N / 4; ++q)
            reinterpret_cast<float4*>(p)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
}
__device__ __forceinline__ int as_int(float x) { return __float_as_int(x); }

// L2 prefetch of a contiguous byte range by the bulk-copy (TMA) unit: no shared memory, no
// completion to wait for.  Address and size must be multiples of 16 bytes.
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Thread 0 asks for the rows [tile * blockDim, (tile + 1) * blockDim) of a row-major array of
// `n_rows` rows of `row_floats` floats: the rows a block will read when it reaches `tile`.
// Issued one wave of blocks ahead, the record streams arrive in L2 while the current wave computes,
// and the blocks' own loads see L2 latency instead of DRAM latency.  The range is clamped to the
// array and rounded inward to 16-byte boundaries.
__device__ __forceinline__ void prefetch_tile(const float* base, int64_t n_rows, int row_floats, int64_t tile) {
    if (threadIdx.x != 0 || base == nullptr) return;
    const int64_t first = tile * blockDim.x;
    if (first >= n_rows) return;
    const int64_t last = min(first + (int64_t)blockDim.x, n_rows);
    int64_t b0 = first * row_floats * 4, b1 = last * row_floats * 4;
    b0 = (b0 + 15) & ~(int64_t)15;
    b1 &= ~(int64_t)15;
    if (b1 > b0) l2_prefetch(reinterpret_cast<const char*>(base) + b0, (uint32_t)(b1 - b0));
}

// Batched meshes with a case mask: is the case of item `idx` (looked up in `case_of`) active?
__device__ __forceinline__ bool case_on(const fvm_mesh_t& m, const int32_t* case_of, int idx) {
    return m.case_active == nullptr || m.case_active[__ldg(case_of + idx)] != 0;
}

// Whether a persistent loop over n items with `stride` threads checks the case of each next item
// before loading its record: only with a case mask and more than four items per thread.
__device__ __forceinline__ bool frozen_skip(const fvm_mesh_t& m, int n, int stride) {
    return m.case_active != nullptr && (int64_t)n > 4 * (int64_t)stride;
}

// One-ahead index loads of the persistent loops.  With `skip_frozen`, nothing is read for an item
// of a frozen case (case mask), so a masked-out case costs one case-id read per item; the check
// puts two dependent loads before the record load, so launches whose threads have only a few
// items (latency-bound) leave it off (see frozen_skip).
// The first 8 floats of facet f's record (its side codes, 1/d, |S|, normal, ...), fetched one
// iteration ahead by the facet loop: the codes come with it, so the record's head is read once.
// Rows of 16 floats (3D) start on 32-byte boundaries (one 256-bit load), rows of 12 (2D) on
// 16-byte ones (two 128-bit loads).  Items not loaded read as zeros (side codes 0, 0).
template <int DIM>
__device__ __forceinline__ void next_head(const fvm_mesh_t& m, int f, int nF, bool skip_frozen, float (&h)[8]) {
    const bool on = f < nF && (!skip_frozen || case_on(m, m.face_case, f));
    const float* r = m.face_rec + (int64_t)f * L<DIM>::FR;
    if (!on) {
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = 0.f;
    } else if constexpr (L<DIM>::FR % 8 == 0) {
        ld8_nc(r, h);
    } else {
        const float4 a = __ldg(reinterpret_cast<const float4*>(r)), b = __ldg(reinterpret_cast<const float4*>(r) + 1);
        h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w; h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
    }
}
// The rest of the record (floats 8 .. FR - 1).
template <int DIM>
__device__ __forceinline__ void record_tail(const fvm_mesh_t& m, int f, float (&rec)[L<DIM>::FR]) {
    constexpr int T = L<DIM>::FR - 8;
    static_assert(T == 8 || T == 4, "facet record width");
    float t[T];
    ld_vec<T>(m.face_rec + (int64_t)f * L<DIM>::FR + 8, t);
#pragma unroll
    for (int q = 0; q < T; ++q) rec[8 + q] = t[q];
}

// The KG stencil columns of cell i in slot order, from its compact record: the KG - 1 stored
// neighbour columns with the cell's own index inserted at its slot `own` (selects only, no
// indexing of register arrays by a runtime value).  Items not loaded get the column 0 everywhere.
template <int DIM>
__device__ __forceinline__ void next_cols(const fvm_mesh_t& m, int i, int NA, int* cols, int& own,
                                          bool skip_frozen) {
    using Ly = L<DIM>;
    const bool on = i < NA && (!skip_frozen || case_on(m, m.cell_case, i));
    static_assert(Ly::KG - 1 <= 4 && Ly::GC == 0, "columns in the record's first 16 bytes");
    const int4 q = on ? __ldg(reinterpret_cast<const int4*>(m.cell_rec + (int64_t)i * Ly::CR)) : make_int4(0, 0, 0, 0);
    const int nq[4] = {q.x, q.y, q.z, q.w};
    int nb[Ly::KG - 1];
#pragma unroll
    for (int k = 0; k < Ly::KG - 1; ++k) nb[k] = nq[k];
    own = (nb[0] >> Ly::SELF_SHIFT) & 7;
    nb[0] &= (1 << Ly::SELF_SHIFT) - 1;
    const int self = on ? i : 0;
#pragma unroll
    for (int k = 0; k < Ly::KG; ++k) {
        const int below = k < Ly::KG - 1 ? nb[k] : 0;
        const int above = k > 0 ? nb[k - 1] : 0;
        cols[k] = k < own ? below : (k == own ? self : above);
    }
}


// n / d with the fast-division intrinsic (__fdividef, within 2 ulp where 2^-126 <= |d| <= 2^126).
// Denominators outside [2^-100, 2^100] have both operands scaled by an exact power of two first,
// so the intrinsic always sees a denominator inside its range.  The limiter and facet kernels use
// it in place of IEEE division: their quotients then differ from correctly rounded ones by at most
// 2 ulp (relative 2.4e-7), far inside the 1e-5 parity bar, and a limiter evaluation costs about a
// third of its former instructions.
__device__ __forceinline__ float fast_div(float n, float d) {
    const float ad = fabsf(d);
    const float s = ad < 0x1p-100f ? 0x1p64f : (ad > 0x1p100f ? 0x1p-64f : 1.f);
    return __fdividef(n * s, d * s);
}

// ------------------------------------------------------------------------------------------
// Slope limiters (limiter.py:29-77).  delta: allowed range, dU: unlimited increment.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float limiter_phi(int p, float delta, float dU, float eps) {
    if (p == 4) {
        const float a = fabsf(delta), b = fabsf(dU), b2 = 2.f * b;
        const float a2 = a * a;
        const float a_eps = a2 * a2 + eps;
        const float S = b2 * fmaf(b2, b2 - a, a2);
        const float phi = fast_div(fmaf(a, S, a_eps), fmaf(b, delta * delta * delta + S, a_eps));
        return a < b2 ? phi : 1.f;
    }
    if (p == 1) {
        const float s = 2.f * ((dU > 0.f ? 1.f : 0.f) - 0.5f) * (fabsf(dU) + 1e-8f);
        return fminf(fmaxf(fast_div(delta, s), 0.f), 1.f);
    }
    if (p == 2) {
        return fast_div(delta * delta + eps + 2.f * delta * dU, delta * delta + 2.f * dU * dU + delta * dU + eps);
    }
    const float a = fabsf(delta), b = fabsf(dU);
    if (p == 3) {
        const float a_eps = a * a * a + eps, S = 4.f * b * b;
        const float phi = fast_div(a_eps + a * S, a_eps + b * (delta * delta + S));
        return a < 2.f * b ? phi : 1.f;
    }
    // p == 5
    const float a2 = a * a;
    const float a_eps = a2 * a2 * a + eps;
    const float S = 8.f * b * b * (a2 - 2.f * b * (a - b));
    const float d2 = delta * delta;
    const float phi = fast_div(a_eps + a * S, a_eps + b * (d2 * d2 + S));
    return a < 2.f * b ? phi : 1.f;
}

// ------------------------------------------------------------------------------------------
// k_bc: boundary facet values.
// ------------------------------------------------------------------------------------------
// Sum of the interior sound speed over characteristic facets [lo, hi): every caller uses the same
// thread -> element mapping and reduction tree, so batched and single-mesh runs agree bitwise.
template <int DIM, bool COH = false>
__device__ __forceinline__ double char_c_sum(const fvm_mesh_t& m, const Phys& p, const float* prims, int lo,
                                             int hi, double* red) {
    double acc = 0.0;
    for (int t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        const int cell = __ldg(m.ch_cell + t);
        acc += (double)sqrtf(p.gR * ld1_mut<COH>(prims + (int64_t)cell * L<DIM>::RS + DIM + 1));
    }
    double v[1] = {acc};
    block_sum<1>(v, red);
    return v[0];
}

// Batched meshes: per-case characteristic gating scale 10 / mean(c), one block per case.
template <int DIM, bool COH>
__device__ __forceinline__ void char_scale_case(const fvm_mesh_t& m, const Phys& p, const float* prims,
                                                double* red_out, int c) {
    __shared__ double red[32];
    if (m.case_active && !m.case_active[c]) return;
    const int lo = __ldg(m.ch_off + c), hi = __ldg(m.ch_off + c + 1);
    const double sum = char_c_sum<DIM, COH>(m, p, prims, lo, hi, red);
    if (threadIdx.x == 0)
        red_out[FVM_RED_DOUBLES + 8 * c + 6] = hi > lo ? (double)(10.0f / (float)(sum / (double)(hi - lo))) : 0.0;
    __syncthreads();
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_char_scale(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                        double* __restrict__ red_out) {
    dependency_wait();
    char_scale_case<DIM, false>(m, p, prims, red_out, blockIdx.x);
}

// Single mesh: the characteristic-BC scale 10 / mean(c) over the group (facet_boundary.py:427),
// recomputed identically by every block (block-wide; 0 when not needed).
template <int DIM, bool COH>
__device__ __forceinline__ float bc_block_scale(const fvm_mesh_t& m, const Phys& p, const float* prims) {
    __shared__ double red[32];
    __shared__ float s_scale;
    float scale = 0.f;
    if (m.n_char > 0 && m.n_cases == 0 && !m.char_scale_given) {
        const double sum = char_c_sum<DIM, COH>(m, p, prims, 0, m.n_char, red);
        if (threadIdx.x == 0) s_scale = 10.0f / (float)(sum / (double)m.n_char);
        __syncthreads();
        scale = s_scale;
        __syncthreads();
    }
    return scale;
}

// Boundary facet b's value (A_bc U + b_bc + A_corr grads_prev, then the characteristic BC).
template <int DIM, bool COH>
__device__ __forceinline__ void bc_item(const fvm_mesh_t& m, const Phys& p, const float* __restrict__ prims,
                                        const float* __restrict__ grads, const int32_t* __restrict__ has_grads,
                                        float* __restrict__ bcv, const double* __restrict__ wred, int b,
                                        float scale) {
    using Ly = L<DIM>;
    constexpr int C = Ly::C;
    if (m.n_cases > 0 && !case_on(m, m.bc_case, b)) return;
    if (m.n_cases > 0) scale = (float)__ldcg(wred + FVM_RED_DOUBLES + 8 * __ldg(m.bc_case + b) + 6);
    else if (m.char_scale_given) scale = (float)__ldcg(wred + FVM_RED_DOUBLES + 6);
    const int cell = __ldg(m.bc_cell + b);
    float U[Ly::RS];
    ld_mut<COH, Ly::RS>(prims + (int64_t)cell * Ly::RS, U);
    const bool prev = (COH ? __ldcg(has_grads) : *has_grads) != 0;
    float out[Ly::RS];
#pragma unroll
    for (int c = 0; c < Ly::RS; ++c) out[c] = 0.f;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const int kind = __ldg(m.bc_kind + b * C + c);
        float v = (kind == 2 ? U[c] : 0.f) + __ldg(m.bc_b + b * C + c);
        if (prev && kind == 2) {
            float corr = 0.f;
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                corr = fmaf(__ldg(m.bc_l + b * DIM + d), ld1_mut<COH>(grads + (int64_t)cell * Ly::GS + Ly::gi(d, c)),
                            corr);
            v += corr;
        }
        out[c] = v;
    }
    const int ch = __ldg(m.bc_char + b);
    if (ch >= 0) {
        // Characteristic BC (facet_boundary.py:436-512).
        float n[DIM], vt[DIM];
        float vn = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            n[d] = __ldg(m.ch_normal + ch * DIM + d);
            vn = fmaf(U[d], n[d], vn);
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) vt[d] = U[d] - vn * n[d];
        const float rho = U[DIM], T = U[DIM + 1];
        const float pr = p.R * rho * T;
        const float c = sqrtf(p.gR * T);
        const float drho = __ldg(m.ch_rho + ch) - rho;
        const float dvn = __ldg(m.ch_vn + ch) - vn;
        const float dp = __ldg(m.ch_p + ch) - pr;
        const float inv_c = 1.f / c;
        const float inv_c2 = inv_c * inv_c;
        const float h_dp = 0.5f * inv_c2 * dp;
        const float h_dvn = 0.5f * rho * inv_c * dvn;
        float x0 = -h_dvn + h_dp, x1 = drho - inv_c2 * dp, x2 = h_dvn + h_dp;
        const float g0 = 0.5f * (1.f - tanhf(scale * (vn - c)));
        const float g1 = 0.5f * (1.f - tanhf(scale * vn));
        const float g2 = 0.5f * (1.f - tanhf(scale * (vn + c)));
        x0 *= g0; x1 *= g1; x2 *= g2;
        const float cor = c / rho;
        const float rho_b = rho + (x0 + x1 + x2);
        const float vn_b = vn + (-cor * x0 + cor * x2);
        const float p_b = pr + (c * c) * (x0 + x2);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const float vtb = g1 * vt[d] + (1.f - g1) * __ldg(m.ch_vt + ch * DIM + d);
            out[d] = vn_b * n[d] + vtb;
        }
        out[DIM] = rho_b;
        out[DIM + 1] = p_b / (p.R * rho_b);
    }
    st_vec<Ly::RS>(bcv + (int64_t)b * Ly::RS, out);
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_bc(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                const float* __restrict__ grads,
                                                const int32_t* __restrict__ has_grads,
                                                float* __restrict__ bcv, const double* __restrict__ wred) {
    dependency_wait();
    const float scale = bc_block_scale<DIM, false>(m, p, prims);
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < m.n_bc) bc_item<DIM, false>(m, p, prims, grads, has_grads, bcv, wred, b, scale);
}

// ------------------------------------------------------------------------------------------
// k_cell: gradient, limiter, limited gradient.
// ------------------------------------------------------------------------------------------
// Persistent grid-stride loop (one wave of resident blocks): each thread loads the next cell's
// gradient-stencil columns one iteration ahead, so the neighbour gathers of a cell are issued at
// the top of its iteration together with its record, one memory round trip instead of two.
template <int DIM, bool COH>
__device__ __forceinline__ void cell_body(const fvm_mesh_t& m, const Phys& p, const float* __restrict__ prims,
                                          const float* __restrict__ bcv, float* __restrict__ grads,
                                          int32_t* __restrict__ has_grads, int waves) {
    using Ly = L<DIM>;
    constexpr int C = Ly::C, K = Ly::K, KG = Ly::KG, RS = Ly::RS;
    const int N = m.n_cells;                              // columns < N are cells (halo included)
    const int NA = m.n_owned > 0 ? m.n_owned : N;         // cells this launch updates: [lo, NA)
    const int lo = m.cell_lo;
    const int stride = gridDim.x * blockDim.x;
    int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) *has_grads = 1;
    const bool skip_frozen = frozen_skip(m, NA - lo, stride);
    int cols[KG], own;
    next_cols<DIM>(m, i, NA, cols, own, skip_frozen);
    for (int64_t tile = blockIdx.x; i < NA; i += stride, tile += gridDim.x) {
        if (waves > 0) prefetch_tile(m.cell_rec + (int64_t)lo * Ly::CR, NA - lo, Ly::CR, tile + (int64_t)waves * gridDim.x);
        if (m.case_active && !case_on(m, m.cell_case, i)) {
            next_cols<DIM>(m, i + stride, NA, cols, own, skip_frozen);
            continue;
        }
        float X[KG][RS];
#pragma unroll
        for (int k = 0; k < KG; ++k) {
            if (cols[k] < N) ld_mut<COH, RS>(prims + (int64_t)cols[k] * RS, X[k]);
            else ld_vec_cg<RS>(bcv + (int64_t)(cols[k] - N) * RS, X[k]);
        }
        // the cell's own primitives are its stencil row at slot `own` (no second load of the row)
        float U[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            U[c] = X[0][c];
#pragma unroll
            for (int k = 1; k < KG; ++k) U[c] = own == k ? X[k][c] : U[c];
        }
        float rec[Ly::CR];
        ld_vec<Ly::CR>(m.cell_rec + (int64_t)i * Ly::CR, rec);
        next_cols<DIM>(m, i + stride, NA, cols, own, skip_frozen);
        float g[DIM][C];
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int c = 0; c < C; ++c) g[d][c] = 0.f;
        float up[C], lo[C];
#pragma unroll
        for (int c = 0; c < C; ++c) up[c] = lo[c] = U[c];
#pragma unroll
        for (int k = 0; k < KG; ++k) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const float w = rec[Ly::GV + d * KG + k];
#pragma unroll
                for (int c = 0; c < C; ++c) g[d][c] = fmaf(w, X[k][c], g[d][c]);
            }
            // every slot of the reference's stencil is valid: the face neighbours and the cell
#pragma unroll
            for (int c = 0; c < C; ++c) {
                up[c] = fmaxf(up[c], X[k][c]);
                lo[c] = fminf(lo[c], X[k][c]);
            }
        }
        const float eps = rec[Ly::EPS];
        float phim[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            up[c] -= U[c];
            lo[c] -= U[c];
            phim[c] = INFINITY;
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                float du = g[0][c] * rec[Ly::DISP + j * DIM];
#pragma unroll
                for (int d = 1; d < DIM; ++d) du = fmaf(g[d][c], rec[Ly::DISP + j * DIM + d], du);
                const float num = du > 0.f ? up[c] : lo[c];
                phim[c] = fminf(phim[c], limiter_phi(p.lim_p, num, du, eps));
            }
        }
        float go[Ly::GS];
#pragma unroll
        for (int q = 0; q < Ly::GS; ++q) go[q] = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int c = 0; c < C; ++c) go[Ly::gi(d, c)] = g[d][c] * phim[c];
        st_vec<Ly::GS>(grads + (int64_t)i * Ly::GS, go);
    }
}

// Generic stencil width (kg > dim + 2, up to FVM_MAX_KG): record width FVM_CELL_REC_KG(DIM, kg),
// offsets from the runtime kg.  The gradient sums the valid slots in column order (the ELL row's
// order, as cell_body does); the limiter's bounds take the face neighbours only (their slots are in
// the record's meta, 4 bits each), which for the dim + 2 stencil are all valid slots but the cell
// itself.  Stencil columns stream through in groups of four, so registers do not grow with kg.
template <int DIM, bool COH>
__device__ __forceinline__ void cell_wide_body(const fvm_mesh_t& m, const Phys& p, const float* __restrict__ prims,
                                               const float* __restrict__ bcv, float* __restrict__ grads,
                                               int32_t* __restrict__ has_grads) {
    using Ly = L<DIM>;
    constexpr int C = Ly::C, K = Ly::K, RS = Ly::RS;
    const int kg = m.kg;
    const int CRW = FVM_CELL_REC_KG(DIM, kg);
    const int GC = DIM * kg, DISP = GC + kg, EPS = DISP + K * DIM, META = EPS + 1;
    const int N = m.n_cells;
    const int NA = m.n_owned > 0 ? m.n_owned : N;
    const int stride = gridDim.x * blockDim.x;
    int i = m.cell_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) *has_grads = 1;
    for (; i < NA; i += stride) {
        if (m.case_active && !case_on(m, m.cell_case, i)) continue;
        const float* rec = m.cell_rec + (int64_t)i * CRW;
        const int meta = as_int(__ldg(rec + META));
        const int nvalid = (meta >> 24) & 31;
        unsigned face = 0;
#pragma unroll
        for (int j = 0; j < K; ++j) face |= 1u << ((meta >> (4 * j)) & 15);
        float U[RS];
        ld_mut<COH, RS>(prims + (int64_t)i * RS, U);
        float g[DIM][C];
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int c = 0; c < C; ++c) g[d][c] = 0.f;
        float up[C], lo[C];
#pragma unroll
        for (int c = 0; c < C; ++c) up[c] = lo[c] = U[c];
        for (int k0 = 0; k0 < nvalid; k0 += 4) {
            float X[4][RS];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (k0 + q < nvalid) {
                    const int col = as_int(__ldg(rec + GC + k0 + q));
                    if (col < N) ld_mut<COH, RS>(prims + (int64_t)col * RS, X[q]);
                    else ld_vec_cg<RS>(bcv + (int64_t)(col - N) * RS, X[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int k = k0 + q;
                if (k >= nvalid) break;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const float w = __ldg(rec + d * kg + k);
#pragma unroll
                    for (int c = 0; c < C; ++c) g[d][c] = fmaf(w, X[q][c], g[d][c]);
                }
                if ((face >> k) & 1u) {
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        up[c] = fmaxf(up[c], X[q][c]);
                        lo[c] = fminf(lo[c], X[q][c]);
                    }
                }
            }
        }
        const float eps = __ldg(rec + EPS);
        float phim[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            up[c] -= U[c];
            lo[c] -= U[c];
            phim[c] = INFINITY;
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            float r[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) r[d] = __ldg(rec + DISP + j * DIM + d);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                float du = g[0][c] * r[0];
#pragma unroll
                for (int d = 1; d < DIM; ++d) du = fmaf(g[d][c], r[d], du);
                const float num = du > 0.f ? up[c] : lo[c];
                phim[c] = fminf(phim[c], limiter_phi(p.lim_p, num, du, eps));
            }
        }
        float go[Ly::GS];
#pragma unroll
        for (int q = 0; q < Ly::GS; ++q) go[q] = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int c = 0; c < C; ++c) go[Ly::gi(d, c)] = g[d][c] * phim[c];
        st_vec<Ly::GS>(grads + (int64_t)i * Ly::GS, go);
    }
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_cell_wide(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                       const float* __restrict__ bcv, float* __restrict__ grads,
                                                       int32_t* __restrict__ has_grads) {
    dependency_wait();
    cell_wide_body<DIM, false>(m, p, prims, bcv, grads, has_grads);
}

#ifndef FVM_CELL_MAXNREG
#define FVM_CELL_MAXNREG 96
#endif
// Register budget of the cell kernel: left to ptxas it settles on 64 with a spill in the loop;
// the budget trades resident warps against registers for the one-ahead loads and the unrolled
// stencil (chosen by timing on the 1.97 M-tet box).
template <int DIM>
__global__ void __maxnreg__(FVM_CELL_MAXNREG) k_cell(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                  const float* __restrict__ bcv, float* __restrict__ grads,
                                                  int32_t* __restrict__ has_grads, int waves) {
    dependency_wait();
    cell_body<DIM, false>(m, p, prims, bcv, grads, has_grads, waves);
}

// ------------------------------------------------------------------------------------------
// k_face: facet fluxes.
// ------------------------------------------------------------------------------------------
// One facet's flux F (the C components, padded with zeros to a row) from its record, side codes
// ca / cb and both sides' primitives P0, P1 and limited gradients G0, G1 (cell sides; a boundary
// side's value is read here): the arithmetic of every facet kernel, so all of them give the same
// bits.
template <int DIM>
__device__ __forceinline__ void face_eval(const fvm_mesh_t& m, const Phys& p, const float* __restrict__ bcv,
                                          int f, int ca, int cb, const float (&rec)[L<DIM>::FR],
                                          const float (&P0)[L<DIM>::RS], const float (&P1)[L<DIM>::RS],
                                          const float (&G0)[L<DIM>::GS], const float (&G1)[L<DIM>::GS],
                                          float (&F)[L<DIM>::RS]) {
    using Ly = L<DIM>;
    constexpr int C = Ly::C, NG = DIM + 1, RS = Ly::RS;
    const float size = rec[Ly::SIZE];
    const float inv_size = 1.f / size;
    float n[DIM], nh[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        n[d] = rec[Ly::NRM + d];
        nh[d] = n[d] * inv_size;
    }
    float UL[RS], UR[RS];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int code = s == 0 ? ca : cb;
        float* Us = s == 0 ? UL : UR;
        if (code >= 0) {
            const float* P = s == 0 ? P0 : P1;
            const float* G = s == 0 ? G0 : G1;
            const int roff = s == 0 ? Ly::RA : Ly::RB;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                float acc = G[Ly::gi(0, c)] * rec[roff];
#pragma unroll
                for (int d = 1; d < DIM; ++d) acc = fmaf(G[Ly::gi(d, c)], rec[roff + d], acc);
                Us[c] = P[c] + acc;
            }
        } else {
            float B[RS];
            ld_vec_cg<RS>(bcv + (int64_t)(-1 - code) * RS, B);
#pragma unroll
            for (int c = 0; c < C; ++c) Us[c] = B[c];
        }
    }
    // Facet-averaged limited gradients of (V, T): gls[d][k] (facet_process.py:362-371).
    float gls[DIM][NG];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
        for (int k = 0; k < NG; ++k) gls[d][k] = (G0[d * NG + k] + G1[d * NG + k]) / 2.f;
    // Normal gradient (A_face_grad row, facet_process.py:420-450).
    float dn[NG];
    if (ca >= 0 && cb >= 0) {
        // The row's two products are summed in the order of the mesh's cell numbering (ascending
        // ELL columns); the record's sign of 1/d says whether side 0 comes first, so a renumbered
        // part of the mesh sums them in the same order as the whole mesh.
        const float ws = rec[Ly::INVD];
        const float w = fabsf(ws);
        const bool side0_first = ws > 0.f;
#pragma unroll
        for (int k = 0; k < NG; ++k) {
            const int comp = k < DIM ? k : DIM + 1;
            const float x0 = P0[comp], x1 = P1[comp];
            dn[k] = side0_first ? fmaf(w, x1, (-w) * x0) : fmaf(-w, x0, w * x1);
        }
    } else {
        const int b = ca < 0 ? -1 - ca : -1 - cb;
#pragma unroll
        for (int k = 0; k < NG; ++k) {
            const int comp = k < DIM ? k : DIM + 1;
            dn[k] = __ldg(m.bc_ga + b * C + comp) * P0[comp] + __ldg(m.bc_gb + b * C + comp);
        }
    }
    // Non-orthogonal correction (facet_process.py:377-385).
    float dFdn[NG], gF[DIM][NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) {
        float sx = gls[0][k] * rec[Ly::XO], sn = gls[0][k] * nh[0];
#pragma unroll
        for (int d = 1; d < DIM; ++d) {
            sx = fmaf(gls[d][k], rec[Ly::XO + d], sx);
            sn = fmaf(gls[d][k], nh[d], sn);
        }
        dFdn[k] = dn[k] - sx;
        const float corr = dFdn[k] - sn;
#pragma unroll
        for (int d = 0; d < DIM; ++d) gF[d][k] = fmaf(corr, nh[d], gls[d][k]);
    }
    const float grad_T_n = dFdn[DIM];

    // Side quantities.
    float mom[2][DIM], rho[2], T[2], Q[2], P[2], cs[2], phi[2], vm2[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const float* Us = s == 0 ? UL : UR;
        rho[s] = Us[DIM];
        T[s] = Us[DIM + 1];
        float v2 = 0.f, ph = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            mom[s][d] = Us[d] * rho[s];
            v2 = fmaf(Us[d], Us[d], v2);
            ph = fmaf(Us[d], n[d], ph);
        }
        vm2[s] = v2;
        phi[s] = ph;
        Q[s] = rho[s] * (p.C_v * T[s] + 0.5f * v2);
        P[s] = p.R * rho[s] * T[s];
        cs[s] = sqrtf(p.gR * T[s]);
    }
    // Stress (fvm_equation.py:101-120, 149-170).  I1 = D00 + D11 also in 3D, as in the reference.
    const float Tm = (T[0] + T[1]) / 2.f;
    float mu0 = p.mu, mub0 = p.mu_b, kappa = p.kappa;
    if (m.n_cases > 0) {
        const int cs_ = __ldg(m.face_case + f);
        mu0 = __ldg(m.case_mu + cs_);
        mub0 = __ldg(m.case_mu_b + cs_);
        kappa = __ldg(m.case_kappa + cs_);
    }
    float D[DIM][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int c = 0; c < DIM; ++c) D[a][c] = 0.5f * (gF[a][c] + gF[c][a]);
    const float I1 = D[0][0] + D[1][1];
    // Sutherland: mu0 (Tm / T_0)^1.5 (T_0 + S) / (Tm + S), the power as q sqrt(q)
    const float q = Tm * p.inv_T0;
    const float mu = fast_div(mu0 * (q * sqrtf(q)) * p.T0pS, Tm + p.S);
    const float mub = mub0 * (Tm * Tm) * p.inv_T0sq;
    const float a0 = -mub * I1, a1 = -2.f * mu;
    float tau[DIM][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int c = 0; c < DIM; ++c) tau[a][c] = (a == c ? a0 : 0.f) + a1 * D[a][c];

#pragma unroll
    for (int c = 0; c < RS; ++c) F[c] = 0.f;
    // Advection (fvm_equation.py:210-231)
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[d] = (mom[0][d] * phi[0] + mom[1][d] * phi[1]) / 2.f;
    F[DIM] = (rho[0] * phi[0] + rho[1] * phi[1]) / 2.f;
    F[DIM + 1] = ((Q[0] + P[0]) * phi[0] + (Q[1] + P[1]) * phi[1]) / 2.f;
    // Pressure (fvm_equation.py:309-321)
    const float Pm = (P[0] + P[1]) / 2.f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[d] += Pm * n[d];
    // Viscous force (fvm_equation.py:246-257)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
        float s = tau[0][c] * n[0];
#pragma unroll
        for (int a = 1; a < DIM; ++a) s = fmaf(tau[a][c], n[a], s);
        F[c] += s;
    }
    // Heating and conduction (fvm_equation.py:272-294)
    float heat = 0.f;
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            const float Vm = (UL[c] + UR[c]) / 2.f;
            heat = fmaf(tau[a][c] * Vm, n[a], heat);
        }
    heat = fmaf(-kappa * grad_T_n, size, heat);
    F[DIM + 1] += heat;
    // Kurganov-Tadmor diffusion (fvm_equation.py:337-368)
    const float vmax = fmaxf(sqrtf(vm2[0]), sqrtf(vm2[1]));
    const float cmax = fmaxf(cs[0], cs[1]);
    const float M = fabsf(fast_div(vmax, cmax + 1e-8f));
    const float vf = fminf(fmaxf(M, p.v_factor), 1.f);
    const float a_vel = vf * cmax + vmax, a_oth = cmax + vmax;
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[d] += 0.5f * (a_vel * (mom[0][d] - mom[1][d])) * size;
    F[DIM] += 0.5f * (a_oth * (rho[0] - rho[1])) * size;
    F[DIM + 1] += 0.5f * (a_oth * (Q[0] - Q[1])) * size;
}

template <int DIM, bool COH>
__device__ __forceinline__ void face_body(const fvm_mesh_t& m, const Phys& p, const float* __restrict__ prims,
                                          const float* __restrict__ bcv, const float* __restrict__ grads,
                                          float* __restrict__ flux, int waves) {
    using Ly = L<DIM>;
    constexpr int RS = Ly::RS, GS = Ly::GS;
    const int nF = m.n_facets;                            // facets this launch evaluates: [lo, nF)
    const int lo = m.facet_lo;
    const int stride = gridDim.x * blockDim.x;
    int f = lo + blockIdx.x * blockDim.x + threadIdx.x;
    const bool skip_frozen = frozen_skip(m, nF - lo, stride);
    float head[8];
    next_head<DIM>(m, f, nF, skip_frozen, head);
    for (int64_t tile = blockIdx.x; f < nF; f += stride, tile += gridDim.x) {
    if (waves > 0) prefetch_tile(m.face_rec + (int64_t)lo * Ly::FR, nF - lo, Ly::FR, tile + (int64_t)waves * gridDim.x);
    const int ca = as_int(head[Ly::FA]), cb = as_int(head[Ly::FB]);
    if (m.case_active && !case_on(m, m.face_case, f)) {
        next_head<DIM>(m, f + stride, nF, skip_frozen, head);
        continue;
    }
    // Both sides: primitives and limited gradient of the cell(s); a boundary side (code < 0) takes
    // the boundary value, and its gradient is the interior cell's (facet_process.py:364-368).
    const int cell0 = ca >= 0 ? ca : cb;
    const int cell1 = cb >= 0 ? cb : ca;
    float P0[RS], P1[RS], G0[GS], G1[GS];
    ld_mut<COH, RS>(prims + (int64_t)cell0 * RS, P0);
    ld_mut<COH, RS>(prims + (int64_t)cell1 * RS, P1);
    ld_vec_cg<GS>(grads + (int64_t)cell0 * GS, G0);
    ld_vec_cg<GS>(grads + (int64_t)cell1 * GS, G1);
    float rec[Ly::FR];
#pragma unroll
    for (int q = 0; q < 8; ++q) rec[q] = head[q];
    record_tail<DIM>(m, f, rec);
    next_head<DIM>(m, f + stride, nF, skip_frozen, head);
    float F[RS];
    face_eval<DIM>(m, p, bcv, f, ca, cb, rec, P0, P1, G0, G1, F);
    st_vec<RS>(flux + (int64_t)f * RS, F);
    }
}

// Facet records staged by the bulk-copy unit.  Each block walks tiles of blockDim.x facets; thread
// 0 has the next tile's records (one contiguous range) copied into the other half of a two-stage
// shared-memory ring with cp.async.bulk, completion counted on that stage's mbarrier, while the
// block works on the current tile -- so the records (half the facet kernel's DRAM bytes) leave the
// per-thread load path and its registers, and each thread issues its side gathers as soon as the
// tile's barrier completes.  Waits are bounded: a thread whose wait gives up reads its record from
// global memory instead (same values), and after any such wait the block stops staging and reads
// every later record from global memory; before the block exits it waits (bounded) for copies still
// in flight.  Bitwise the same results as k_face (face_eval).
constexpr long long kStageWaitLimit = 1LL << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done = 0;
    for (long long it = 0; it < kStageWaitLimit && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred q;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
    }
    return done != 0;
}
__device__ __forceinline__ void stage_copy(float* dst, const float* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

template <int DIM>
__global__ void __launch_bounds__(kMaxBlock) k_face_staged(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                         const float* __restrict__ bcv,
                                                         const float* __restrict__ grads, float* __restrict__ flux) {
    dependency_wait();
    using Ly = L<DIM>;
    constexpr int RS = Ly::RS, GS = Ly::GS, FR = Ly::FR;
    extern __shared__ __align__(128) float s_rec[];       // [2][blockDim.x][FR]
    __shared__ __align__(8) uint64_t bar[2];
    const int B = blockDim.x;
    const int lo = m.facet_lo, nF = m.n_facets;
    const int64_t n = (int64_t)nF - lo;
    const int64_t ntiles = (n + B - 1) / B;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int64_t tile, int st) {
        const int64_t first = (int64_t)lo + tile * B;
        const int64_t rows = min((int64_t)B, (int64_t)nF - first);
        stage_copy(s_rec + (int64_t)st * B * FR, m.face_rec + first * FR, (uint32_t)(rows * FR * 4), &bar[st]);
    };
    bool staged = true;
    int issued_last = -1;                                  // local index of the last tile copied (thread 0)
    if (threadIdx.x == 0 && blockIdx.x < ntiles) {
        issue(blockIdx.x, 0);
        issued_last = 0;
    }
    int j = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++j) {
        const int st = j & 1;
        if (threadIdx.x == 0 && staged && tile + gridDim.x < ntiles) {
            issue(tile + gridDim.x, st ^ 1);               // that stage was last read before the previous sync
            issued_last = j + 1;
        }
        const bool ok = staged && stage_wait(&bar[st], (uint32_t)((j >> 1) & 1));
        const int64_t f = (int64_t)lo + tile * B + threadIdx.x;
        if (f < nF && !(m.case_active && !case_on(m, m.face_case, (int)f))) {
            float rec[FR];
            if (ok) {
                const float* r = s_rec + ((int64_t)st * B + threadIdx.x) * FR;
#pragma unroll
                for (int q = 0; q < FR; q += 4) {
                    const float4 t = *reinterpret_cast<const float4*>(r + q);
                    rec[q] = t.x; rec[q + 1] = t.y; rec[q + 2] = t.z; rec[q + 3] = t.w;
                }
            } else {
                ld_vec<FR>(m.face_rec + f * FR, rec);
            }
            const int ca = as_int(rec[Ly::FA]), cb = as_int(rec[Ly::FB]);
            const int cell0 = ca >= 0 ? ca : cb;
            const int cell1 = cb >= 0 ? cb : ca;
            float P0[RS], P1[RS], G0[GS], G1[GS];
            ld_vec<RS>(prims + (int64_t)cell0 * RS, P0);
            ld_vec<RS>(prims + (int64_t)cell1 * RS, P1);
            ld_vec_cg<GS>(grads + (int64_t)cell0 * GS, G0);
            ld_vec_cg<GS>(grads + (int64_t)cell1 * GS, G1);
            float F[RS];
            face_eval<DIM>(m, p, bcv, (int)f, ca, cb, rec, P0, P1, G0, G1, F);
            st_vec<RS>(flux + f * RS, F);
        }
        staged = staged && !__syncthreads_or(!ok);
    }
    // copies that may still be in flight after a wait gave up: wait for them (bounded) before the
    // block's shared memory is released
    if (threadIdx.x == 0 && !staged) {
        for (int k = max(0, issued_last - 1); k <= issued_last; ++k) stage_wait(&bar[k & 1], (uint32_t)((k >> 1) & 1));
    }
}

// Register budget of the facet kernel: by default whatever the compiler picks for 512-thread
// blocks; FVM_FACE_MAXNREG caps it (fewer registers per thread, more resident warps).
#ifdef FVM_FACE_MAXNREG
#define FVM_FACE_BOUNDS __maxnreg__(FVM_FACE_MAXNREG)
#else
#define FVM_FACE_BOUNDS __launch_bounds__(kMaxBlock)
#endif
template <int DIM>
__global__ void FVM_FACE_BOUNDS k_face(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                  const float* __restrict__ bcv,
                                                  const float* __restrict__ grads, float* __restrict__ flux,
                                                  int waves) {
    dependency_wait();
    face_body<DIM, false>(m, p, prims, bcv, grads, flux, waves);
}

// ------------------------------------------------------------------------------------------
// k_face_div: owner-computes residual (divergence-kernel variant 1, residual evaluations only).
// ------------------------------------------------------------------------------------------
// dU/dt of each cell from its own facets' fluxes, with no flux array: lanes 4q .. 4q + 3 of a warp
// own cell q's facet slots 0 .. K - 1 (the fourth lane idles in 2D); each evaluates its facet with
// face_eval, and the group's first lane sums the slots in order k = 0, 1, ... with the fused
// multiply-adds of k_div_stage, so dU/dt is bitwise that of k_face followed by k_div_stage.  Every
// interior facet is evaluated twice (once from each side) in exchange for the flux array's write,
// its gathered re-read and one launch.  Whole meshes only (no cell or facet sub-range).
template <int DIM>
__global__ void __launch_bounds__(kMaxBlock) k_face_div(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                      const float* __restrict__ bcv,
                                                      const float* __restrict__ grads, float* __restrict__ dudt) {
    dependency_wait();
    using Ly = L<DIM>;
    constexpr int C = Ly::C, RS = Ly::RS, GS = Ly::GS, FR = Ly::FR, K = Ly::K;
    static_assert(K <= 4, "four lanes per cell");
    const unsigned full = 0xffffffffu;
    const int NA = m.n_owned > 0 ? m.n_owned : m.n_cells;
    const int lane = threadIdx.x & 31, k = lane & 3, base = lane & ~3;
    const int64_t step = ((int64_t)gridDim.x * blockDim.x) >> 2;
    // warp-uniform loop: the warp's first cell decides, so every lane reaches the shuffles
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 2; i - (lane >> 2) < NA; i += step) {
        const bool cell_on = i < NA && (m.case_active == nullptr || case_on(m, m.cell_case, (int)i));
        const bool live = cell_on && k < K && k < m.kf;
        float F[RS], w = 0.f;
#pragma unroll
        for (int c = 0; c < RS; ++c) F[c] = 0.f;
        if (live) {
            const float* drec = m.div_rec + i * Ly::DR;
            w = __ldg(drec + k);
            const int f = as_int(__ldg(drec + K + k));
            float rec[FR];
            ld_vec<FR>(m.face_rec + (int64_t)f * FR, rec);
            const int ca = as_int(rec[Ly::FA]), cb = as_int(rec[Ly::FB]);
            const int cell0 = ca >= 0 ? ca : cb;
            const int cell1 = cb >= 0 ? cb : ca;
            float P0[RS], P1[RS], G0[GS], G1[GS];
            ld_vec<RS>(prims + (int64_t)cell0 * RS, P0);
            ld_vec<RS>(prims + (int64_t)cell1 * RS, P1);
            ld_vec_cg<GS>(grads + (int64_t)cell0 * GS, G0);
            ld_vec_cg<GS>(grads + (int64_t)cell1 * GS, G1);
            face_eval<DIM>(m, p, bcv, f, ca, cb, rec, P0, P1, G0, G1, F);
        }
        float r[C];
#pragma unroll
        for (int c = 0; c < C; ++c) r[c] = 0.f;
#pragma unroll
        for (int s = 0; s < K; ++s) {
            const float ws = __shfl_sync(full, w, base + s);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float fs = __shfl_sync(full, F[c], base + s);
                if (s < m.kf) r[c] = fmaf(ws, fs, r[c]);
            }
        }
        if (cell_on && k == 0)
#pragma unroll
            for (int c = 0; c < C; ++c) dudt[i * C + c] = r[c];
    }
}

// Both sides' limited facet values [F][2][C] (the reference's U_face_all, facet_process.py:349-354),
// rebuilt exactly as face_body rebuilds them: a cell side is U + sum_d grad_lim[d] r[d], a boundary
// side is the boundary value.  On demand only (the residual never stores them).
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_facet_values(fvm_mesh_t m, const float* __restrict__ prims,
                                                          const float* __restrict__ bcv,
                                                          const float* __restrict__ grads, float* __restrict__ out) {
    using Ly = L<DIM>;
    constexpr int C = Ly::C, RS = Ly::RS, GS = Ly::GS;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.n_facets) return;
    float rec[Ly::FR];
    ld_vec<Ly::FR>(m.face_rec + (int64_t)f * Ly::FR, rec);
    const int code[2] = {as_int(rec[Ly::FA]), as_int(rec[Ly::FB])};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        float v[C];
        if (code[s] >= 0) {
            float P[RS], G[GS];
            ld_vec<RS>(prims + (int64_t)code[s] * RS, P);
            ld_vec<GS>(grads + (int64_t)code[s] * GS, G);
            const int roff = s == 0 ? Ly::RA : Ly::RB;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                float acc = G[Ly::gi(0, c)] * rec[roff];
#pragma unroll
                for (int d = 1; d < DIM; ++d) acc = fmaf(G[Ly::gi(d, c)], rec[roff + d], acc);
                v[c] = P[c] + acc;
            }
        } else {
            float B[RS];
            ld_vec<RS>(bcv + (int64_t)(-1 - code[s]) * RS, B);
#pragma unroll
            for (int c = 0; c < C; ++c) v[c] = B[c];
        }
#pragma unroll
        for (int c = 0; c < C; ++c) out[((int64_t)f * 2 + s) * C + c] = v[c];
    }
}

// ------------------------------------------------------------------------------------------
// k_div_stage: divergence + stage combination.
// ------------------------------------------------------------------------------------------
template <int C, int RS>
__device__ __forceinline__ void state_to_prim(const float* U, float inv_Cv, float (&P)[RS]) {
    constexpr int DIM = C - 2;
    const float rho = U[DIM];
    float v2 = 0.f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        P[d] = U[d] / rho;
        v2 = fmaf(P[d], P[d], v2);
    }
    P[DIM] = rho;
    P[DIM + 1] = inv_Cv * (U[DIM + 1] / rho - 0.5f * v2);
#pragma unroll
    for (int c = C; c < RS; ++c) P[c] = 0.f;
}

template <int C>
__device__ __forceinline__ void load_state(const float* p, float (&v)[C]) {
#pragma unroll
    for (int c = 0; c < C; ++c) v[c] = __ldcg(p + c);
}
template <int C>
__device__ __forceinline__ void store_state(float* p, const float (&v)[C]) {
#pragma unroll
    for (int c = 0; c < C; ++c) p[c] = v[c];
}

// Speed scale inv_h (|u| + c) of a conserved state, FP64 (CFL time step).
template <int DIM>
__device__ __forceinline__ double cfl_speed(const fvm_mesh_t& m, const Phys& p, const float* U, int i) {
    double v2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) v2 += (double)U[d] / U[DIM] * ((double)U[d] / U[DIM]);
    const double T = ((double)U[DIM + 1] / U[DIM] - 0.5 * v2) / (double)p.C_v;
    return __ldg(m.inv_h + i) * (sqrt(v2) + sqrt((double)p.gamma * (double)p.R * fmax(T, 0.0)));
}

// Batched meshes: per-case reductions of one item per lane, warp-level when the warp's live lanes
// share a case, per-lane atomics otherwise (all lanes of the warp must call it).
template <int DIM>
__device__ __forceinline__ void reduce_batched_item(const fvm_mesh_t& m, const Phys& p, const float* U, bool live,
                                                    int i, int cse, bool want_cons, bool want_cfl, double* red) {
    constexpr int C = DIM + 2;
    const int lane = threadIdx.x & 31;
    const int c0 = __shfl_sync(0xffffffffu, cse, 0);
    const bool uniform = __all_sync(0xffffffffu, !live || cse == c0);
    double* slot = red + FVM_RED_DOUBLES + 8 * cse;
    if (want_cfl) {
        double sp = live ? cfl_speed<DIM>(m, p, U, i) : 0.0;
        if (uniform) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sp = fmax(sp, __shfl_down_sync(0xffffffffu, sp, o));
            if (lane == 0 && sp > 0.0) atomic_max_pos(red + FVM_RED_DOUBLES + 8 * c0, sp);
        } else if (live) {
            atomic_max_pos(slot, sp);
        }
    }
    if (want_cons) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            double v = live ? __ldg(m.volumes + i) * (double)U[c] : 0.0;
            if (uniform) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) atomicAdd(red + FVM_RED_DOUBLES + 8 * c0 + 1 + c, v);
            } else if (live) {
                atomicAdd(slot + 1 + c, v);
            }
        }
    }
}

// What one k_div_stage launch does after the divergence.
enum DivMode { DIV_RESIDUAL = 0, DIV_STAGE = 1, DIV_FINAL = 2, DIV_FINAL_ADAPT = 3 };

// Persistent grid-stride loop, warp-uniform (every lane of a warp runs the same iterations, so the
// batched reductions may shuffle): each thread loads the next cell's divergence record one iteration
// ahead, so the flux gathers of a cell start at the top of its iteration.  Single-mesh reductions
// are accumulated per thread and combined once per block after the loop.
template <int DIM, int MODE, bool COH>
__device__ __forceinline__ void div_body(const fvm_mesh_t& m, const Phys& p, const float* __restrict__ flux,
                                         const StageArgs& a, float* __restrict__ state, float* __restrict__ prims,
                                         float* __restrict__ kbuf, const float* __restrict__ dt,
                                         double* __restrict__ red, float* __restrict__ dudt, int waves) {
    using Ly = L<DIM>;
    constexpr int C = Ly::C, RS = Ly::RS;
    constexpr bool FINAL = MODE >= DIV_FINAL, ADAPT = MODE == DIV_FINAL_ADAPT;
    const int N = m.n_cells;                              // row stride of the increment buffer
    const int NA = m.n_owned > 0 ? m.n_owned : N;         // cells this launch updates
    const int stride = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const bool do_cons = FINAL && a.cons, do_cfl = FINAL && a.cfl;
    double cons_acc[C], ad_acc[ADAPT ? 3 * C : 1], cfl_acc = 0.0;
#pragma unroll
    for (int c = 0; c < C; ++c) cons_acc[c] = 0.0;
#pragma unroll
    for (int c = 0; c < (ADAPT ? 3 * C : 1); ++c) ad_acc[c] = 0.0;
    int i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    float nxt[Ly::DR];
    const bool skip_frozen = frozen_skip(m, NA, stride);
    if (i0 + lane < NA && (!skip_frozen || case_on(m, m.cell_case, i0 + lane)))
        ld_vec<Ly::DR>(m.div_rec + (int64_t)(i0 + lane) * Ly::DR, nxt);
    else
#pragma unroll
        for (int q = 0; q < Ly::DR; ++q) nxt[q] = 0.f;
    for (int64_t tile = blockIdx.x; i0 < NA; i0 += stride, tile += gridDim.x) {
        if (waves > 0) {
            prefetch_tile(m.div_rec, NA, Ly::DR, tile + (int64_t)waves * gridDim.x);
            if (MODE != DIV_RESIDUAL) prefetch_tile(state, NA, C, tile + (int64_t)waves * gridDim.x);
        }
        const int i = i0 + lane;
        const bool live = i < NA && (m.case_active == nullptr || case_on(m, m.cell_case, i));
        float rec[Ly::DR];
#pragma unroll
        for (int q = 0; q < Ly::DR; ++q) rec[q] = nxt[q];
        float r[C];
#pragma unroll
        for (int c = 0; c < C; ++c) r[c] = 0.f;
        if (live) {
#pragma unroll
            for (int k = 0; k < Ly::K; ++k) {
                if (k < m.kf) {
                    const float w = rec[k];
                    float Fk[RS];
                    ld_vec_cg<RS>(flux + (int64_t)as_int(rec[Ly::K + k]) * RS, Fk);
#pragma unroll
                    for (int c = 0; c < C; ++c) r[c] = fmaf(w, Fk[c], r[c]);
                }
            }
        }
        if (i + stride < NA && (!skip_frozen || case_on(m, m.cell_case, i + stride)))
            ld_vec<Ly::DR>(m.div_rec + (int64_t)(i + stride) * Ly::DR, nxt);
        if (MODE == DIV_RESIDUAL) {
            if (live) store_state<C>(dudt + (int64_t)i * C, r);
            continue;
        }
        const int cse = (m.n_cases > 0 && live) ? __ldg(m.cell_case + i) : 0;
        const float h = COH ? __ldcg(dt + cse) : dt[cse];
        float kk[C], U0[C], inc[C], U[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            kk[c] = h * r[c];
            inc[c] = 0.f;
            U0[c] = U[c] = 0.f;
        }
        if (live) {
            if (a.store_k) store_state<C>(kbuf + ((int64_t)a.s * N + i) * C, kk);
            load_state<C>(state + (int64_t)i * C, U0);
            for (int t = 0; t < a.n_terms; ++t) {
                float kt[C];
                if (a.idx[t] == a.s) {
#pragma unroll
                    for (int c = 0; c < C; ++c) kt[c] = kk[c];
                } else {
                    load_state<C>(kbuf + ((int64_t)a.idx[t] * N + i) * C, kt);
                }
#pragma unroll
                for (int c = 0; c < C; ++c) inc[c] = fmaf(a.coef[t], kt[c], inc[c]);
            }
#pragma unroll
            for (int c = 0; c < C; ++c) U[c] = U0[c] + inc[c];
            if (FINAL) store_state<C>(state + (int64_t)i * C, U);
            float P[RS];
            state_to_prim<C, RS>(U, p.inv_Cv, P);
            st_vec<RS>(prims + (int64_t)i * RS, P);
        }
        if (!FINAL) continue;
        if (ADAPT && live) {
            // Column norms of dU_high - dU_low, dU_high and U0 (integrators.py:54), in FP64.
            float lo[C];
#pragma unroll
            for (int c = 0; c < C; ++c) lo[c] = 0.f;
            for (int t = 0; t < a.n_lo; ++t) {
                float kt[C];
                if (a.idx_lo[t] == a.s) {
#pragma unroll
                    for (int c = 0; c < C; ++c) kt[c] = kk[c];
                } else {
                    load_state<C>(kbuf + ((int64_t)a.idx_lo[t] * N + i) * C, kt);
                }
#pragma unroll
                for (int c = 0; c < C; ++c) lo[c] = fmaf(a.coef_lo[t], kt[c], lo[c]);
            }
#pragma unroll
            for (int c = 0; c < (ADAPT ? C : 0); ++c) {
                const double e = (double)inc[c] - (double)lo[c];
                ad_acc[c] += e * e;
                ad_acc[C + c] += (double)inc[c] * inc[c];
                ad_acc[2 * C + c] += (double)U0[c] * U0[c];
            }
        }
        if (m.n_cases > 0) {
            reduce_batched_item<DIM>(m, p, U, live, i, cse, do_cons, do_cfl, red);
        } else if (live) {
            if (do_cons)
#pragma unroll
                for (int c = 0; c < C; ++c) cons_acc[c] += __ldg(m.volumes + i) * (double)U[c];
            if (do_cfl) cfl_acc = fmax(cfl_acc, cfl_speed<DIM>(m, p, U, i));
        }
    }
    if (!FINAL || m.n_cases > 0) return;
    __shared__ double smem[32 * (ADAPT ? 3 * C : C)];
    if (ADAPT) {
        block_sum<ADAPT ? 3 * C : 1>(ad_acc, smem);
        if (threadIdx.x == 0)
            for (int c = 0; c < 3 * C; ++c) atomicAdd(red + c, ad_acc[c]);
        __syncthreads();
    }
    if (do_cons) {
        block_sum<C>(cons_acc, smem);
        if (threadIdx.x == 0)
            for (int c = 0; c < C; ++c) atomicAdd(red + 24 + c, cons_acc[c]);
        __syncthreads();
    }
    if (do_cfl) {
        const double sp = block_max(cfl_acc, smem);
        if (threadIdx.x == 0) atomic_max_pos(red + 16, sp);
    }
}

template <int DIM, int MODE>
__global__ void __launch_bounds__(kMaxBlock) k_div_stage(fvm_mesh_t m, Phys p, const float* __restrict__ flux,
                                                       StageArgs a, float* __restrict__ state,
                                                       float* __restrict__ prims, float* __restrict__ kbuf,
                                                       const float* __restrict__ dt,
                                                       double* __restrict__ red,
                                                       float* __restrict__ dudt, int waves) {
    dependency_wait();
    div_body<DIM, MODE, false>(m, p, flux, a, state, prims, kbuf, dt, red, dudt, waves);
}

// Step-end bookkeeping: adaptive dt (integrators.py:42-62) or CFL dt, conservation sums.
// Batched meshes (n_cases > 0): one thread per case handles its CFL dt and sums.
// The sums were accumulated by atomics of other blocks (in the fused step, of the same launch):
// read them through L2.
__device__ __forceinline__ void finalize_body(int C, int adaptive, float atol, float rtol, float mtol,
                                              float alpha_hi, float alpha_lo, float order, float cfl, int cons,
                                              double* red, float* dt, double* cons_out, int n_cases,
                                              const uint8_t* __restrict__ active) {
    if (n_cases > 0) {
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cases; c += gridDim.x * blockDim.x) {
            if (active && !active[c]) continue;
            double* slot = red + FVM_RED_DOUBLES + 8 * c;
            if (cfl > 0.f) {
                const double smax = __ldcg(slot);
                if (smax > 0.0) dt[c] = (float)((double)cfl / smax);
                slot[0] = 0.0;
            }
            if (cons) {
                for (int k = 0; k < C; ++k) {
                    if (cons_out) cons_out[c * C + k] = __ldcg(slot + 1 + k);
                    slot[1 + k] = 0.0;
                }
            }
        }
        return;
    }
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (adaptive) {
        double E = 0.0;
        for (int c = 0; c < C; ++c) {
            const double nd = sqrt(__ldcg(red + c)), nh = sqrt(__ldcg(red + C + c)), nu = sqrt(__ldcg(red + 2 * C + c));
            E += nd / ((double)atol + (double)rtol * nh + (double)mtol * nu);
            red[c] = red[C + c] = red[2 * C + c] = 0.0;
        }
        E /= C;
        const float Ef = (float)E;
        const float factor = 0.9f * powf(Ef, -1.f / order);
        const float alpha = Ef > 1.f ? alpha_hi : alpha_lo;
        dt[0] = dt[0] * (alpha + (1.f - alpha) * factor);
        red[40] = E;
    }
    if (cfl > 0.f) {
        const double smax = __ldcg(red + 16);
        if (smax > 0.0) dt[0] = (float)((double)cfl / smax);
        red[16] = 0.0;
    }
    if (cons) {
        for (int c = 0; c < C; ++c) {
            if (cons_out) cons_out[c] = __ldcg(red + 24 + c);
            red[24 + c] = 0.0;
        }
    }
}

__global__ void k_finalize(int C, int adaptive, float atol, float rtol, float mtol, float alpha_hi,
                           float alpha_lo, float order, float cfl, int cons, double* red, float* dt,
                           double* cons_out, int n_cases, const uint8_t* __restrict__ active) {
    dependency_wait();
    finalize_body(C, adaptive, atol, rtol, mtol, alpha_hi, alpha_lo, order, cfl, cons, red, dt, cons_out, n_cases,
                  active);
}

// ------------------------------------------------------------------------------------------
// Fused step: every phase of every stage of one step in one cooperative launch.
//
// For small meshes a step is latency bound: 3-4 dependent launches per stage, each too short to
// fill the GPU.  k_step_fused runs the same phase bodies (boundary values, cell gradients, facet
// fluxes, divergence + stage update, step-end bookkeeping) back to back in one persistent grid of
// co-resident blocks (cooperative launch), separated by grid-wide barriers.  Loads of arrays written
// earlier in the launch use the coherent (.cg) path.  Every per-item computation and every
// block-level reduction order is the one of the separate kernels, so the result is bitwise the
// same.  Barrier waits are bounded: a wait that gives up sets the status word and the launch runs
// to its end (with wrong results) instead of hanging; the host checks it (fvm_fused_status).
// ------------------------------------------------------------------------------------------
constexpr long long kBarrierSpinLimit = 1LL << 22;

struct FusedArgs {
    int stages;
    StageArgs st[FVM_MAX_STAGES];
    int need_final;                       // last stage: adaptive / CFL / conservation bookkeeping
    int adaptive;
    float atol, rtol, mtol, alpha_hi, alpha_lo, order, cfl;
    float* state;
    float* prims;
    float* grads;
    int32_t* has_grads;
    float* k;
    float* dt;
    double* cons;
    float* bcv;
    float* flux;
    double* red;
    unsigned* bar;                        // [0] arrivals, [1] generation
    int* status;                          // set to 1 when a barrier wait gave up
};

__device__ __forceinline__ void grid_barrier(unsigned* bar, int* status) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1u == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > kBarrierSpinLimit) {
                    atomicExch(status, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// Barrier self-test: every block but `skip` meets at grid_barrier twice; with skip >= 0 that block
// never arrives, so the others' bounded waits give up and set the status word.
__global__ void __launch_bounds__(64) k_barrier_selftest(unsigned* bar, int* status, int skip, long long limit) {
    if ((int)blockIdx.x == skip) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1u == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > limit) {
                    atomicExch(status, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
    }
    __syncthreads();
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_step_fused(fvm_mesh_t m, Phys p, FusedArgs f) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (int s = 0; s < f.stages; ++s) {
        const StageArgs& a = f.st[s];
        if (m.n_bc > 0) {
            if (m.n_cases > 0 && m.n_char > 0) {
                for (int c = blockIdx.x; c < m.n_cases; c += gridDim.x)
                    char_scale_case<DIM, true>(m, p, f.prims, f.red, c);
                grid_barrier(f.bar, f.status);
            }
            const float scale = bc_block_scale<DIM, true>(m, p, f.prims);
            for (int b = tid; b < m.n_bc; b += nth)
                bc_item<DIM, true>(m, p, f.prims, f.grads, f.has_grads, f.bcv, f.red, b, scale);
            grid_barrier(f.bar, f.status);
        }
        if (m.kg == DIM + 2) cell_body<DIM, true>(m, p, f.prims, f.bcv, f.grads, f.has_grads, 0);
        else cell_wide_body<DIM, true>(m, p, f.prims, f.bcv, f.grads, f.has_grads);
        grid_barrier(f.bar, f.status);
        face_body<DIM, true>(m, p, f.prims, f.bcv, f.grads, f.flux, 0);
        grid_barrier(f.bar, f.status);
        if (!a.final_)
            div_body<DIM, DIV_STAGE, true>(m, p, f.flux, a, f.state, f.prims, f.k, f.dt, f.red, nullptr, 0);
        else if (a.adaptive)
            div_body<DIM, DIV_FINAL_ADAPT, true>(m, p, f.flux, a, f.state, f.prims, f.k, f.dt, f.red, nullptr, 0);
        else
            div_body<DIM, DIV_FINAL, true>(m, p, f.flux, a, f.state, f.prims, f.k, f.dt, f.red, nullptr, 0);
        grid_barrier(f.bar, f.status);
        if (a.final_ && f.need_final) {
            finalize_body(DIM + 2, f.adaptive, f.atol, f.rtol, f.mtol, f.alpha_hi, f.alpha_lo, f.order, f.cfl, a.cons,
                          f.red, f.dt, f.cons, m.n_cases, m.case_active);
            grid_barrier(f.bar, f.status);
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_state_to_prims(int N, float inv_Cv, const float* __restrict__ state,
                                                            float* __restrict__ prims) {
    dependency_wait();
    using Ly = L<DIM>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float U[Ly::C], P[Ly::RS];
#pragma unroll
    for (int c = 0; c < Ly::C; ++c) U[c] = __ldg(state + (int64_t)i * Ly::C + c);
    state_to_prim<Ly::C, Ly::RS>(U, inv_Cv, P);
    st_vec<Ly::RS>(prims + (int64_t)i * Ly::RS, P);
}

// [N][C] primitives -> padded [N][RS] rows (fvm_residual takes the reference's layout).
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_pad_prims(int N, const float* __restrict__ src, float* __restrict__ dst) {
    dependency_wait();
    using Ly = L<DIM>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float P[Ly::RS];
#pragma unroll
    for (int c = 0; c < Ly::RS; ++c) P[c] = c < Ly::C ? __ldg(src + (int64_t)i * Ly::C + c) : 0.f;
    st_vec<Ly::RS>(dst + (int64_t)i * Ly::RS, P);
}

// Conservation sums sum vol U and the CFL speed maximum of a state: a persistent grid-stride loop.
// Single mesh: each thread accumulates over its cells and the block combines once (one atomic
// per block and quantity).  Batched meshes: warp-uniform iterations, per-item warp reductions
// into the per-case slots (reduce_batched_item).
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_reduce_state(fvm_mesh_t m, Phys p, const float* __restrict__ state,
                                                          int want_cfl, int want_cons, double* red) {
    constexpr int C = DIM + 2;
    const int NA = m.n_owned > 0 ? m.n_owned : m.n_cells;
    const int stride = gridDim.x * blockDim.x;
    if (m.n_cases == 0) {
        __shared__ double smem[32 * C];
        double cons[C], sp = 0.0;
#pragma unroll
        for (int c = 0; c < C; ++c) cons[c] = 0.0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NA; i += stride) {
            float U[C];
#pragma unroll
            for (int c = 0; c < C; ++c) U[c] = __ldg(state + (int64_t)i * C + c);
            if (want_cons) {
                const double vol = __ldg(m.volumes + i);
#pragma unroll
                for (int c = 0; c < C; ++c) cons[c] += vol * (double)U[c];
            }
            if (want_cfl) sp = fmax(sp, cfl_speed<DIM>(m, p, U, i));
        }
        if (want_cons) {
            block_sum<C>(cons, smem);
            if (threadIdx.x == 0)
                for (int c = 0; c < C; ++c) atomicAdd(red + 24 + c, cons[c]);
            __syncthreads();
        }
        if (want_cfl) {
            sp = block_max(sp, smem);
            if (threadIdx.x == 0) atomic_max_pos(red + 16, sp);
        }
        return;
    }
    // Batched: each warp takes one contiguous chunk of cells and accumulates per lane while the
    // case stays the same (a case's cells are contiguous); a change of case flushes the partial
    // results with one warp reduction and one atomic per quantity into the old case's slots.
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warps = stride >> 5;
    const int64_t w = (int64_t)(blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t chunk = (((int64_t)NA + warps - 1) / warps + 31) & ~(int64_t)31;
    const int64_t beg = w * chunk, end = beg + chunk < NA ? beg + chunk : (int64_t)NA;
    int cur = -1;                                      // case of the accumulators (warp-uniform)
    double acc[C], amax = 0.0;
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0.0;
    auto flush = [&]() {
        if (cur < 0) return;
        double* slot = red + FVM_RED_DOUBLES + 8 * cur;
        if (want_cfl) {
            double v = amax;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(full, v, o));
            if (lane == 0 && v > 0.0) atomic_max_pos(slot, v);
        }
        if (want_cons)
#pragma unroll
            for (int c = 0; c < C; ++c) {
                double v = acc[c];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
                if (lane == 0) atomicAdd(slot + 1 + c, v);
            }
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] = 0.0;
        amax = 0.0;
    };
    for (int64_t i0 = beg; i0 < end; i0 += 32) {
        const int64_t i = i0 + lane;
        const bool live = i < end;
        const int cse = live ? __ldg(m.cell_case + i) : -1;
        double v[C], sp = 0.0;
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = 0.0;
        if (live) {
            float U[C];
#pragma unroll
            for (int c = 0; c < C; ++c) U[c] = __ldg(state + i * C + c);
            if (want_cons) {
                const double vol = __ldg(m.volumes + i);
#pragma unroll
                for (int c = 0; c < C; ++c) v[c] = vol * (double)U[c];
            }
            if (want_cfl) sp = cfl_speed<DIM>(m, p, U, (int)i);
        }
        unsigned pending = __ballot_sync(full, live);
        while (pending) {                              // once per distinct case among the lanes
            const int lc = __shfl_sync(full, cse, __ffs(pending) - 1);
            if (lc != cur) {
                flush();
                cur = lc;
            }
            const bool mine = live && cse == lc;
            if (mine) {
#pragma unroll
                for (int c = 0; c < C; ++c) acc[c] += v[c];
                amax = fmax(amax, sp);
            }
            pending &= ~__ballot_sync(full, mine);
        }
    }
    flush();
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
static Phys make_phys(const fvm_physics_t* ph) {
    Phys p;
    p.T_0 = ph->T_0;
    p.mu = ph->mu;
    p.mu_b = ph->mu_b;
    p.S = ph->S_const;
    p.C_v = ph->C_v;
    p.gamma = ph->gamma;
    p.kappa = ph->kappa;
    p.v_factor = ph->v_factor;
    p.lim_p = ph->lim_p;
    // Python-scalar constants of the reference, evaluated in double and rounded once to float.
    const double R = (double)ph->C_v * ((double)ph->gamma - 1.0);
    p.R = (float)R;
    p.gR = (float)((double)ph->gamma * R);
    p.inv_Cv = (float)(1.0 / (double)ph->C_v);
    p.T0pS = (float)((double)ph->T_0 + (double)ph->S_const);
    p.T0sq = (float)((double)ph->T_0 * (double)ph->T_0);
    p.inv_T0 = (float)(1.0 / (double)ph->T_0);
    p.inv_T0sq = (float)(1.0 / ((double)ph->T_0 * (double)ph->T_0));
    return p;
}

static bool aligned32(const void* p) { return ((uintptr_t)p & 31u) == 0; }   // rows use 256-bit accesses

static inline int owned_cells(const fvm_mesh_t* m) { return m->n_owned > 0 ? m->n_owned : m->n_cells; }

static bool mesh_ok(const fvm_mesh_t* m) {
    if (!m || (m->dim != 2 && m->dim != 3) || m->n_comp != m->dim + 2) return false;
    if (m->n_cells <= 0 || m->n_facets <= 0 || m->n_bc < 0 || m->n_char < 0) return false;
    if (m->kg < m->dim + 2 || m->kg > FVM_MAX_KG || m->kf < 1 || m->kf > m->dim + 1) return false;
    if (!m->cell_rec || !m->div_rec || !m->face_rec || !m->inv_h || !m->volumes) return false;
    if (!aligned32(m->cell_rec) || !aligned32(m->div_rec) || !aligned32(m->face_rec)) return false;
    if (m->n_bc > 0 && (!m->bc_cell || !m->bc_kind || !m->bc_b || !m->bc_l || !m->bc_ga || !m->bc_gb ||
                        !m->bc_char))
        return false;
    if (m->n_char > 0 && (!m->ch_cell || !m->ch_normal || !m->ch_rho || !m->ch_vn || !m->ch_p || !m->ch_vt))
        return false;
    if (m->n_cases < 0) return false;
    if (m->n_owned < 0 || m->n_owned > m->n_cells || m->char_scale_given < 0 || m->char_scale_given > 1) return false;
    if (m->n_cases > 0 && (m->n_owned > 0 || m->char_scale_given)) return false;
    if (m->cell_lo < 0 || m->cell_lo > owned_cells(m) || m->facet_lo < 0 || m->facet_lo > m->n_facets) return false;
    if (m->n_cases > 0 && (m->cell_lo || m->facet_lo)) return false;
    if (m->n_cases == 0 && m->case_active) return false;
    if (m->n_cases > 0 && (!m->cell_case || !m->face_case || !m->ch_off || !m->case_mu || !m->case_mu_b ||
                           !m->case_kappa || (m->n_bc > 0 && !m->bc_case)))
        return false;
    return true;
}

static bool work_ok(const fvm_mesh_t* m, const fvm_work_t* w) {
    return w && w->flux && w->red && aligned32(w->flux) && (m->n_bc == 0 || (w->bc_vals && aligned32(w->bc_vals)));
}

static inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// Threads per block of the cell, facet and divergence kernels (set by the autotuner through
// fvm_set_block_size).  The boundary kernels keep kBlock: their per-block reduction order must not
// change between single-mesh and batched runs.
static int g_block_cell = kBlock, g_block_face = kBlock, g_block_div = kBlock;
// Record prefetch distance in waves of resident blocks per kernel: -1 = default (off: with the
// persistent kernels' index look-ahead it measured slower on the 2M-tet box), 0 = off.
static int g_pf_cell = -1, g_pf_face = -1, g_pf_div = -1;
// Facet kernel variant (fvm_set_variant): 0 = records loaded by each thread (k_face), 1 = records
// staged through shared memory by the bulk-copy unit (k_face_staged).  Same results.
static int g_face_variant = 0;
// Residual evaluations (fvm_residual, fvm_residual_state): 0 = facet kernel then divergence
// kernel, 1 = owner-computes k_face_div (whole meshes; same bits).  Stages always use 0.
static int g_div_variant = 0;
static inline int waves_of(int setting) { return setting < 0 ? 0 : setting; }

// Resident blocks of `kernel` at `threads` per block over the whole GPU (one wave), cached.
template <typename Kern>
static int wave_blocks(Kern kernel, int threads) {
    struct Entry { const void* k; int threads, dev, blocks; };
    static Entry cache[128];
    static int n_cache = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    for (int e = 0; e < n_cache; ++e)
        if (cache[e].k == (const void*)kernel && cache[e].threads == threads && cache[e].dev == dev)
            return cache[e].blocks;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    const int blocks = per_sm * sms;
    if (n_cache < 128) cache[n_cache++] = Entry{(const void*)kernel, threads, dev, blocks};
    return blocks;
}
static inline unsigned blocks_of(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }
// Grid of a persistent grid-stride kernel: one wave of resident blocks, or fewer if n is small.
static inline unsigned persistent_grid(int64_t n, int threads, int wave) {
    const unsigned all = blocks_of(n, threads);
    return wave > 0 && (unsigned)wave < all ? (unsigned)wave : all;
}
template <int DIM>
static inline unsigned reduce_grid(const fvm_mesh_t* m) {
    return persistent_grid(owned_cells(m), kBlock, wave_blocks(k_reduce_state<DIM>, kBlock));
}
static inline unsigned fin_blocks(const fvm_mesh_t* m) {
    return m->n_cases > 0 ? (unsigned)((m->n_cases + 127) / 128) : 1u;
}

// Boundary values and limited cell gradients for the padded primitives `prims`.
template <int DIM>
static int launch_begin(const fvm_mesh_t* m, const Phys& p, const float* prims, float* grads,
                        int32_t* has_grads, const fvm_work_t* w, cudaStream_t s) {
    if (m->n_bc > 0) {
        if (m->n_cases > 0 && m->n_char > 0)
            FVM_LAUNCH(KID_BC, s, launch(k_char_scale<DIM>, dim3(m->n_cases), dim3(kBlock), 0, s, *m, p, prims, w->red));
        FVM_LAUNCH(KID_BC, s, launch(k_bc<DIM>, dim3(blocks_for(m->n_bc)), dim3(kBlock), 0, s, *m, p, prims, grads, has_grads,
                                                                               w->bc_vals, w->red));
    }
    if (owned_cells(m) - m->cell_lo <= 0) return launch_status();   // empty range: nothing to launch
    if (m->kg != DIM + 2) {
        const unsigned gw = persistent_grid(owned_cells(m) - m->cell_lo, kBlock, wave_blocks(k_cell_wide<DIM>, kBlock));
        FVM_LAUNCH(KID_CELL, s, launch(k_cell_wide<DIM>, dim3(gw), dim3(kBlock), 0, s, *m, p, prims, w->bc_vals, grads, has_grads));
        return launch_status();
    }
    const unsigned gc =
        persistent_grid(owned_cells(m) - m->cell_lo, g_block_cell, wave_blocks(k_cell<DIM>, g_block_cell));
    FVM_LAUNCH(KID_CELL, s, launch(k_cell<DIM>, dim3(gc), dim3(g_block_cell), 0, s, *m, p, prims, w->bc_vals, grads, has_grads,
                                                                    waves_of(g_pf_cell)));
    return launch_status();
}

// Resident blocks of the staged facet kernel at `threads` per block (its dynamic shared memory
// counted), cached per block size and device.
template <int DIM>
static int staged_wave(int threads) {
    static int cache[2][kMaxBlock / 32 + 1][64];
    static bool attr[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return 0;
    int& c = cache[DIM - 2][threads / 32][dev];
    if (c > 0) return c;
    const int smem = 2 * threads * L<DIM>::FR * 4;
    if (!attr[dev]) {
        if (cudaFuncSetAttribute(k_face_staged<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 2 * kMaxBlock * L<DIM>::FR * 4) != cudaSuccess)
            return 0;
        attr[dev] = true;
    }
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_face_staged<DIM>, threads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    c = per_sm * sms;
    return c;
}

template <int DIM>
static int launch_face(const fvm_mesh_t* m, const Phys& p, const float* prims, const float* grads,
                       const fvm_work_t* w, cudaStream_t s) {
    if (m->n_facets - m->facet_lo <= 0) return launch_status();
    if (g_face_variant == 1) {
        const int wave = staged_wave<DIM>(g_block_face);
        if (wave <= 0) {
            launch_status();
            return FVM_E_CUDA;
        }
        const unsigned gf = persistent_grid(m->n_facets - m->facet_lo, g_block_face, wave);
        const size_t smem = (size_t)2 * g_block_face * L<DIM>::FR * 4;
        FVM_LAUNCH(KID_FACE, s, launch(k_face_staged<DIM>, dim3(gf), dim3(g_block_face), smem, s, *m, p, prims, w->bc_vals, grads,
                                                                                  w->flux));
        return launch_status();
    }
    const unsigned gf =
        persistent_grid(m->n_facets - m->facet_lo, g_block_face, wave_blocks(k_face<DIM>, g_block_face));
    FVM_LAUNCH(KID_FACE, s, launch(k_face<DIM>, dim3(gf), dim3(g_block_face), 0, s, *m, p, prims, w->bc_vals, grads, w->flux,
                                                                    waves_of(g_pf_face)));
    return launch_status();
}

// bc -> cell -> face for the padded primitives `prims`; leaves fluxes in work->flux.
template <int DIM>
static int launch_fluxes(const fvm_mesh_t* m, const Phys& p, const float* prims, float* grads,
                         int32_t* has_grads, const fvm_work_t* w, cudaStream_t s) {
    const int rc = launch_begin<DIM>(m, p, prims, grads, has_grads, w, s);
    return rc ? rc : launch_face<DIM>(m, p, prims, grads, w, s);
}

template <int DIM, int MODE>
static void launch_div_mode(const fvm_mesh_t* m, const Phys& p, const float* flux, const StageArgs& a, float* state,
                            float* prims, float* kbuf, const float* dt, double* red, float* dudt, cudaStream_t s) {
    const unsigned grid =
        persistent_grid(owned_cells(m), g_block_div, wave_blocks(k_div_stage<DIM, MODE>, g_block_div));
    FVM_LAUNCH(KID_DIV_STAGE, s, launch(k_div_stage<DIM, MODE>, dim3(grid), dim3(g_block_div), 0, s, 
                                     *m, p, flux, a, state, prims, kbuf, dt, red, dudt, waves_of(g_pf_div)));
}

// Divergence (+ stage combination): picks the kernel variant for what the launch must do.
template <int DIM>
static int launch_div(const fvm_mesh_t* m, const Phys& p, const float* flux, const StageArgs& a, float* state,
                      float* prims, float* kbuf, const float* dt, double* red, float* dudt, cudaStream_t s) {
    if (dudt)
        launch_div_mode<DIM, DIV_RESIDUAL>(m, p, flux, a, state, prims, kbuf, dt, red, dudt, s);
    else if (!a.final_)
        launch_div_mode<DIM, DIV_STAGE>(m, p, flux, a, state, prims, kbuf, dt, red, dudt, s);
    else if (a.adaptive)
        launch_div_mode<DIM, DIV_FINAL_ADAPT>(m, p, flux, a, state, prims, kbuf, dt, red, dudt, s);
    else
        launch_div_mode<DIM, DIV_FINAL>(m, p, flux, a, state, prims, kbuf, dt, red, dudt, s);
    return launch_status();
}

// dU/dt from the padded primitives in work->prims: bc -> cell -> face -> divergence, or with the
// owner-computes variant bc -> cell -> k_face_div (whole meshes; same bits).
template <int DIM>
static int launch_residual(const fvm_mesh_t* m, const Phys& p, float* grads, int32_t* has_grads, float* dudt,
                           const fvm_work_t* w, cudaStream_t s) {
    if (g_div_variant == 1 && m->cell_lo == 0 && m->facet_lo == 0 && owned_cells(m) > 0) {
        const int rc = launch_begin<DIM>(m, p, w->prims, grads, has_grads, w, s);
        if (rc) return rc;
        const unsigned g = persistent_grid(4 * (int64_t)owned_cells(m), g_block_face,
                                           wave_blocks(k_face_div<DIM>, g_block_face));
        FVM_LAUNCH(KID_DIV_STAGE, s, launch(k_face_div<DIM>, dim3(g), dim3(g_block_face), 0, s, *m, p, w->prims, w->bc_vals, grads,
                                                                                dudt));
        return launch_status();
    }
    const int rc = launch_fluxes<DIM>(m, p, w->prims, grads, has_grads, w, s);
    if (rc) return rc;
    StageArgs a{};
    return launch_div<DIM>(m, p, w->flux, a, nullptr, nullptr, nullptr, nullptr, nullptr, dudt, s);
}

template <int DIM>
static int residual_impl(const fvm_mesh_t* m, const Phys& p, const float* prims_user, float* grads,
                         int32_t* has_grads, float* dudt, const fvm_work_t* w, cudaStream_t s) {
    FVM_LAUNCH(KID_STATE_TO_PRIMS, s, launch(k_pad_prims<DIM>, dim3(blocks_for(m->n_cells)), dim3(kBlock), 0, s, 
                                          m->n_cells, prims_user, w->prims));
    return launch_residual<DIM>(m, p, grads, has_grads, dudt, w, s);
}

// dU/dt of a conserved state: one kernel writes the padded primitives into work->prims (the
// stage kernels' conversion), then the residual kernels as in residual_impl.
template <int DIM>
static int residual_state_impl(const fvm_mesh_t* m, const Phys& p, const float* state, float* grads,
                               int32_t* has_grads, float* dudt, const fvm_work_t* w, cudaStream_t s) {
    FVM_LAUNCH(KID_STATE_TO_PRIMS, s, launch(k_state_to_prims<DIM>, dim3(blocks_for(m->n_cells)), dim3(kBlock), 0, s, 
                                          m->n_cells, p.inv_Cv, state, w->prims));
    return launch_residual<DIM>(m, p, grads, has_grads, dudt, w, s);
}

static StageArgs stage_args(const fvm_tableau_t* tab, int s) {
    StageArgs a{};
    const int S = tab->stages;
    a.s = s;
    a.final_ = s == S - 1;
    if (!a.final_) {
        for (int j = 0; j <= s; ++j)
            if (tab->a[s + 1][j] != 0.f) {
                a.idx[a.n_terms] = j;
                a.coef[a.n_terms++] = tab->a[s + 1][j];
            }
        bool needed = tab->b[s] != 0.f || (tab->adaptive && tab->b2[s] != 0.f);
        for (int i = s + 2; i < S; ++i) needed = needed || tab->a[i][s] != 0.f;
        a.store_k = needed;
    } else {
        for (int j = 0; j < S; ++j)
            if (tab->b[j] != 0.f) {
                a.idx[a.n_terms] = j;
                a.coef[a.n_terms++] = tab->b[j];
            }
        if (tab->adaptive) {
            for (int j = 0; j < S; ++j)
                if (tab->b2[j] != 0.f) {
                    a.idx_lo[a.n_lo] = j;
                    a.coef_lo[a.n_lo++] = tab->b2[j];
                }
        }
        a.store_k = 0;
        a.adaptive = tab->adaptive;
        a.cfl = tab->cfl > 0.f;
    }
    return a;
}

static int finalize_impl(const fvm_mesh_t* m, const fvm_tableau_t* tab, const fvm_solver_bufs_t* b,
                         const fvm_work_t* w, int cons, cudaStream_t st) {
    FVM_LAUNCH(KID_FINALIZE, st,
               launch(k_finalize, dim3(fin_blocks(m)), dim3(128), 0, st, m->n_comp, tab->adaptive, tab->atol, tab->rtol, tab->mtol,
                                                         tab->alpha_hi_err, tab->alpha_lo_err, tab->order, tab->cfl,
                                                         cons, w->red, b->dt, b->cons, m->n_cases, m->case_active));
    return launch_status();
}

// Facet fluxes, divergence and stage combination of stage s (the cell gradients are in b->grads);
// on the last stage also the dt / conservation bookkeeping unless the caller defers it.
template <int DIM>
static int stage_finish(const fvm_mesh_t* m, const Phys& p, const fvm_tableau_t* tab, int s,
                        const fvm_solver_bufs_t* b, const fvm_work_t* w, int finalize, cudaStream_t st) {
    int rc = launch_face<DIM>(m, p, b->prims, b->grads, w, st);
    if (rc) return rc;
    StageArgs a = stage_args(tab, s);
    a.cons = a.final_ && b->cons != nullptr;
    rc = launch_div<DIM>(m, p, w->flux, a, b->state, b->prims, b->k, b->dt, w->red, nullptr, st);
    if (rc) return rc;
    if (finalize && a.final_ && (a.adaptive || a.cfl || a.cons)) rc = finalize_impl(m, tab, b, w, a.cons, st);
    return rc;
}

// The phases of stage s that `phases` selects, in their order (FVM_PHASE_* bits).
template <int DIM>
static int stage_phase_impl(const fvm_mesh_t* m, const Phys& p, const fvm_tableau_t* tab, int s,
                            const fvm_solver_bufs_t* b, const fvm_work_t* w, int phases, int finalize,
                            cudaStream_t st) {
    int rc = FVM_OK;
    if (phases & (FVM_PHASE_BC | FVM_PHASE_CELLS)) {
        fvm_mesh_t mm = *m;
        if (!(phases & FVM_PHASE_BC)) mm.n_bc = 0;                                   // cells only
        if (!(phases & FVM_PHASE_CELLS)) mm.cell_lo = owned_cells(m);               // boundary values only
        rc = launch_begin<DIM>(&mm, p, b->prims, b->grads, b->has_grads, w, st);
        if (rc) return rc;
    }
    if (phases & FVM_PHASE_FACES) {
        rc = launch_face<DIM>(m, p, b->prims, b->grads, w, st);
        if (rc) return rc;
    }
    if (phases & FVM_PHASE_DIV) {
        fvm_mesh_t mm = *m;
        mm.cell_lo = 0;
        StageArgs a = stage_args(tab, s);
        a.cons = a.final_ && b->cons != nullptr;
        rc = launch_div<DIM>(&mm, p, w->flux, a, b->state, b->prims, b->k, b->dt, w->red, nullptr, st);
        if (rc) return rc;
        if (finalize && a.final_ && (a.adaptive || a.cfl || a.cons)) rc = finalize_impl(&mm, tab, b, w, a.cons, st);
    }
    return rc;
}

template <int DIM>
static int stage_impl(const fvm_mesh_t* m, const Phys& p, const fvm_tableau_t* tab, int s,
                      const fvm_solver_bufs_t* b, const fvm_work_t* w, cudaStream_t st) {
    const int rc = launch_begin<DIM>(m, p, b->prims, b->grads, b->has_grads, w, st);
    return rc ? rc : stage_finish<DIM>(m, p, tab, s, b, w, 1, st);
}

// Partitioned meshes: sum of the interior sound speed over this part's characteristic facets and
// their count -> red[FVM_RED_DOUBLES + 6], red[FVM_RED_DOUBLES + 7].
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_char_partial(fvm_mesh_t m, Phys p, const float* __restrict__ prims,
                                                          double* __restrict__ red_out) {
    __shared__ double red[32];
    const double sum = char_c_sum<DIM>(m, p, prims, 0, m.n_char, red);
    if (threadIdx.x == 0) {
        red_out[FVM_RED_DOUBLES + 6] = sum;
        red_out[FVM_RED_DOUBLES + 7] = (double)m.n_char;
    }
}

template <int DIM>
static int multistep_impl(const fvm_mesh_t* m, const Phys& p, int store, int n_terms, const int32_t* idx,
                          const float* coef, const fvm_solver_bufs_t* b, const fvm_work_t* w,
                          cudaStream_t st) {
    int rc = launch_fluxes<DIM>(m, p, b->prims, b->grads, b->has_grads, w, st);
    if (rc) return rc;
    StageArgs a{};
    a.s = store;
    a.store_k = 1;
    a.final_ = 1;
    a.n_terms = n_terms;
    for (int t = 0; t < n_terms; ++t) {
        a.idx[t] = idx[t];
        a.coef[t] = coef[t];
    }
    a.cons = b->cons != nullptr;
    rc = launch_div<DIM>(m, p, w->flux, a, b->state, b->prims, b->k, b->dt, w->red, nullptr, st);
    if (rc) return rc;
    if (a.cons) {
        FVM_LAUNCH(KID_FINALIZE, st, launch(k_finalize, dim3(fin_blocks(m)), dim3(128), 0, st, m->n_comp, 0, 0.f, 0.f, 0.f, 0.f, 0.f,
                                                                              1.f, 0.f, 1, w->red, b->dt, b->cons,
                                                                              m->n_cases, m->case_active));
        rc = launch_status();
    }
    return rc;
}

}  // namespace fvm

using namespace fvm;

static int check_common(const fvm_mesh_t* mesh) {
    if (mesh && mesh->dim >= 2 && mesh->dim <= 3 && mesh->kg > FVM_MAX_KG) return FVM_E_UNSUPPORTED;
    return mesh_ok(mesh) ? FVM_OK : FVM_E_ARG;
}

extern "C" int fvm_residual(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const float* prims,
                            float* grads, int32_t* has_grads, float* dudt, const fvm_work_t* work,
                            void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !prims || !grads || !has_grads || !dudt || !work_ok(mesh, work) || !work->prims ||
        !aligned32(work->prims) || !aligned32(grads))
        return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t s = (cudaStream_t)stream;
    return mesh->dim == 2 ? residual_impl<2>(mesh, p, prims, grads, has_grads, dudt, work, s)
                          : residual_impl<3>(mesh, p, prims, grads, has_grads, dudt, work, s);
}

extern "C" int fvm_residual_state(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const float* state,
                                  float* grads, int32_t* has_grads, float* dudt, const fvm_work_t* work,
                                  void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !state || !grads || !has_grads || !dudt || !work_ok(mesh, work) || !work->prims ||
        !aligned32(work->prims) || !aligned32(grads))
        return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t s = (cudaStream_t)stream;
    return mesh->dim == 2 ? residual_state_impl<2>(mesh, p, state, grads, has_grads, dudt, work, s)
                          : residual_state_impl<3>(mesh, p, state, grads, has_grads, dudt, work, s);
}

extern "C" int fvm_facet_values(const fvm_mesh_t* mesh, const float* prims_padded, const float* grads,
                                const fvm_work_t* work, float* out, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!prims_padded || !grads || !out || !work || (mesh->n_bc > 0 && !work->bc_vals) || !aligned32(prims_padded) ||
        !aligned32(grads))
        return FVM_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (mesh->dim == 2)
        FVM_LAUNCH(KID_FACE, s, k_facet_values<2><<<blocks_for(mesh->n_facets), kBlock, 0, s>>>(
                                    *mesh, prims_padded, work->bc_vals, grads, out));
    else
        FVM_LAUNCH(KID_FACE, s, k_facet_values<3><<<blocks_for(mesh->n_facets), kBlock, 0, s>>>(
                                    *mesh, prims_padded, work->bc_vals, grads, out));
    return launch_status();
}

// ------------------------------------------------------------------------------------------
// Allocation-free residual (fvm_residual_noalloc).
//
// Some callers cannot allocate device memory where they call the residual: an application whose
// own pool allocator has already reserved the GPU's memory, or a time-critical loop that forbids
// allocation once it runs (cudaMalloc / cudaFree can also wait for the whole device to go idle,
// stalling unrelated streams).  This variant takes its scratch -- boundary values, padded
// primitives and fluxes (plus per-case slots of batched meshes) -- from one file-scope device array
// of FVM_NOALLOC_SCRATCH_BYTES, which every GPU that loads this library keeps until the process
// exits.  The residual overwrites every scratch element it reads before reading it, so nothing has
// to be cleared between calls.  All calls on a device share the array: calls that overlap on the
// GPU (different streams, or different host threads) race and must be serialised by the caller.
// ------------------------------------------------------------------------------------------
constexpr int64_t kNoAllocFloats = FVM_NOALLOC_SCRATCH_BYTES / 4;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

static constexpr int kMaxDevices = 64;
static float* g_noalloc_dev_ptr[kMaxDevices];   // device address of g_noalloc_scratch, per device

// The symbol's device address, looked up once per device with that device current (host code may
// not use the symbol's name as an address) and kept for the life of the process: a
// cudaDeviceReset on that device would leave the kept address naming freed memory, which the
// header rules out for callers.  Returns nullptr on failure.
static float* noalloc_scratch_address() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    float* p = __atomic_load_n(&g_noalloc_dev_ptr[dev], __ATOMIC_ACQUIRE);
    if (p) return p;
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || addr == nullptr) return nullptr;
    __atomic_store_n(&g_noalloc_dev_ptr[dev], static_cast<float*>(addr), __ATOMIC_RELEASE);
    return static_cast<float*>(addr);
}

static inline int64_t align64(int64_t n) { return (n + 63) / 64 * 64; }   // 256-byte units of floats

static bool bufs_ok(const fvm_solver_bufs_t* b) {
    return b && b->state && b->prims && b->grads && b->k && b->dt && b->has_grads && aligned32(b->prims) &&
           aligned32(b->grads);
}

static bool tab_ok(const fvm_tableau_t* t) { return t && t->stages >= 1 && t->stages <= FVM_MAX_STAGES; }

extern "C" int fvm_stage(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const fvm_tableau_t* tab,
                         int32_t s, const fvm_solver_bufs_t* bufs, const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !tab_ok(tab) || s < 0 || s >= tab->stages || !bufs_ok(bufs) || !work_ok(mesh, work))
        return FVM_E_ARG;
    if (mesh->n_cases > 0 && tab->adaptive) return FVM_E_UNSUPPORTED;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? stage_impl<2>(mesh, p, tab, s, bufs, work, st)
                          : stage_impl<3>(mesh, p, tab, s, bufs, work, st);
}

extern "C" int fvm_step(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const fvm_tableau_t* tab,
                        const fvm_solver_bufs_t* bufs, const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !tab_ok(tab) || !bufs_ok(bufs) || !work_ok(mesh, work)) return FVM_E_ARG;
    if (mesh->n_cases > 0 && tab->adaptive) return FVM_E_UNSUPPORTED;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    for (int s = 0; s < tab->stages; ++s) {
        const int rc = mesh->dim == 2 ? stage_impl<2>(mesh, p, tab, s, bufs, work, st)
                                      : stage_impl<3>(mesh, p, tab, s, bufs, work, st);
        if (rc) return rc;
    }
    return FVM_OK;
}

extern "C" int fvm_char_partial(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const float* prims,
                                const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !prims || !work || !work->red || mesh->n_cases > 0) return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    if (mesh->dim == 2)
        FVM_LAUNCH(KID_BC, st, k_char_partial<2><<<1, kBlock, 0, st>>>(*mesh, p, prims, work->red));
    else
        FVM_LAUNCH(KID_BC, st, k_char_partial<3><<<1, kBlock, 0, st>>>(*mesh, p, prims, work->red));
    return launch_status();
}

extern "C" int fvm_stage_begin(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const fvm_solver_bufs_t* bufs,
                               const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !bufs_ok(bufs) || !work_ok(mesh, work)) return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? launch_begin<2>(mesh, p, bufs->prims, bufs->grads, bufs->has_grads, work, st)
                          : launch_begin<3>(mesh, p, bufs->prims, bufs->grads, bufs->has_grads, work, st);
}

extern "C" int fvm_stage_end(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const fvm_tableau_t* tab, int32_t s,
                             const fvm_solver_bufs_t* bufs, const fvm_work_t* work, int32_t finalize, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !tab_ok(tab) || s < 0 || s >= tab->stages || !bufs_ok(bufs) || !work_ok(mesh, work))
        return FVM_E_ARG;
    if (mesh->n_cases > 0 && tab->adaptive) return FVM_E_UNSUPPORTED;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? stage_finish<2>(mesh, p, tab, s, bufs, work, finalize != 0, st)
                          : stage_finish<3>(mesh, p, tab, s, bufs, work, finalize != 0, st);
}

extern "C" int fvm_stage_phase(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const fvm_tableau_t* tab,
                               int32_t s, const fvm_solver_bufs_t* bufs, const fvm_work_t* work, int32_t phases,
                               int32_t finalize, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !tab_ok(tab) || s < 0 || s >= tab->stages || !bufs_ok(bufs) || !work_ok(mesh, work) ||
        phases <= 0 || phases > 15)
        return FVM_E_ARG;
    if (mesh->n_cases > 0 && tab->adaptive) return FVM_E_UNSUPPORTED;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? stage_phase_impl<2>(mesh, p, tab, s, bufs, work, phases, finalize != 0, st)
                          : stage_phase_impl<3>(mesh, p, tab, s, bufs, work, phases, finalize != 0, st);
}

extern "C" int fvm_stage_finalize(const fvm_mesh_t* mesh, const fvm_tableau_t* tab, const fvm_solver_bufs_t* bufs,
                                  const fvm_work_t* work, void* stream) {
    if (!mesh_ok(mesh) || !tab_ok(tab) || !bufs_ok(bufs) || !work || !work->red) return FVM_E_ARG;
    if (!(tab->adaptive || tab->cfl > 0.f || bufs->cons)) return FVM_OK;
    return finalize_impl(mesh, tab, bufs, work, bufs->cons != nullptr, (cudaStream_t)stream);
}

extern "C" int fvm_multistep(const fvm_mesh_t* mesh, const fvm_physics_t* phys, int32_t store,
                             int32_t n_terms, const int32_t* idx, const float* coef,
                             const fvm_solver_bufs_t* bufs, const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !bufs_ok(bufs) || !work_ok(mesh, work) || n_terms < 0 ||
        n_terms > FVM_MAX_STAGES || (n_terms > 0 && (!idx || !coef)) || store < 0)
        return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? multistep_impl<2>(mesh, p, store, n_terms, idx, coef, bufs, work, st)
                          : multistep_impl<3>(mesh, p, store, n_terms, idx, coef, bufs, work, st);
}

// Barrier words and status of the fused step live in work->red[60], [61] (slots no reduction uses).
static unsigned* fused_bar(const fvm_work_t* w) { return reinterpret_cast<unsigned*>(w->red + 60); }
static int* fused_status(const fvm_work_t* w) { return reinterpret_cast<int*>(w->red + 61); }

template <int DIM>
static int fused_impl(const fvm_mesh_t* m, const Phys& p, FusedArgs& f, cudaStream_t st) {
    static int blocks_per_sm[2] = {-1, -1}, sms = 0;
    int& bps = blocks_per_sm[DIM - 2];
    if (bps < 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_step_fused<DIM>, kBlock, 0) != cudaSuccess) {
            bps = -1;
            launch_status();
            return FVM_E_CUDA;
        }
    }
    if (bps < 1) return FVM_E_UNSUPPORTED;
    // enough blocks for the largest phase, at most all co-resident ones
    const int64_t items = std::max<int64_t>({(int64_t)owned_cells(m), (int64_t)m->n_facets, (int64_t)m->n_bc});
    const unsigned grid = (unsigned)std::min<int64_t>((int64_t)bps * sms, std::max<int64_t>(1, (items + kBlock - 1) / kBlock));
    fvm_mesh_t mc = *m;
    void* args[] = {&mc, const_cast<Phys*>(&p), &f};
    if (cudaMemsetAsync(f.bar, 0, sizeof(unsigned), st) != cudaSuccess) {   // arrivals start at zero
        launch_status();
        return FVM_E_CUDA;
    }
    prof_begin(KID_FUSED, st);
    const cudaError_t e =
        cudaLaunchCooperativeKernel((const void*)k_step_fused<DIM>, dim3(grid), dim3(kBlock), args, 0, st);
    prof_end(st);
    if (e != cudaSuccess) {
        launch_status();
        return FVM_E_CUDA;
    }
    return launch_status();
}

static void fill_fused(FusedArgs& f, const fvm_tableau_t* tab, const fvm_solver_bufs_t* b, const fvm_work_t* w) {
    f.need_final = tab->adaptive || tab->cfl > 0.f || b->cons != nullptr;
    f.adaptive = tab->adaptive;
    f.atol = tab->atol; f.rtol = tab->rtol; f.mtol = tab->mtol;
    f.alpha_hi = tab->alpha_hi_err; f.alpha_lo = tab->alpha_lo_err; f.order = tab->order; f.cfl = tab->cfl;
    f.state = b->state; f.prims = b->prims; f.grads = b->grads; f.has_grads = b->has_grads; f.k = b->k;
    f.dt = b->dt; f.cons = b->cons; f.bcv = w->bc_vals; f.flux = w->flux; f.red = w->red;
    f.bar = fused_bar(w); f.status = fused_status(w);
}

extern "C" int fvm_step_fused(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const fvm_tableau_t* tab,
                              const fvm_solver_bufs_t* bufs, const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !tab_ok(tab) || !bufs_ok(bufs) || !work_ok(mesh, work)) return FVM_E_ARG;
    if (mesh->n_cases > 0 && tab->adaptive) return FVM_E_UNSUPPORTED;
    if (mesh->n_owned > 0 || mesh->char_scale_given) return FVM_E_UNSUPPORTED;   // partitions use the split stages
    if (mesh->cell_lo || mesh->facet_lo) return FVM_E_UNSUPPORTED;
    FusedArgs f{};
    f.stages = tab->stages;
    for (int s = 0; s < tab->stages; ++s) {
        f.st[s] = stage_args(tab, s);
        f.st[s].cons = f.st[s].final_ && bufs->cons != nullptr;
    }
    fill_fused(f, tab, bufs, work);
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? fused_impl<2>(mesh, p, f, st) : fused_impl<3>(mesh, p, f, st);
}

extern "C" int fvm_multistep_fused(const fvm_mesh_t* mesh, const fvm_physics_t* phys, int32_t store, int32_t n_terms,
                                   const int32_t* idx, const float* coef, const fvm_solver_bufs_t* bufs,
                                   const fvm_work_t* work, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !bufs_ok(bufs) || !work_ok(mesh, work) || n_terms < 0 || n_terms > FVM_MAX_STAGES ||
        (n_terms > 0 && (!idx || !coef)) || store < 0)
        return FVM_E_ARG;
    if (mesh->n_owned > 0 || mesh->char_scale_given || mesh->cell_lo || mesh->facet_lo) return FVM_E_UNSUPPORTED;
    FusedArgs f{};
    f.stages = 1;
    StageArgs& a = f.st[0];
    a.s = store;
    a.store_k = 1;
    a.final_ = 1;
    a.n_terms = n_terms;
    for (int t = 0; t < n_terms; ++t) {
        a.idx[t] = idx[t];
        a.coef[t] = coef[t];
    }
    a.cons = bufs->cons != nullptr;
    fvm_tableau_t tab{};
    tab.stages = 1;
    tab.order = 1.f;
    fill_fused(f, &tab, bufs, work);
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    return mesh->dim == 2 ? fused_impl<2>(mesh, p, f, st) : fused_impl<3>(mesh, p, f, st);
}

extern "C" int fvm_barrier_selftest(int32_t blocks, int32_t skip_block, int32_t* status) {
    if (blocks < 2 || blocks > 64 || skip_block >= blocks || !status) return FVM_E_ARG;
    unsigned* d = nullptr;   // [0] arrivals, [1] generation, [2] status
    if (cudaMalloc(&d, 3 * sizeof(unsigned)) != cudaSuccess || cudaMemset(d, 0, 3 * sizeof(unsigned)) != cudaSuccess) {
        launch_status();
        if (d) cudaFree(d);
        return FVM_E_CUDA;
    }
    unsigned* bar = d;
    int* st = reinterpret_cast<int*>(d + 2);
    int skip = skip_block;
    long long limit = 1LL << 16;            // ~5 ms of polling: the test's waits run out quickly
    void* args[] = {&bar, &st, &skip, &limit};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_barrier_selftest, dim3(blocks), dim3(64), args, 0, 0);
    if (e == cudaSuccess) e = cudaMemcpy(status, st, sizeof(int32_t), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        launch_status();
        return FVM_E_CUDA;
    }
    return FVM_OK;
}

extern "C" int fvm_fused_status(const fvm_work_t* work, int32_t* status) {
    if (!work || !work->red || !status) return FVM_E_ARG;
    if (cudaMemcpy(status, fused_status(work), sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
        launch_status();
        return FVM_E_CUDA;
    }
    return FVM_OK;
}

extern "C" int fvm_state_to_prims(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const float* state,
                                  float* prims, void* stream) {
    if (!mesh_ok(mesh) || !phys || !state || !prims || !aligned32(prims)) return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    if (mesh->dim == 2)
        FVM_LAUNCH(KID_STATE_TO_PRIMS, st, launch(k_state_to_prims<2>, dim3(blocks_for(owned_cells(mesh))), dim3(kBlock), 0, st, 
                                               owned_cells(mesh), p.inv_Cv, state, prims));
    else
        FVM_LAUNCH(KID_STATE_TO_PRIMS, st, launch(k_state_to_prims<3>, dim3(blocks_for(owned_cells(mesh))), dim3(kBlock), 0, st, 
                                               owned_cells(mesh), p.inv_Cv, state, prims));
    return launch_status();
}

extern "C" int fvm_cfl_dt(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const float* state, float cfl,
                          float* dt, const fvm_work_t* work, void* stream) {
    if (!mesh_ok(mesh) || !phys || !state || !dt || !work || !work->red || !(cfl > 0.f)) return FVM_E_ARG;
    const Phys p = make_phys(phys);
    cudaStream_t st = (cudaStream_t)stream;
    if (mesh->dim == 2)
        FVM_LAUNCH(KID_REDUCE_STATE, st, k_reduce_state<2><<<reduce_grid<2>(mesh), kBlock, 0, st>>>(
                                             *mesh, p, state, 1, 0, work->red));
    else
        FVM_LAUNCH(KID_REDUCE_STATE, st, k_reduce_state<3><<<reduce_grid<3>(mesh), kBlock, 0, st>>>(
                                             *mesh, p, state, 1, 0, work->red));
    int rc = launch_status();
    if (rc) return rc;
    FVM_LAUNCH(KID_FINALIZE, st, launch(k_finalize, dim3(fin_blocks(mesh)), dim3(128), 0, st, mesh->n_comp, 0, 0.f, 0.f, 0.f, 0.f,
                                                                             0.f, 1.f, cfl, 0, work->red, dt,
                                                                             nullptr, mesh->n_cases, nullptr));
    return launch_status();
}

extern "C" int fvm_conservation(const fvm_mesh_t* mesh, const float* state, double* out, const fvm_work_t* work,
                                void* stream) {
    if (!mesh_ok(mesh) || !state || !out || !work || !work->red) return FVM_E_ARG;
    Phys p{};
    cudaStream_t st = (cudaStream_t)stream;
    if (mesh->dim == 2)
        FVM_LAUNCH(KID_REDUCE_STATE, st, k_reduce_state<2><<<reduce_grid<2>(mesh), kBlock, 0, st>>>(
                                             *mesh, p, state, 0, 1, work->red));
    else
        FVM_LAUNCH(KID_REDUCE_STATE, st, k_reduce_state<3><<<reduce_grid<3>(mesh), kBlock, 0, st>>>(
                                             *mesh, p, state, 0, 1, work->red));
    int rc = launch_status();
    if (rc) return rc;
    FVM_LAUNCH(KID_FINALIZE, st, launch(k_finalize, dim3(fin_blocks(mesh)), dim3(128), 0, st, mesh->n_comp, 0, 0.f, 0.f, 0.f, 0.f,
                                                                             0.f, 1.f, 0.f, 1, work->red, nullptr,
                                                                             out, mesh->n_cases, nullptr));
    return launch_status();
}

extern "C" int fvm_residual_noalloc(const fvm_mesh_t* mesh, const fvm_physics_t* phys, const float* prims,
                                    float* grads, int32_t* has_grads, float* dudt, void* stream) {
    if (const int rc = check_common(mesh)) return rc;
    if (!phys || !prims || !grads || !has_grads || !dudt || !aligned32(grads)) return FVM_E_ARG;
    if (mesh->char_scale_given) return FVM_E_ARG;   // its scratch holds no per-part slots
    const int64_t R = FVM_ROW(mesh->dim);
    const int64_t n_bc = align64((int64_t)mesh->n_bc * R);
    const int64_t n_prims = align64((int64_t)mesh->n_cells * R);
    const int64_t n_flux = align64((int64_t)mesh->n_facets * R);
    const int64_t n_red = align64(2 * ((int64_t)FVM_RED_DOUBLES + 8 * (int64_t)mesh->n_cases));
    if (n_bc + n_prims + n_flux + n_red > kNoAllocFloats) return FVM_E_CAPACITY;
    float* base = noalloc_scratch_address();
    if (!base) {
        launch_status();
        return FVM_E_CUDA;
    }
    fvm_work_t w;
    w.bc_vals = base;
    w.prims = base + n_bc;
    w.flux = base + n_bc + n_prims;
    w.red = reinterpret_cast<double*>(base + n_bc + n_prims + n_flux);
    const Phys p = make_phys(phys);
    cudaStream_t s = (cudaStream_t)stream;
    return mesh->dim == 2 ? residual_impl<2>(mesh, p, prims, grads, has_grads, dudt, &w, s)
                          : residual_impl<3>(mesh, p, prims, grads, has_grads, dudt, &w, s);
}

extern "C" int fvm_set_prefetch(int32_t kernel_id, int32_t waves_ahead) {
    if (waves_ahead < -1 || waves_ahead > 8) return FVM_E_ARG;
    switch (kernel_id) {
        case KID_CELL: g_pf_cell = waves_ahead; return FVM_OK;
        case KID_FACE: g_pf_face = waves_ahead; return FVM_OK;
        case KID_DIV_STAGE: g_pf_div = waves_ahead; return FVM_OK;
        default: return FVM_E_ARG;
    }
}

extern "C" int fvm_set_variant(int32_t kernel_id, int32_t variant) {
    if ((kernel_id != KID_FACE && kernel_id != KID_DIV_STAGE) || variant < 0 || variant > 1) return FVM_E_ARG;
    (kernel_id == KID_FACE ? g_face_variant : g_div_variant) = variant;
    return FVM_OK;
}

extern "C" int fvm_set_block_size(int32_t kernel_id, int32_t threads) {
    if (threads < 64 || threads > kMaxBlock || threads % 32 != 0) return FVM_E_ARG;
    switch (kernel_id) {
        case KID_CELL: g_block_cell = threads; return FVM_OK;
        case KID_FACE: g_block_face = threads; return FVM_OK;
        case KID_DIV_STAGE: g_block_div = threads; return FVM_OK;
        default: return FVM_E_ARG;
    }
}
