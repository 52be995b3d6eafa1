/*
 * fvm_b200.h -- C ABI of the B200 finite-volume residual library (libfvm_b200.so).
 *
 * All pointers are device pointers unless stated otherwise; all arrays are dense and
 * row-major as documented per field.  Every entry point returns 0 on success or a negative
 * FVM_E_* code (the CUDA launch error, if any, is folded into FVM_E_CUDA and can be read
 * with fvm_last_cuda_error()).  Work is enqueued on `stream` (a cudaStream_t passed as
 * void*, NULL = legacy default stream); nothing synchronises the host.
 *
 * The reference (Merlotec/fvm_solver) is Python; the interfaces replaced here are its
 * sparse-operator seam and its residual / integrator seam:
 *   fvm_ell_spmv / fvm_ell_spmm   <- time_fvm/utils/ell_kernel.py:135 (ell_spmv),
 *                                    :176 (ell_spmm); called through SPM.spMV / SPM.spMM
 *                                    (time_fvm/utils/sparse.py:14-21, 34-38)
 *   fvm_residual                  <- FVMEquation.forward (time_fvm/fvm_equation.py:406-435),
 *                                    including FacetCalc.compute_facet
 *                                    (time_fvm/fvm_stepping/facet_process.py:332-385)
 *   fvm_stage / fvm_step          <- Butcher._step / ButcherAdapt._step / RK3_SSP4._step and
 *                                    Adaptive.update_stepsize
 *                                    (time_fvm/time_solvers/integrators.py:42-94, 322-393)
 *   fvm_cfl_dt                    <- no reference counterpart (CFL time step, FP64 reduction)
 *   fvm_conservation              <- no reference counterpart (FP64 sum of vol * U)
 */
#ifndef FVM_B200_H
#define FVM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FVM_OK 0
#define FVM_E_ARG (-1)      /* invalid argument (null pointer, size out of range) */
#define FVM_E_CUDA (-2)     /* a CUDA launch failed; see fvm_last_cuda_error() */
#define FVM_E_UNSUPPORTED (-3)
#define FVM_E_CAPACITY (-4)    /* the mesh needs more scratch than fvm_residual_noalloc has */

#define FVM_MAX_STAGES 12
#define FVM_MAX_KG 16
#define FVM_MAX_ELL_K 16    /* widest ELL row fvm_ell_spmv / fvm_ell_spmm take (FVM_E_UNSUPPORTED above) */
#define FVM_RED_DOUBLES 64
#define FVM_NOALLOC_SCRATCH_BYTES (16 * 1024 * 1024)

/* Row layouts.  Records and gathered rows are padded so every row is read and written with
 * 32-byte (or, for 4-float rows, 16-byte) vector accesses; all row arrays must be 32-byte aligned:
 *   primitives, fluxes, boundary values: FVM_ROW(dim) floats per row (4 in 2D, 8 in 3D), the first
 *     C = dim + 2 used (V..., rho, T for primitives; the conserved order for fluxes);
 *   limited gradients: FVM_GROW(dim) floats per cell (8 / 16); entry (d, V_k) at d*(dim+1) + k,
 *     (d, T) at d*(dim+1) + dim, (d, rho) at dim*(dim+1) + d;
 *   state and stage increments keep the plain [N][C] layout. */
#define FVM_ROW(dim) ((dim) == 2 ? 4 : 8)
#define FVM_GROW(dim) ((dim) == 2 ? 8 : 16)
#define FVM_CELL_REC(dim) ((dim) == 2 ? 20 : 32)
/* Cell record width of a mesh with kg gradient slots (kg = dim + 2: FVM_CELL_REC). */
#define FVM_CELL_REC_KG(dim, kg) ((((dim) * (kg) + (kg) + ((dim) + 1) * (dim) + 2) + 7) / 8 * 8)
#define FVM_FACE_REC(dim) ((dim) == 2 ? 16 : 16)
#define FVM_DIV_REC 8

/* Mesh tables (built by fvm_solver_b200/tables.py).  N cells, F facets, Fb boundary facets,
 * Fc characteristic facets, K = dim + 1 facets per cell, KG = kg gradient slots: dim + 2 (the
 * reference's face-neighbour stencil) up to FVM_MAX_KG (a widened stencil); the cell record is then
 * FVM_CELL_REC_KG(dim, kg) floats wide.
 * Integer fields inside float records are stored bit-cast (int32 bits in a float slot). */
typedef struct fvm_mesh {
    int32_t dim, n_comp, n_cells, n_facets, n_bc, n_char, kg, kf;
    /* Cell records.  kg = dim + 2 (the reference's stencil): [N][FVM_CELL_REC] = the KG - 1
     * neighbour columns in slot order (into [cells ; boundary facets]; bits 28..30 of the first
     * hold the slot of the cell itself, whose column is its own index), padded to 4 slots, then
     * LSQ gradient weights [dim][KG] in slot order, centroid->facet displacements [K][dim],
     * limiter epsilon.
     * kg > dim + 2: [N][FVM_CELL_REC_KG] = weights [dim][KG], columns [KG], displacements, epsilon,
     * meta (bits 4j..4j+3: slot of face neighbour j; bits 24..28: valid slots), padding. */
    const float *cell_rec;
    /* [N][FVM_DIV_REC]: divergence weights +-1/vol [K], facet indices [K] */
    const float *div_rec;
    const double *inv_h;      /* [N] max facet area / volume (CFL)                          */
    const double *volumes;    /* [N]                                                        */
    /* [F][FVM_FACE_REC]: side-0 cell, side-1 cell (a boundary side holds -1 - boundary index),
     * +-1/d (negative when the side-1 cell has the lower index: the order in which the facet's
     * normal-gradient row sums its two terms), |S|, area normal [dim], non-orthogonal correction
     * vector [dim], centroid->facet
     * displacement of side 0 [dim] and of side 1 [dim] */
    const float *face_rec;
    /* boundary facets */
    const int32_t *bc_cell;   /* [Fb] adjacent cell                                         */
    const int32_t *bc_kind;   /* [Fb][C] 1 Dirichlet, 2 Neumann, 0 other                    */
    const float *bc_b;        /* [Fb][C] face-value offset                                  */
    const float *bc_l;        /* [Fb][dim] tangential lever arm (non-orthogonal correction) */
    const float *bc_ga;       /* [Fb][C] face-gradient coefficient                          */
    const float *bc_gb;       /* [Fb][C] face-gradient offset                               */
    const int32_t *bc_char;   /* [Fb] index into the characteristic arrays or -1             */
    const int32_t *ch_cell;   /* [Fc] cell adjacent to each characteristic facet             */
    const float *ch_normal;   /* [Fc][dim] outward unit normals                             */
    const float *ch_rho, *ch_vn, *ch_p;            /* [Fc]                                  */
    const float *ch_vt;       /* [Fc][dim]                                                  */
    /* Batched meshes: n_cases > 0 means the tables are several independent meshes
     * concatenated (cells, facets, boundary and characteristic facets each contiguous per
     * case, all indices global).  Each case has its own time step (dt[case]), gas transport
     * coefficients, characteristic-BC sound-speed mean, CFL and conservation reductions.
     * n_cases = 0 and NULL pointers: a single mesh. */
    int32_t n_cases;
    const int32_t *cell_case; /* [N]  case of each cell                                     */
    const int32_t *face_case; /* [F]  case of each facet                                    */
    const int32_t *bc_case;   /* [Fb] case of each boundary facet                           */
    const int32_t *ch_off;    /* [n_cases + 1] characteristic-facet offsets per case         */
    const float *case_mu, *case_mu_b, *case_kappa;   /* [n_cases] transport coefficients    */
    /* Partitioned meshes (one part of a mesh split across ranks, single mesh only): cells
     * [0, n_owned) are this part's own cells, [n_owned, n_cells) a one-cell-deep halo of copies
     * of other parts' cells.  Gradients, divergences, stage updates and the CFL / conservation
     * reductions cover owned cells only; the halo's primitives and limited gradients are written
     * by the caller's exchange.  0 = every cell owned.  char_scale_given = 1: the
     * characteristic-BC scale 10 / mean(c) is read from work->red[FVM_RED_DOUBLES + 6] (the
     * caller forms it from every part's fvm_char_partial) instead of being computed here. */
    int32_t n_owned;
    int32_t char_scale_given;
    /* Batched meshes only: [n_cases] bytes, 0 = the case is frozen -- its boundary facets, cells and
     * facets are skipped by every kernel and its dt / conservation slots are left alone (a
     * corrector's fallback advances only the cases whose proposal failed).  NULL = all active. */
    const uint8_t *case_active;
    /* Sub-ranges (single meshes only; 0 = from the start): the cell kernel updates cells
     * [cell_lo, n_owned or n_cells), the facet kernel evaluates facets [facet_lo, n_facets) --
     * with n_owned / n_facets lowered in a copy of the struct a caller runs any contiguous range,
     * e.g. a part's inner cells and facets while its halo exchange is in flight. */
    int32_t cell_lo;
    int32_t facet_lo;
} fvm_mesh_t;

/* Gas and scheme constants (ConfigFVM fields, time_fvm/config_fvm.py:52-63). */
typedef struct fvm_physics {
    float T_0, mu, mu_b, S_const, C_v, gamma, kappa, v_factor;
    int32_t lim_p;
} fvm_physics_t;

/* Caller-owned scratch for one mesh. */
typedef struct fvm_work {
    float *bc_vals;     /* [Fb][FVM_ROW] boundary facet values                          */
    float *prims;       /* [N][FVM_ROW] padded primitives (used by fvm_residual only)   */
    float *flux;        /* [F][FVM_ROW] facet fluxes                                    */
    double *red;        /* [FVM_RED_DOUBLES + 8 * n_cases], zero-initialised once; a partitioned
                         * mesh (char_scale_given, fvm_char_partial) needs FVM_RED_DOUBLES + 8 */
} fvm_work_t;

/* Explicit Runge-Kutta tableau (optionally with an embedded low-order row). */
typedef struct fvm_tableau {
    int32_t stages;
    float a[FVM_MAX_STAGES][FVM_MAX_STAGES];
    float b[FVM_MAX_STAGES];
    float b2[FVM_MAX_STAGES];
    int32_t adaptive;                 /* 1: Adaptive.update_stepsize after the step            */
    float atol, rtol, mtol, alpha_hi_err, alpha_lo_err, order;
    float cfl;                        /* > 0: dt = cfl * min h / (|u| + c) after the step      */
} fvm_tableau_t;

/* Time-stepping buffers (caller-owned). */
typedef struct fvm_solver_bufs {
    float *state;       /* [N][C] conserved state, updated in place                      */
    float *prims;       /* [N][FVM_ROW] primitives of the current stage input             */
    float *grads;       /* [N][FVM_GROW] limited gradients, carried across evaluations    */
    float *k;           /* [stages][N][C] stage increments dt * f                          */
    float *dt;          /* [max(1, n_cases)] time step per case (device)                  */
    int32_t *has_grads; /* [1] device flag: grads hold a previous evaluation              */
    double *cons;       /* [max(1, n_cases)][C] optional: FP64 sum of vol * U after each step
                         * (may be NULL)                                                  */
} fvm_solver_bufs_t;

/* Last CUDA error recorded by this library (cudaError_t value), 0 if none. */
int fvm_last_cuda_error(void);
/* Library build identifier, e.g. "fvm_b200 sm_100a". Host string. */
const char *fvm_version(void);

/* Launch profiling (no reference counterpart).  Between fvm_profile_start(capacity) and
 * fvm_profile_stop() every kernel this library launches is bracketed by two CUDA events recorded
 * on its stream (also when the launches are captured into a CUDA graph).  fvm_profile_stop returns
 * the number of launches recorded (FVM_E_ARG if more than `capacity` were attempted);
 * fvm_profile_read fills host arrays with each launch's kernel id and duration in ms, waiting for
 * the events.  Kernel ids: 0 ell_spmv, 1 ell_spmm, 2 bc, 3 cell, 4 face, 5 div_stage,
 * 6 finalize, 7 state_to_prims, 8 reduce_state, 9 batched, 10 corrector, 11 fused step. */
int fvm_profile_start(int32_t capacity);
/* Kernel variant (no reference counterpart; results unchanged): for the facet kernel
 * (kernel_id 4), 0 = each thread loads its facet record, 1 = the records of a block's next tile
 * are staged in shared memory by the bulk-copy unit (cp.async.bulk + mbarrier, two stages); for
 * the divergence kernel (kernel_id 5), 1 = residual evaluations (fvm_residual, fvm_residual_state
 * on a whole mesh) compute each cell's facet fluxes in the divergence kernel itself (owner computes:
 * no flux array, every interior facet evaluated from both sides), 0 = facet kernel then divergence
 * kernel; stages always use 0. */
int fvm_set_variant(int32_t kernel_id, int32_t variant);
/* Launch overlap (no reference counterpart; results unchanged; default 1): 1 = the boundary,
 * cell, facet, divergence, conversion and finalisation kernels are launched with programmatic
 * stream serialisation, so each is launched while the previous kernel of its stream (or CUDA
 * graph) drains and waits on the device (griddepcontrol.wait) for that kernel's completion and
 * writes; 0 = plain stream order. */
int fvm_set_launch_overlap(int32_t on);
/* Launch configuration (no reference counterpart): threads per block of the cell (id 3), facet
 * (id 4) and divergence/stage (id 5) kernels for all later launches of this process; a multiple
 * of 32 in [64, 512].  Results do not depend on it (each thread's arithmetic is unchanged); the
 * autotuner (fvm_solver_b200/autotune.py) picks it per mesh. */
int fvm_set_block_size(int32_t kernel_id, int32_t threads);
/* Record prefetch (no reference counterpart): for the same kernel ids, each block has the bulk-copy
 * unit prefetch into L2 the records (and, for the stage kernel, the state rows) it or another block
 * will read `waves_ahead` waves of resident blocks later; -1 = the default (0), 0 = off, at most 8.
 * Results do not depend on it. */
int fvm_set_prefetch(int32_t kernel_id, int32_t waves_ahead);
int fvm_profile_stop(void);
int fvm_profile_read(int32_t n, int32_t *ids, float *ms);

/* y[M] = A x (+ bias).  A in slot-major ELL: vals[K][M], cols[K][M] (int32).  x is read with
 * stride incx, y written with stride incy.  bias may be NULL. */
int fvm_ell_spmv(const float *vals, const int32_t *cols, int64_t M, int32_t K,
                 const float *x, int64_t incx, const float *bias, float *y, int64_t incy,
                 void *stream);

/* Y[M][B] = A X (+ bias[:, None]).  X is [N][B] with leading dimension ldx, Y [M][B] with ldy. */
int fvm_ell_spmm(const float *vals, const int32_t *cols, int64_t M, int32_t K,
                 const float *X, int64_t ldx, int32_t B, const float *bias, float *Y, int64_t ldy,
                 void *stream);

/* dU/dt [N][C] (conserved variables) of the primitives prims [N][C].  grads [N][FVM_GROW] is
 * read as the previous limited gradient when the device flag *has_grads != 0 (the reference's
 * FacetCalc.cell_grads is not None) and overwritten with this evaluation's limited gradient;
 * the call sets *has_grads = 1.  Meshes with kg > dim + 2 take the generic-width cell kernel. */
int fvm_residual(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const float *prims,
                 float *grads, int32_t *has_grads, float *dudt, const fvm_work_t *work,
                 void *stream);

/* dU/dt of a conserved state [N][C] (no reference counterpart: the reference converts with
 * FluidConstitution.state_to_primative, fvm_equation.py:35-44, before FVMEquation.forward): one
 * kernel converts to padded primitives in work->prims (the stage kernels' arithmetic), then the
 * residual as fvm_residual. */
int fvm_residual_state(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const float *state, float *grads,
                       int32_t *has_grads, float *dudt, const fvm_work_t *work, void *stream);

/* Both sides' limited facet values out[F][2][C] -- the reference's U_face_all, split by
 * FacetCalc.compute_facet into Vs_facet / rho_facet / T_facet (facet_process.py:349-359) -- for
 * the padded primitives, limited gradients and boundary values (work->bc_vals) of the last
 * residual evaluation on them; exactly the values the facet kernel uses.  On demand only. */
int fvm_facet_values(const fvm_mesh_t *mesh, const float *prims_padded, const float *grads, const fvm_work_t *work,
                     float *out, void *stream);

/* Allocation-free fvm_residual.  No counterpart in the reference: it exists for callers that
 * cannot allocate device memory where they call the residual -- an application whose own pool
 * allocator has already reserved the GPU's memory, or a time-critical loop that forbids
 * allocation once it runs (cudaMalloc / cudaFree can also wait for the device to go idle).
 * Same arguments and results as fvm_residual, minus `work`: the scratch (boundary values,
 * padded primitives, fluxes) lives in one static device array of FVM_NOALLOC_SCRATCH_BYTES
 * (16 MiB) that every GPU loading the library keeps until the process exits.  A mesh whose
 * scratch does not fit -- 4 * (align64(Fb*R) + align64(N*R) + align64(F*R)
 * + align64(2*(64 + 8*n_cases))) bytes with R = FVM_ROW(dim), i.e. up to about 340 000 facets
 * (170 000 tetrahedra) in 3D or 600 000 facets (400 000 triangles) in 2D -- is rejected with
 * FVM_E_CAPACITY before anything is launched; a partitioned mesh with char_scale_given = 1 is
 * rejected with FVM_E_ARG (the scratch has no per-part slots).  The function never allocates;
 * the first call on each device looks up the array's device address (with that device
 * current) and keeps it for the life of the process, so make that first call before any stream
 * capture, and do not call this function on a device after cudaDeviceReset in the same process
 * (the kept address would name freed memory).  Every call overwrites the
 * scratch it reads, so no clearing is needed; all calls on a device share the array, so calls
 * that overlap on the GPU race and must be serialised by the caller. */
int fvm_residual_noalloc(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const float *prims,
                         float *grads, int32_t *has_grads, float *dudt, void *stream);

/* Fused step (no reference counterpart): the whole of fvm_step (all stages) -- or of
 * fvm_multistep -- in one cooperative launch of co-resident blocks, phases separated by grid-wide
 * barriers; bitwise the same results.  Meant for small meshes, where a step is launch-latency
 * bound (the autotuner times both).  Its barrier words live in work->red[60..61]; a barrier wait
 * that gives up (iteration limit) sets a status word instead of hanging, read back with
 * fvm_fused_status (1 = a wait gave up and the results are invalid; the word stays set).
 * Partitioned meshes are FVM_E_UNSUPPORTED. */
int fvm_step_fused(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const fvm_tableau_t *tab,
                   const fvm_solver_bufs_t *bufs, const fvm_work_t *work, void *stream);
int fvm_multistep_fused(const fvm_mesh_t *mesh, const fvm_physics_t *phys, int32_t store, int32_t n_terms,
                        const int32_t *idx, const float *coef, const fvm_solver_bufs_t *bufs,
                        const fvm_work_t *work, void *stream);
int fvm_fused_status(const fvm_work_t *work, int32_t *status);
/* Self-test of the fused step's bounded grid barrier (no reference counterpart): a cooperative
 * launch of `blocks` blocks (2..64) meets at one barrier; with skip_block >= 0 that block never
 * arrives, the others' waits give up after a short iteration limit and *status becomes 1 (0 when
 * every block arrives).  Allocates and frees a few bytes of device memory; synchronous. */
int fvm_barrier_selftest(int32_t blocks, int32_t skip_block, int32_t *status);

/* Split stage for partitioned meshes (no reference counterpart): a stage is fvm_stage_begin
 * (boundary values + limited cell gradients of the owned cells from bufs->prims), then the
 * caller's exchange of the halo cells' limited gradients, then fvm_stage_end (facet fluxes,
 * divergence, stage combination and the next stage's primitives of the owned cells).  With
 * finalize = 0 the last stage leaves its reductions in work->red (adaptive sums [0, 3C), CFL max
 * at [16], conservation sums at [24, 24 + C)) for the caller to combine across parts, then
 * fvm_stage_finalize turns them into dt / conservation output.  fvm_stage_begin + fvm_stage_end
 * with finalize = 1 launch exactly what fvm_stage launches. */
int fvm_stage_begin(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const fvm_solver_bufs_t *bufs,
                    const fvm_work_t *work, void *stream);
int fvm_stage_end(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const fvm_tableau_t *tab, int32_t s,
                  const fvm_solver_bufs_t *bufs, const fvm_work_t *work, int32_t finalize, void *stream);
int fvm_stage_finalize(const fvm_mesh_t *mesh, const fvm_tableau_t *tab, const fvm_solver_bufs_t *bufs,
                       const fvm_work_t *work, void *stream);
/* Any phases of stage s (no reference counterpart), bits of `phases`: FVM_PHASE_BC (boundary
 * values), FVM_PHASE_CELLS (limited gradients of cells [cell_lo, n_owned)), FVM_PHASE_FACES (fluxes
 * of facets [facet_lo, n_facets)), FVM_PHASE_DIV (divergence, stage combination and the next
 * stage's primitives of the owned cells; the last stage's reductions as fvm_stage_end with
 * `finalize`).  fvm_stage_begin = BC | CELLS, fvm_stage_end = FACES | DIV; a partitioned stage that
 * overlaps its exchanges runs BC | CELLS on the inner cells, CELLS on the rest, FACES on the inner
 * facets, FACES on the rest, then DIV. */
#define FVM_PHASE_BC 1
#define FVM_PHASE_CELLS 2
#define FVM_PHASE_FACES 4
#define FVM_PHASE_DIV 8
int fvm_stage_phase(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const fvm_tableau_t *tab, int32_t s,
                    const fvm_solver_bufs_t *bufs, const fvm_work_t *work, int32_t phases, int32_t finalize,
                    void *stream);
/* Partitioned meshes: this part's sum of the interior sound speed over its characteristic
 * facets and their count into work->red[FVM_RED_DOUBLES + 6] and [+ 7] (padded primitives
 * `prims`).  The caller sums both over the parts and stores 10 / (float)(sum / count) at [+ 6]
 * before fvm_stage_begin when mesh->char_scale_given = 1 (facet_boundary.py:427). */
int fvm_char_partial(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const float *prims,
                     const fvm_work_t *work, void *stream);

/* One explicit stage s of `tab` (residual of bufs->prims, then the stage combination); the
 * last stage writes the new state and, per `tab`, updates dt.  Adaptive tableaus are
 * single-mesh only (FVM_E_UNSUPPORTED for batched meshes). */
int fvm_stage(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const fvm_tableau_t *tab,
              int32_t s, const fvm_solver_bufs_t *bufs, const fvm_work_t *work, void *stream);

/* A whole step: all stages and the dt update.  bufs->prims must hold the primitives of
 * bufs->state when the step starts (fvm_state_to_prims after setting the state); every step
 * leaves them consistent for the next one. */
int fvm_step(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const fvm_tableau_t *tab,
             const fvm_solver_bufs_t *bufs, const fvm_work_t *work, void *stream);

/* Multistep combination U <- U + sum_j coef[j] * k[idx[j]] (Adams-Bashforth); the residual of
 * the current state is stored, times dt, into k[store]. */
int fvm_multistep(const fvm_mesh_t *mesh, const fvm_physics_t *phys, int32_t store,
                  int32_t n_terms, const int32_t *idx, const float *coef,
                  const fvm_solver_bufs_t *bufs, const fvm_work_t *work, void *stream);

/* prims [N][FVM_ROW] <- primitives of state [N][C]. */
int fvm_state_to_prims(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const float *state,
                       float *prims, void *stream);

/* dt[case] <- cfl * min_i 1 / (inv_h_i (|u_i| + c_i)) over the case's cells (FP64 reduction). */
int fvm_cfl_dt(const fvm_mesh_t *mesh, const fvm_physics_t *phys, const float *state,
               float cfl, float *dt, const fvm_work_t *work, void *stream);

/* out[case][C] <- sum_i vol_i * state[i][c] over the case's cells, in FP64. */
int fvm_conservation(const fvm_mesh_t *mesh, const float *state, double *out,
                     const fvm_work_t *work, void *stream);

/* ---- learned corrector (no reference counterpart) ------------------------------------------
 * D[M][N] = epilogue(A[M][K] . B[N][K]^T) on the 5th-generation tensor cores (tcgen05, BF16
 * operands, FP32 accumulation in tensor memory).  A, B: bf16 row-major with leading dimensions
 * lda, ldb (multiples of 8, 16-byte aligned); N in {32, 64, 128, 256}; K a multiple of 64; M any.
 * Epilogue, in order: + bias[N] (may be NULL), store the pre-activation to `preact` (NULL = skip),
 * act (0 identity, 1 SiLU), + resid[M][ldr] (NULL = skip), store fp32 to Df and/or bf16 to Db
 * (leading dimension ldd).  k_splits > 1 splits K over that many CTAs per row tile, each
 * atomically adding its FP32 partial into Df (no other epilogue allowed).  *err is set to 1 if
 * a tensor-core completion wait times out (the kernel then returns without hanging). */
int fvm_gemm_bf16(const void *A, int64_t lda, const void *B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                  int32_t k_splits, const float *bias, const float *resid, int64_t ldr, float *Df, void *Db,
                  int64_t ldd, float *preact, int32_t act, int32_t *err, void *stream);

/* Corrector kernels (no reference counterpart).  The network's activations are an fp32 residual
 * stream h [N][64] (rows 32-byte aligned); GEMM operands are bf16; nbr is an int32 [N][KN] neighbour
 * table (-1 = none, adjacency symmetric, KN <= 8). */
/* One message-passing layer in one persistent kernel (inference):
 *   h_out_i = h_i + SiLU([bf16(h_i), bf16(mean_{j in nbr(i)} h_j)] . Wt^T + bias)
 * with Wt bf16 [64][128] (K-major); the mean is an fp32 sum over the valid neighbours in table
 * order times 1 / count.  With out != NULL (the last layer) the decoder is applied in the
 * epilogue instead: out_i[o] = bo[o] + sum_c h_out_i[c] Wo[o][c] (fp32 fma over c ascending, O <= 8
 * outputs, Wo fp32 [O][64]) and h_out may be NULL.  Bitwise equal to fvm_mp_gather_f32 +
 * fvm_gemm_bf16 (bias, SiLU, residual h) + fvm_decoder_f32.  h_out must not alias h.  A bounded
 * mbarrier wait that gives up sets *err (results invalid). */
int fvm_mp_layer(const float *h, const int32_t *nbr, int32_t M, int32_t KN, const void *Wt, const float *bias,
                 float *h_out, const float *Wo, const float *bo, int32_t O, float *out, int32_t *err, void *stream);
/* out[i] = [bf16(h_i), bf16(mean_{j in nbr(i)} h_j)]  (bf16 [N][128]) from the fp32 stream. */
int fvm_mp_gather_f32(const float *h, const int32_t *nbr, int32_t N, int32_t KN, void *out, void *stream);
/* dh_out[i] = dh_in[i] + dA[i][:W] + sum_{j in nbr(i)} dA[j][W:] / deg(j)  (fp32; dh_in may be NULL). */
int fvm_mp_scatter_back(const float *dA, const int32_t *nbr, int32_t N, int32_t W, int32_t KN, const float *dh_in,
                        float *dh_out, void *stream);
/* dZ = dh * SiLU'(Z) -> bf16 [N][W] and (if dZT) bf16 [W][ldT]; db[c] += sum_i dZ[i][c] (if db). */
int fvm_silu_back(const float *dh, const float *Z, int32_t N, int32_t W, void *dZ, void *dZT, int64_t ldT, float *db,
                  void *stream);
/* dst[c][r] = src[r][c] for a bf16 [R][Cc] matrix (leading dimensions lds, ldd). */
int fvm_transpose_bf16(const void *src, int32_t R, int32_t Cc, int64_t lds, void *dst, int64_t ldd, void *stream);
/* out[i][o] = bo[o] + sum_c h[i][c] Wo[o][c] (fp32 fma over c ascending; h fp32 [N][64], O <= 8). */
int fvm_decoder_f32(const float *h, const float *Wo, const float *bo, int32_t N, int32_t O, float *out, void *stream);
/* Decoder backward: dh = dOut Wo; dWo += dOut^T h; dbo += column sums of dOut (h fp32 [N][64]). */
int fvm_decoder_back_f32(const float *h, const float *Wo, const float *dOut, int32_t N, int32_t O, float *dh,
                         float *dWo, float *dbo, void *stream);
/* loss[0] += mean((pred - tgt)^2) over n_elem values (FP64); dpred = 2 (pred - tgt) / n_elem. */
int fvm_mse(const float *pred, const float *tgt, int64_t n_elem, double *loss, float *dpred, void *stream);
/* Adam on fp32 master weights p with gradient g (zeroed afterwards), moments m, v; step >= 1.
 * Refreshes the bf16 copy pb (if not NULL) and its [cols][rows] transpose pbT (if not NULL). */
int fvm_adam(float *p, float *g, float *m, float *v, int64_t n, float lr, float beta1, float beta2, float eps,
             int32_t step, void *pb, void *pbT, int32_t rows, int32_t cols, void *stream);
/* X[i] = [(U_i - mean) * inv_std (C values), geo[i] (G values), zeros] as bf16 [N][XW]. */
int fvm_corrector_features(const float *state, int32_t N, int32_t C, const float *mean, const float *inv_std,
                           const float *geo, int32_t G, void *X, int32_t XW, void *stream);
/* new_state = state + scale[c] * out (fp32 [N][C]). */
int fvm_apply_increment(const float *state, const float *out, const float *scale, int32_t N, int32_t C,
                        float *new_state, void *stream);
/* Corrector inputs with the residual baseline (C = 4 or 5): base[i] = kdt_case[case(i)] * r0[i]
 * (fp32 [N][C]) and the bf16 feature rows X[i] = [(state_i - mean[:C]) * inv_std[:C],
 * (base_i - mean[C:]) * inv_std[C:], geo_i, 0...] (XW entries, 2C + G <= XW, X 16-byte aligned).
 * cell_case (int32 [N]) may be NULL for one mesh (case 0). */
int fvm_corrector_inputs(const float *state, const float *r0, const float *kdt_case, const int32_t *cell_case,
                         int32_t N, int32_t C, const float *mean, const float *inv_std, const float *geo, int32_t G,
                         float *base, void *X, int32_t XW, void *stream);
/* prop = state + base + scale[c] * out - shift[case(i)][c]  (fp32 [N][C]; shift [cases][C] or NULL). */
int fvm_corrector_combine(const float *state, const float *base, const float *out, const float *scale,
                          const float *shift, const int32_t *cell_case, int32_t N, int32_t C, float *prop,
                          void *stream);

/* The corrector's acceptance checks for a batch (C = 4 or 5, cells of a case contiguous; r0 =
 * dU/dt at U, r1 at the proposal P): per case the FP64 sums over its cells of vol U, vol P, vol r0
 * (C each), vol |r0|^2, vol |r1|^2, the count of inadmissible cells of P (density or internal
 * energy <= 0, or not finite) and vol |P - U - k dt_c (r0 + r1) / 2|^2; then ok[c] = 1 iff
 * drift <= drift_tol, |r1|^2 <= ratio^2 |r0|^2, drift finite, no inadmissible cell and, when
 * consistency > 0, the distance to the trapezoidal rule is at most consistency * k dt_c |r0|
 * (volume-weighted norms), where drift = max over mass and energy of
 * |sum vol P - (sum vol U + k dt_c sum vol r0)| / |sum vol U|.  sums: [n_cases][3C + 4] doubles,
 * zero on the first call (each call leaves it zero); keep (or NULL) receives the sums. */
int fvm_corrector_checks(const float *U, const float *P, const float *r0, const float *r1, const float *volumes,
                         const int32_t *cell_case, int32_t N, int32_t C, int32_t n_cases, const float *dt, int32_t k,
                         double drift_tol, double ratio, double consistency, double *sums, uint8_t *ok, double *keep,
                         void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FVM_B200_H */
