/*
 * ptstokes.h -- C ABI of libptstokes.so, the B200 (sm_100a) pseudo-transient Stokes
 * solver. Drop-in for the hot path of PTsolvers/PseudoTransientStokes.jl: the PT
 * iteration of 2D/3D viscous and Maxwell visco-elastic Stokes flow on a staggered grid.
 *
 * The reference has no library boundary: each script defines its stencil kernels with
 * ParallelStencil and calls them positionally, e.g.
 *   @parallel compute_Pt_τ!(Pt, τxx, ..., Vx, Vy, Vz, Mus, Gdτ, r, G, dt, _dx, _dy, _dz)
 *   (scripts/stokes_3D/Stokes3D_ve_perf.jl:200-201).
 * Each entry point below replaces one such kernel call (cited per function); a Julia
 * `ccall` shim, a Python `ctypes` binding or C code calls them with plain pointers.
 *
 * Conventions
 *  - A context owns every device field of one problem. Host arrays passed in are
 *    Float64, column-major (x fastest), with the reference's own extents for that
 *    field (pts_field_shape); they are borrowed for the duration of the call.
 *  - Every call returns PTS_OK (0) or a negative PTS_E_* code; pts_last_error()
 *    gives the message. Nothing throws or exits across the ABI.
 *  - One context = one CUDA stream. Calls on different contexts are independent;
 *    a single context is not thread-safe. Calls are asynchronous on the context's
 *    stream unless documented as synchronous.
 */
#ifndef PTSTOKES_H
#define PTSTOKES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PTS_ABI_VERSION 3

#if defined(__GNUC__)
#define PTS_API __attribute__((visibility("default")))
#else
#define PTS_API
#endif

/* ---- status codes ---- */
#define PTS_OK 0
#define PTS_E_INVAL (-1)    /* bad argument (size, field id, variant, pointer) */
#define PTS_E_CUDA (-2)     /* CUDA runtime error */
#define PTS_E_NOMEM (-3)    /* device allocation failed */
#define PTS_E_NAN (-4)      /* residual check found NaN/Inf: `isnan(err) && error("NaN")`
                               (scripts/Stokes2D_ve.jl:171) */
#define PTS_E_STATE (-5)    /* call not valid for this context's variant / state */

/* ---- solver variants: which reference script's kernels and expression order ---- */
enum pts_variant {
    PTS_2D_V = 0,        /* scripts/Stokes2D.jl             2D viscous, roles P/τ/dV/V, /dx form   */
    PTS_2D_VE = 1,       /* scripts/Stokes2D_ve.jl          2D Maxwell VE, roles P/τ/dV/V          */
    PTS_2D_VE_PERF = 2,  /* scripts/Stokes2D_ve_perf.jl     2D VE, fused Pt_τ + V, _dx form        */
    PTS_3D_VE = 3,       /* scripts/stokes_3D/Stokes3D_ve_multixpu.jl (one rank), roles P/τ/dV/V */
    PTS_3D_VE_PERF = 4,  /* scripts/stokes_3D/Stokes3D_ve_perf.jl, fused Pt_τ + V             */
    PTS_3D_V = 5,        /* 3D viscous: the 3D fused kernels without elastic terms (no script) */
    /* The damped ("accel. 1") scheme: numerical compressibility β_n, a damped rate
     * dV/dτ = damp*dV/dτ + R and per-face pseudo-time steps (pts_set_damping). */
    PTS_2D_V_DAMP = 6,   /* scripts/previous_damp/Stokes2D0.jl     2D viscous, roles P/τ/dV/V     */
    PTS_2D_VE_DAMP = 7,  /* scripts/previous_damp/Stokes2D_ve0.jl  2D Maxwell VE, roles P/τ/dV/V  */
    PTS_3D_V_DAMP = 8    /* scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl (one rank), 3D viscous */
};

enum pts_precision {
    PTS_FP64 = 0,  /* plain FP64: the reference's arithmetic, bit for bit */
    PTS_MIXED = 1  /* FP32 inner PT sweeps on a correction, FP64 defect correction outside */
};

/* Problem description (physics + numerics of the script's Stokes2D_()/Stokes3D_()). */
typedef struct pts_desc {
    int32_t variant;    /* enum pts_variant */
    int32_t precision;  /* enum pts_precision */
    int32_t nx, ny, nz; /* cells (nz ignored in 2D); each >= 3 */
    int32_t nout;       /* error-check cadence `nout` (e.g. Stokes3D_ve_multixpu.jl:130) */
    double lx, ly, lz;  /* domain extents */
    double G, dt;       /* shear modulus and physical step (VE); ignored for viscous */
    double r, Re, CFL;  /* iteration parameters r, Re, CFL (Stokes3D_ve_perf.jl:129-131) */
    double max_l;       /* length in dτ_Rho = Vpdτ*max_l/Re/μ_eff; 0 => max(lx,ly[,lz]) */
    double eps;         /* tolerance ε on err (Stokes3D_ve_perf.jl:132) */
    double iter_max;    /* `while err > ε && iter <= iterMax` */
    int32_t mixed_inner;    /* MIXED: FP32 sweeps between FP64 corrections. The correction runs
                             * with every check, so this must be 0 or nout (others: PTS_E_INVAL) */
    int32_t single_pass;    /* 3D: 0 = two launches per iteration; one launch per iteration with
                             * 1 = inputs staged in shared memory by bulk copies, 2 = inputs read
                             * directly (L1/L2) */
    int32_t adjoint;        /* PTS_3D_V / PTS_3D_VE_PERF: 1 = solve the transposed (adjoint) system */
    int32_t stencil;        /* 3D compute_Pt_τ! and compute_V! + bc (FP64 two-kernel path, and the
                             * FP32 sweeps of MIXED): 0 = z-marching kernels whose input planes
                             * the tensor-memory accelerator stages in shared memory; 1 = one
                             * thread per cell or face, operands read directly. Same arithmetic
                             * (FP64: same bits). */
    int32_t stencil_tile;   /* z-marching kernel: tile configuration 0 .. pts_stencil_tiles(precision)-1
                             * (0 = default; see pts_stencil_tile_info); 2D contexts: the y-marching
                             * compute_Pt_τ!, 0 .. pts_stencil_tiles_2d()-1 */
    /* 2D (PTS_2D_V, PTS_2D_VE, PTS_2D_VE_PERF): stencil 0 also selects a y-marching
     * compute_Pt_τ! with TMA-staged tiles (stencil_kz = rows per block, 0 = 128); same bits. */
    int32_t stencil_kz;     /* z-marching kernels: z-planes per thread block (0 = default 32) */
    int32_t stencil_vtile;  /* z-marching compute_V! + bc: tile configuration
                             * 0 .. pts_stencil_vtiles(precision)-1 (0 = default) */
    int32_t mixed_sweep;    /* MIXED with stencil 0: 0 = two z-marching kernels per FP32 sweep
                             * (default, the faster on a B200); 1 + q = compute_V! + bc of one
                             * sweep and compute_Pt_τ! of the next in one z-marching pass with
                             * tile configuration q < pts_mixed_sweep_tiles() (27 arrays per
                             * sweep instead of 37; a second set of the ten corrections is
                             * allocated). The same FP32 expressions either way. */
} pts_desc;

/* Fields, by the reference's names. Extents are the reference's (pts_field_shape). */
enum pts_field {
    PTS_F_PT = 0,
    PTS_F_VX, PTS_F_VY, PTS_F_VZ,
    PTS_F_TXX, PTS_F_TYY, PTS_F_TZZ, PTS_F_TXY, PTS_F_TXZ, PTS_F_TYZ,
    PTS_F_TXX_O, PTS_F_TYY_O, PTS_F_TZZ_O, PTS_F_TXY_O, PTS_F_TXZ_O, PTS_F_TYZ_O,
    PTS_F_MUS,      /* Mus (smoothed viscosity)            */
    PTS_F_MUS_TAU,  /* Musτ (local-max viscosity)          */
    PTS_F_GDTAU,    /* Gdτ                                 */
    PTS_F_DTAU_RHO, /* dτ_Rho                              */
    PTS_F_DIVV,     /* ∇V                                  */
    PTS_F_RX, PTS_F_RY, PTS_F_RZ,
    PTS_F_DVX, PTS_F_DVY, PTS_F_DVZ,
    PTS_F_RHOG,     /* ρg (batched sweep only)            */
    /* Momentum sources on the interior faces (extents of Rx, Ry, Rz), added to the residual:
     * R = ∇·τ − ∇P + F. Absent (zero) until first set; 3D_V and 3D_VE_PERF, FP64 two-kernel path. */
    PTS_F_FX, PTS_F_FY, PTS_F_FZ,
    PTS_F_GRAD,     /* ∂J/∂log μ per cell (nx, ny, nz), written by pts_gradient_logmu */
    /* Pseudo-time steps of the damped variants, written by pts_compute_iter_params
     * (compute_timesteps!, Stokes2D_ve0.jl:27-32); the damped rates dVxdτ, dVydτ are
     * held in the dVx, dVy fields. */
    PTS_F_DTAU_VX,  /* dτVx, the extent of Rx */
    PTS_F_DTAU_VY,  /* dτVy, the extent of Ry */
    PTS_F_DTAU_VZ,  /* dτVz, the extent of Rz (3D) */
    PTS_F_DTAU_PT,  /* dτPt, one per cell */
    PTS_F_COUNT
};

/* Result of one convergence check (Stokes3D_ve_perf.jl:210-218). The norms are
 * ‖R‖/(Pmax-Pmin)*L/√len and ‖∇V‖/(Vmax-Vmin)*L/√len with L = lx for every norm, as the
 * scripts do, unless pts_set_norm_scales says otherwise. */
typedef struct pts_check {
    double err;                                       /* max of the four norms      */
    double norm_Rx, norm_Ry, norm_Rz, norm_divV;      /* norm_Rz = 0 in 2D          */
    double Vmin, Vmax, Pmin, Pmax;                    /* over Vx and Pt             */
} pts_check;

/* Outcome of one physical step's PT loop. */
typedef struct pts_solve_info {
    int64_t iters;       /* PT iterations done (`iter` at loop exit)          */
    int32_t converged;   /* 1 if the loop ended on err <= eps, 0 on iter_max  */
    int32_t nchecks;     /* residual checks done                              */
    pts_check last;      /* last check (err = 2*eps if none was done)         */
} pts_solve_info;

typedef struct pts_ctx pts_ctx;

/* ---- lifetime ---- */
PTS_API int pts_create(const pts_desc* desc, pts_ctx** out);   /* allocates + zeroes all fields (@zeros) */
PTS_API int pts_destroy(pts_ctx* ctx);
PTS_API const char* pts_last_error(const pts_ctx* ctx);        /* ctx may be NULL (creation errors) */
PTS_API int pts_abi_version(void);
PTS_API int pts_sync(pts_ctx* ctx);                            /* wait for the context's stream */
/* Tile configurations of the z-marching compute_Pt_τ! (pts_desc.stencil_tile) for a
 * precision (PTS_FP64 kernel, or the FP32 sweep of PTS_MIXED): their count, and per
 * configuration the tile height in cells (the width is 32) and the number of shared-memory
 * plane slots. No reference counterpart (ParallelStencil picks its launch shape itself). */
PTS_API int pts_stencil_tiles(int32_t precision);
/* The number of tile configurations of the z-marching compute_V! + bc (pts_desc.stencil_vtile). */
PTS_API int pts_stencil_vtiles(int32_t precision);
/* Change a context's pts_desc.stencil, stencil_tile, stencil_kz and stencil_vtile (same
 * meaning) without re-creating it, e.g. to time the tile configurations on the problem
 * itself. Results do not depend on the choice (FP64: bit for bit). No reference counterpart. */
PTS_API int pts_set_stencil(pts_ctx* ctx, int32_t stencil, int32_t tile, int32_t kz, int32_t vtile);
PTS_API int pts_stencil_tile_info(int32_t precision, int32_t tile, int32_t* tile_y, int32_t* ring_slots);
/* The context's cudaStream_t (as void*), to order or time the caller's own work with it. */
PTS_API int pts_stream(pts_ctx* ctx, void** stream);

/* ---- fields (Data.Array arguments of the kernels) ---- */
PTS_API int pts_field_shape(const pts_ctx* ctx, int32_t field, int64_t shape[3]);
PTS_API int pts_set_field(pts_ctx* ctx, int32_t field, const double* host, int64_t n);   /* synchronous */
PTS_API int pts_get_field(pts_ctx* ctx, int32_t field, double* host, int64_t n);         /* synchronous */
/* Same, with a device pointer to a dense column-major array (a CuArray's pointer). */
PTS_API int pts_set_field_device(pts_ctx* ctx, int32_t field, const double* dev, int64_t n);
PTS_API int pts_get_field_device(pts_ctx* ctx, int32_t field, double* dev, int64_t n);

/* ---- problem set-up on the device ---- */
/* Initial conditions of the scripts: Mus = mus0, Mus = musi where the squared distance of
 * the cell centre from the box centre is < radius2, pure-shear V with strain rate ebg,
 * every other field zero (Stokes3D_ve_perf.jl:164-172, Stokes2D.jl:106-114). */
PTS_API int pts_init_inclusion(pts_ctx* ctx, double mus0, double musi, double radius2, double ebg);
/* One inclusion of pts_init_inclusions: a circle (2D) or sphere (3D). */
typedef struct pts_inclusion {
    double x, y, z;  /* centre, relative to the domain centre (the scripts' Xi, Yi); z unused in 2D */
    double r2;       /* squared radius */
    double mus;      /* viscosity inside */
} pts_inclusion;
/* create_inclusions! (scripts/Stokes2D_param.jl:83-99) over a list of `count` inclusions
 * (0 <= count <= PTS_MAX_INCLUSIONS), each with its own radius and viscosity, in 2D or 3D:
 * Mus = the viscosity of the first inclusion whose squared distance from the cell centre is
 * below its r2, else mus0; pure-shear V with strain rate ebg; every other field zero (as
 * pts_init_inclusion). The list is read before the call returns. */
#define PTS_MAX_INCLUSIONS 65536
PTS_API int pts_init_inclusions(pts_ctx* ctx, const pts_inclusion* list, int32_t count, double mus0, double ebg);
/* ---- z-slab decomposition over several GPUs (the ImplicitGlobalGrid part of
 * scripts/stokes_3D/Stokes3D_ve_multixpu.jl, along z): each rank holds nz local planes that
 * overlap its neighbours by two (nz_g = P*(nz-2) + 2, init_global_grid, :138), and the host
 * exchanges the halo planes of V after every PT iteration (update_halo!(Vx, Vy, Vz), :238)
 * and of Mus, Musτ during set-up (:182-195), and reduces the check over ranks (:243-248).
 * ptstokes.multi drives it over torch.distributed. */
/* Before the set-up: this context is the slab [zoff, zoff+nz) of a global grid of nz_global
 * z-cells: dz = lz/nz_global, and the initial conditions use the global z coordinate
 * (z_g(iz, dz, A), :174-176). */
PTS_API int pts_set_decomposition(pts_ctx* ctx, int32_t zoff, int32_t nz_global);
/* Copy z-plane k (0-based, the field's reference extents) of a 3D field to or from a dense
 * device buffer of extent(1)*extent(2) doubles; synchronous. */
PTS_API int pts_get_plane_device(pts_ctx* ctx, int32_t id, int32_t k, double* dev, int64_t n);
PTS_API int pts_set_plane_device(pts_ctx* ctx, int32_t id, int32_t k, const double* dev, int64_t n);
/* compute_V! + bc (pts_compute_V_bc) on the face planes k in [k0, k1) only (0 <= k0 <= k1 <=
 * nz+1), enqueued on `stream` (NULL: the context's stream); asynchronous. The boundary and
 * inner regions of @hide_communication b_width (Stokes3D_ve_multixpu.jl:136,230-239): after
 * pts_compute_Pt_tau, the planes next to the slab ends are updated first so their halo
 * exchange overlaps the inner planes' update on another stream. A face update reads V only
 * at its own point and writes bc copies only next to the first and last interior planes, so
 * disjoint ranges may run concurrently. FP64 3D_VE, 3D_VE_PERF, 3D_V contexts without
 * momentum sources or adjoint mode. */
PTS_API int pts_compute_V_bc_planes(pts_ctx* ctx, int32_t k0, int32_t k1, void* stream);
/* The local pieces of the check, to be reduced over ranks (norm_g, minimum_g, maximum_g,
 * :243-248): {Σ Rx², Σ Ry², Σ Rz², Σ ∇V², min Vx, max Vx, min Pt, max Pt}; synchronous. */
PTS_API int pts_check_partials(pts_ctx* ctx, double out[8]);
/* The lengths L of norm_Rx, norm_Ry, norm_Rz and norm_∇V (default lx for all four). The
 * aspect-ratio script scales norm_Rx by lx and norm_Ry, norm_∇V by ly
 * (scripts/Stokes2D_ve_param.jl:175-177). */
PTS_API int pts_set_norm_scales(pts_ctx* ctx, double sRx, double sRy, double sRz, double sdiv);
/* The form of the FP32 sweeps of a MIXED context (pts_desc.mixed_sweep), and the number of
 * tile configurations of the one-pass form. */
PTS_API int pts_set_mixed_sweep(pts_ctx* ctx, int32_t mixed_sweep);
PTS_API int pts_mixed_sweep_tiles(void);
/* Tile configurations of the 2D y-marching compute_Pt_τ! (pts_desc.stencil_tile of 2D contexts). */
PTS_API int pts_stencil_tiles_2d(void);
/* smooth!(Mus2, Mus, fact) nsweeps times with the Mus/Mus2 swap (Stokes3D_ve_perf.jl:173-177). */
PTS_API int pts_smooth(pts_ctx* ctx, int32_t nsweeps, double fact);
/* Musτ .= Mus; compute_maxloc!(Musτ, Mus); bc_x!/bc_y!/bc_z!(Musτ) (Stokes3D_ve_perf.jl:178-182). */
PTS_API int pts_compute_maxloc(pts_ctx* ctx);
/* compute_iter_params! (Stokes3D_ve_perf.jl:34-39; viscous Stokes2D.jl:27-31); for the
 * damped variants compute_timesteps! (Stokes2D_ve0.jl:27-32). */
PTS_API int pts_compute_iter_params(pts_ctx* ctx);
/* Numerics of the damped variants (Stokes2D_ve0.jl:95-98, Stokes3D0_multixpu.jl:105-108):
 * Vdmp (damp = 1 - Vdmp/n per direction), β_n, Vsc, Ptsc. A new context has the scripts'
 * values: 4, 2, 1, 3 in 2D and 4, 3, 1, 5 in 3D. Call before pts_compute_iter_params;
 * PTS_E_INVAL for the other variants, Vsc or Ptsc <= 0, or β_n <= -1. */
PTS_API int pts_set_damping(pts_ctx* ctx, double Vdmp, double beta_n, double Vsc, double Ptsc);

/* ---- PT iteration roles ---- */
PTS_API int pts_assign_tau(pts_ctx* ctx);        /* assign_τ!  (Stokes3D_ve_perf.jl:41-49)              */
PTS_API int pts_compute_P(pts_ctx* ctx);         /* compute_P! (Stokes3D_ve_multixpu.jl:57-61): ∇V, Pt  */
PTS_API int pts_compute_tau(pts_ctx* ctx);       /* compute_τ! (Stokes3D_ve_multixpu.jl:69-77)          */
PTS_API int pts_compute_dV(pts_ctx* ctx);        /* compute_dV! (Stokes3D_ve_multixpu.jl:79-84)         */
PTS_API int pts_compute_V(pts_ctx* ctx);         /* compute_V! (Stokes3D_ve_multixpu.jl:86-91)          */
PTS_API int pts_apply_bc(pts_ctx* ctx);          /* the bc_x!/bc_y!/bc_z! calls on V (…_perf.jl:202-207) */
PTS_API int pts_compute_Pt_tau(pts_ctx* ctx);    /* compute_Pt_τ! (Stokes3D_ve_perf.jl:69-78)           */
PTS_API int pts_compute_V_bc(pts_ctx* ctx);      /* compute_V! + bc (Stokes3D_ve_perf.jl:83-88,202-207)  */
/* MIXED: one half of an FP32 sweep on the current corrections, asynchronous, no fold:
 * which = 0 the δ-form compute_Pt_τ!, 1 the δ-form compute_V! + bc (for timing them). */
PTS_API int pts_sweep32_kernel(pts_ctx* ctx, int32_t which);
/* Per-kernel timing (on = 1): every block of PT iterations records a CUDA event before its
 * first kernel and after each kernel it launches (the check's too), inside the check
 * block's graph as event-record nodes. pts_kernel_times gives the elapsed ms between
 * consecutive events of the last block enqueued, in launch order (FP64 two-kernel path:
 * compute_Pt_τ!, compute_V! + bc, ..., the check); synchronous. */
PTS_API int pts_set_kernel_timing(pts_ctx* ctx, int32_t on);
PTS_API int pts_kernel_times(pts_ctx* ctx, float* ms, int64_t cap, int64_t* count);
/* compute_Res! + the norms of the check (Stokes3D_ve_perf.jl:209-219). Synchronous. */
PTS_API int pts_compute_res(pts_ctx* ctx, pts_check* out);

/* ---- drivers ---- */
/* n PT iterations (roles + BCs) on the fast path, no checks. Asynchronous. */
PTS_API int pts_iterate(pts_ctx* ctx, int64_t n);
/* One physical step's PT loop: `while err > ε && iter <= iterMax` with a check every
 * nout iterations (Stokes3D_ve_perf.jl:198-223). Synchronous. Returns PTS_OK whether
 * the loop ended on the tolerance or on iter_max (info->converged tells which) and
 * PTS_E_NAN when a check's err is NaN (`if isnan(err) error("NaN") end`, :219). */
PTS_API int pts_solve(pts_ctx* ctx, pts_solve_info* info);
/* nt physical steps: assign_τ! (VE) then pts_solve, as the time loop
 * `for it = 1:nt` (Stokes3D_ve_perf.jl:194-226). iters_per_step (length nt) may be NULL;
 * info (may be NULL) receives the last step's outcome with iters = ittot. */
PTS_API int pts_run(pts_ctx* ctx, int32_t nt, int64_t* iters_per_step, pts_solve_info* info);

/* ---- adjoint of the 3D viscous solve (PTS_3D_V, FP64; visco-elastic PTS_3D_VE_PERF below) ----
 * No counterpart in the reference. The converged PTS_3D_V iterate solves A(μ)[V;P] = b with
 * A = [[K, -G], [div∘B, 0]]: B extends the interior velocities to the free-slip ghosts by
 * copying, the walls' normal velocities are data, K = D·2μ·S·B (S the strain rates, D the
 * stress divergence on the interior faces). The copies make K unsymmetric, so the adjoint
 * of a misfit J(V) solves the transposed system: a PTS_3D_V context created with
 * desc.adjoint = 1 and the same Mus, zero fields and the momentum source F = ∂J/∂V
 * (PTS_F_FX/FY/FZ), solved with pts_solve. In that mode the ghosts stay zero (no copies)
 * and the residual of every ghost face -- the same stencil, reading zeros where no stress
 * point exists -- is added to the residual of the interior face it copies (the transpose of
 * the copy). Then, with λ the adjoint velocity,
 *   ∂J/∂log μ_c = -μ_c [2 Σ_n ε̇_n(V) ε̇_n(λ) + Σ_{edges e around c} ε̇_s(V) ε̇_s(λ)]
 * (normal rates on the cells compute_τ! updates, shear rates on the interior edges, each
 * edge averaging 4 cells), with log μ the viscosity the solver uses (after any smoothing). */
/* τ = 2·Mus·ε̇(V) (the fixed point of compute_τ!), then the check: Rx, Ry, Rz = ∇·τ − ∇P + F
 * (folded onto the interior faces in adjoint mode) and ∇V of the current fields -- one
 * application of A or its transpose, for symmetry tests. Synchronous. */
PTS_API int pts_apply_operator(pts_ctx* ctx, pts_check* out);
/* ∂J/∂log μ into fwd's PTS_F_GRAD from fwd's V (the forward solution) and adj's V (the adjoint
 * solution of an adjoint-mode context); same grid, both PTS_3D_V FP64. Synchronous.
 *
 * Visco-elastic (two PTS_3D_VE_PERF contexts, no counterpart in the reference): a converged
 * physical step has τ = η(2ε̇ + τ_o/(G dt)), η = 1/(1/μ + 1/(G dt)) (μ̄ on the shear edges).
 * The adjoint of nt steps is the same time loop in adjoint mode run backwards: the source
 * ∂J/∂V in the step that adjoints the last forward step, zero afterwards, and assign_τ!
 * (τ_o ← τ) between steps exactly as forward. With τ the forward step's converged stresses
 * (restored into fwd from a per-step checkpoint) and τa the matching adjoint step's,
 * one step contributes
 *   ∂J/∂log μ_c += -[Σ_n τa_n τ_n/(2μ_c) + μ_c Σ_{edges e around c} τa_e τ_e/(4 μ̄_e²)];
 * pts_gradient_logmu writes that term, pts_gradient_logmu_add adds it. */
PTS_API int pts_gradient_logmu(pts_ctx* fwd, pts_ctx* adj);
PTS_API int pts_gradient_logmu_add(pts_ctx* fwd, pts_ctx* adj);

/* ---- batched 2D viscous sweep: many uneven grids, one persistent launch ----
 * Replaces the reference's parameter sweeps, which run one Julia process per instance
 * (scripts/runme_Stokes2D_{shear,gravity}_weak.jl:23-25 launching Stokes2D_param.jl). Each
 * instance has that script's numerics -- its compute_τ! form (:48-55), buoyancy term (:59)
 * and uniform iteration parameters from Musτ .= μs0 (:190-192) -- on a box lx x ly
 * (Stokes2D_ve_param.jl:99-102) with one centred inclusion (viscosity musi, density
 * contrast rhogi) and pure shear ebg. All instances iterate in one cooperative launch; an
 * instance stops when its check (every nout iterations; Stokes2D_param.jl:203-210 with one
 * tolerance, norms scaled by ly) reaches eps, or after its iterMax. */
typedef struct pts_batch_instance {
    int32_t nx, ny;   /* cells, each >= 3 */
    double lx, ly;    /* box */
    double musi;      /* inclusion viscosity (matrix 1) */
    double radius2;   /* squared inclusion radius (centred) */
    double rhogi;     /* inclusion ρg (matrix 0) */
    double ebg;       /* background pure-shear strain rate */
} pts_batch_instance;

typedef struct pts_batch_desc {
    int32_t nout;      /* check cadence */
    int32_t tile;      /* tile shape 0..3 = 32x4, 32x8, 64x4, 32x16 (pts_batch_set_tile) */
    double eps;        /* tolerance */
    double iter_max;   /* `iter <= iterMax`; <= 0: 100*max(nx,ny) per instance (Stokes2D_param.jl:146) */
    double r, Re, CFL; /* iteration parameters (Stokes2D_param.jl:150-152) */
    int32_t reserved[4];
} pts_batch_desc;

typedef struct pts_batch pts_batch;
PTS_API int pts_batch_create(const pts_batch_desc* desc, const pts_batch_instance* inst, int32_t n, pts_batch** out);
PTS_API int pts_batch_destroy(pts_batch* b);
PTS_API const char* pts_batch_last_error(const pts_batch* b);
/* ICs and smooth! x10 of Mus and ρg for every instance (Stokes2D_param.jl:179-189) */
PTS_API int pts_batch_setup(pts_batch* b);
PTS_API int pts_batch_set_tile(pts_batch* b, int32_t tile);
/* The persistent launch (captured in a CUDA graph when the CUDA driver allows it): runs until
 * every instance has converged or passed its iterMax; iter_limit >= 0 is a further ceiling
 * common to all. Synchronous. iters/err/converged (length n, may be NULL) receive each
 * instance's outcome; converged is 0 for an instance stopped by iterMax or by NaN (the call
 * then returns PTS_E_NAN). */
PTS_API int pts_batch_solve(pts_batch* b, int64_t iter_limit, int64_t* iters, double* err, int32_t* converged,
                            int32_t* used_graph);
/* A field of one instance (fields Pt Vx Vy τxx τyy τxy Mus Musτ Gdτ dτ_Rho ∇V Rx Ry ρg;
 * Musτ, Gdτ and dτ_Rho are uniform per instance and are returned as that value filled) */
PTS_API int pts_batch_get_field(pts_batch* b, int32_t instance, int32_t field, double* host, int64_t n);
PTS_API int pts_batch_stream(pts_batch* b, void** stream);

/* ---- batched 2D visco-elastic aspect-ratio sweep: all instances in one persistent launch ----
 * Replaces scripts/runme_Stokes2D_aspect_ratio.jl:1-24, which runs one Julia process of
 * scripts/Stokes2D_ve_param.jl per (FACT, NSUB, RESOL). Each instance is that script:
 * ly = ly, lx = nsub*ly, nx = nsub*(ny+1)-1, ny = RESOL (:99-107), matrix viscosity 1 and
 * nsub inclusions of radius 1 and viscosity musi (:133-141), G = dt = 1, pure shear 1,
 * 10 smooth! sweeps, local-max iteration parameters with min_lxy = fact*min(lx,ly)
 * (:110, :142-150), and nt physical steps, each `assign_τ!; while err > ε && iter <= iterMax`
 * with a check every nout iterations, norm_Rx scaled by lx and norm_Ry, norm_∇V by ly
 * (:152-186). The descriptor gives eps, r, Re, CFL and the tile shape; nout <= 0 gives
 * each instance the script's nout = nx, iter_max <= 0 its iterMax = 100nx. The rest of the
 * batch API applies: pts_batch_setup builds the ICs of every instance, pts_batch_solve runs
 * every instance's nt steps (iters receives each instance's ittot, converged is 1 when its
 * last step reached eps; an instance whose check gives NaN is frozen, as the script stops
 * there, and the call returns PTS_E_NAN), pts_batch_get_field reads Pt Vx Vy τxx τyy τxy
 * τxx_o τyy_o τxy_o Mus Musτ Gdτ dτ_Rho ∇V Rx Ry. */
typedef struct pts_batch_ve_instance {
    int32_t ny;      /* RESOL: cells in y (>= 3) */
    int32_t nsub;    /* NSUB: subdomains along x, one inclusion each (>= 1) */
    int32_t nt;      /* physical steps (1..64; the script: 5) */
    int32_t reserved;
    double fact;     /* FACT: min_lxy = fact*min(lx,ly) */
    double ly;       /* box height (the script: 10) */
    double musi;     /* inclusion viscosity (the script: 1e-3) */
} pts_batch_ve_instance;
PTS_API int pts_batch_create_ve(const pts_batch_desc* desc, const pts_batch_ve_instance* inst, int32_t n,
                                pts_batch** out);
/* PT iterations of each finished step of one instance (Stokes2D_ve_param.jl:186, the iter
 * added to ittot): up to max_steps values into iters, the number of finished steps into
 * nsteps. Visco-elastic sweeps only. */
PTS_API int pts_batch_steps(pts_batch* b, int32_t instance, int64_t* iters, int32_t max_steps, int32_t* nsteps);

/* ---- convergence check without any allocation ----
 * This entry point has no counterpart in the reference. It is for callers that cannot
 * allocate device memory: programs whose device memory all belongs to another allocator
 * (CUDA.jl's pool for Julia CuArrays, PyTorch's caching allocator) or that partition the
 * GPU up front and forbid later cudaMalloc calls. It computes the same check as
 * pts_compute_res -- compute_Res! and the norms of Stokes3D_ve_perf.jl:90-96,210-218 --
 * directly on the caller's arrays, and calls no cudaMalloc, cudaFree or allocating library.
 *   desc     sizes, extents and variant; only PTS_2D_VE_PERF, PTS_3D_VE_PERF, PTS_3D_V
 *   fields   device pointers indexed by pts_field (PTS_F_PT .. PTS_F_TYZ): dense column-major
 *            Float64 arrays with the reference's extents; in 2D Vz, τzz, τxz, τyz are unused
 *   out      device pointer to a pts_check the result is written to (err is NaN on NaN)
 *   stream   cudaStream_t to run on (NULL: the default stream); the call is asynchronous
 * Limit: the block partials of the reduction live in a fixed 256 KB array inside the
 * library (held by every GPU that loads it, until exit), which bounds the grid:
 * ceil((nx+1)/32) * ceil(ny/8) <= 4096; larger sizes return PTS_E_INVAL with a message in
 * pts_last_error(NULL). The first call on a device looks up that array's device address
 * (once per device, with the device current); make that first call before any stream
 * capture. All calls share the array and overwrite what they read, so calls whose kernels
 * overlap on the GPU race and must be ordered by the caller. */
PTS_API int pts_check_noalloc(const pts_desc* desc, const double* const fields[10], pts_check* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PTSTOKES_H */
