// pts_internal.h -- shared layout, parameter and launch declarations of libptstokes.
//
// Data layout in HBM ("unified staggered layout"): every field of a problem is stored in
// its own array of the same padded extent px x py x pz, px = round_up(nx+1, 16) (so each
// x-row starts on a 128-byte boundary), py = ny+1, pz = nz+1 (pz = 1 in 2D). A field
// element lives at the unified staggered coordinate (i,j,k) of the point it describes:
//   cell centre (i,j,k)            Pt, Mus, Musτ, Gdτ, dτ_Rho, ∇V, τxx, τyy, τzz
//   x-face i (between cells i-1,i) Vx, Rx, dVx;   y-face j: Vy ...;   z-face k: Vz ...
//   x-face i, y-face j, cell k     τxy (edge);    τxz: x-face,cell,z-face;  τyz: cell,y-face,z-face
// so a neighbour in x/y/z is always at offset +-1 / +-px / +-px*py whatever the field. The
// reference's arrays (1-based, column-major, each with its own extent) map to this layout
// with a per-field start offset (field_info() in pts_abi.cu); set/get convert once.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ptstokes.h"

namespace pts {

enum Variant {
    V2D = PTS_2D_V,
    VE2D = PTS_2D_VE,
    VE2D_PERF = PTS_2D_VE_PERF,
    VE3D = PTS_3D_VE,
    VE3D_PERF = PTS_3D_VE_PERF,
    V3D = PTS_3D_V,
    V2D_DAMP = PTS_2D_V_DAMP,
    VE2D_DAMP = PTS_2D_VE_DAMP,
    V3D_DAMP = PTS_3D_V_DAMP,
};

inline bool variant_is3d(int v) { return v == VE3D || v == VE3D_PERF || v == V3D || v == V3D_DAMP; }
inline bool variant_elastic(int v) { return v != V2D && v != V3D && v != V2D_DAMP && v != V3D_DAMP; }
inline bool variant_damped(int v) { return v == V2D_DAMP || v == VE2D_DAMP || v == V3D_DAMP; }
// "perf" variants multiply by _dx = 1/dx (explicit-index kernels); the others divide by dx.
inline bool variant_perf(int v) { return v == VE2D_PERF || v == VE3D_PERF || v == V3D; }
// ∇V of the check: from compute_P! before the V update (role variants), or recomputed
// from the current V by compute_Res! (perf variants).
inline bool variant_divV_from_P(int v) { return !variant_perf(v); }

struct Geom {
    int nx, ny, nz;   // cells (nz = 1 in 2D)
    int px, py, pz;   // padded extents of every field array
    int64_t pxy;      // px * py
    int64_t n;        // px * py * pz elements per field
};

__host__ __device__ inline int64_t gidx(const Geom& g, int i, int j, int k) {
    return (int64_t)i + (int64_t)g.px * ((int64_t)j + (int64_t)g.py * (int64_t)k);
}

// Element index inside one field in 32 bits: every problem that fits on one device has
// fewer than 2^31 elements per field (pts_create rejects larger ones), and 32-bit offsets
// save the 64-bit multiply-adds on each of a stencil's ~30 loads.
typedef int idx_t;
__host__ __device__ inline idx_t gidx32(const Geom& g, int i, int j, int k) { return i + g.px * (j + g.py * k); }

// Scalars of the scripts' "Derived numerics" (Stokes3D_ve_perf.jl:135-138).
struct Num {
    double dx, dy, dz, _dx, _dy, _dz;
    double r, G, dt, gdt;  // gdt = G*dt
    double Vpdt, max_l, Re;
    double lx, ly, lz;
    int adjoint;  // 3D_V: iterate the transposed (adjoint) system, ghosts folded (pts_abi.cu)
    int zoff;     // z-slab decomposition: global index of this context's first z-plane (ICs)
    double nsc[4];  // lengths that scale norm_Rx, norm_Ry, norm_Rz, norm_∇V in the check
    // damped variants (Stokes2D_ve0.jl:95-105, Stokes3D0_multixpu.jl:105-120): Vdmp, β_n,
    // Vsc, Ptsc and the derived dampX = 1-Vdmp/nx (Y, Z alike), min_dxy2 = min(dx,dy[,dz])^2,
    // max_nxy = max(nx,ny[,nz])
    double Vdmp, beta_n, Vsc, Ptsc, dampX, dampY, dampZ, min_dxy2, max_nxy;
};

template <typename T>
struct FieldsT {
    T *Pt, *Vx, *Vy, *Vz;
    T *txx, *tyy, *tzz, *txy, *txz, *tyz;
    T *txx_o, *tyy_o, *tzz_o, *txy_o, *txz_o, *tyz_o;
    T *Mus, *Must, *Gdt, *dtRho, *divV;
    T *Rx, *Ry, *Rz, *dVx, *dVy, *dVz;
    T *Mus2;
    T *rhog, *rhog2;  // buoyancy ρg of the batched sweep (Stokes2D_param.jl), else null
    T *Fx, *Fy, *Fz;  // momentum sources on interior faces (adjoint solves), else null
    T *grad;          // ∂J/∂log μ per cell, else null
    T *dtVx, *dtVy, *dtVz, *dtPt;  // pseudo-time steps of the damped variants, else null
};
using Fields64 = FieldsT<double>;

// Per-block partials of the check reduction: sums of squares of Rx, Ry, Rz, ∇V and
// min/max of Vx and Pt (Stokes3D_ve_perf.jl:211-216).
constexpr int kCheckSlots = 8;
// Device result block written by the check finaliser.
struct CheckResult {
    double err, nRx, nRy, nRz, ndiv, vmin, vmax, pmin, pmax;
    double flag_nan;
    double sRx, sRy, sRz, sdiv;  // the sums of squares the norms come from
};

// ---- launchers implemented in pts_kernels64.cu (FP64, no FMA contraction) ----
enum RoleMask { ROLE_P = 1, ROLE_TAU = 2 };
cudaError_t launch_Pt_tau(int variant, const Geom& g, const Fields64& f, const Num& n, int roles, bool store_divV,
                          cudaStream_t s);
cudaError_t launch_V_bc(int variant, const Geom& g, const Fields64& f, const Num& n, bool apply_update,
                        cudaStream_t s);
// compute_V! + bc on the face planes [k0, k1) only (3D_VE, 3D_VE_PERF, 3D_V; no sources, not adjoint)
cudaError_t launch_V_bc_planes(int variant, const Geom& g, const Fields64& f, const Num& n, int k0, int k1,
                               cudaStream_t s);
cudaError_t launch_dV(int variant, const Geom& g, const Fields64& f, const Num& n, cudaStream_t s);
cudaError_t launch_add_dV(int variant, const Geom& g, const Fields64& f, cudaStream_t s);
cudaError_t launch_check(int variant, const Geom& g, const Fields64& f, const Num& n, double* partials,
                         int nblocks_cap, CheckResult* result, cudaStream_t s);
int check_num_blocks(int variant, const Geom& g);
cudaError_t launch_init_inclusion(int variant, const Geom& g, const Fields64& f, const Num& n, double mus0,
                                  double musi, double radius2, double ebg, cudaStream_t s);
cudaError_t launch_init_inclusions(int variant, const Geom& g, const Fields64& f, const Num& n,
                                   const pts_inclusion* d_inc, int count, double mus0, double ebg, cudaStream_t s);
cudaError_t launch_smooth(int variant, const Geom& g, double* dst, const double* src, double fact, cudaStream_t s);
cudaError_t launch_maxloc(int variant, const Geom& g, double* must, const double* mus, cudaStream_t s);
cudaError_t launch_iter_params(int variant, const Geom& g, const Fields64& f, const Num& n, cudaStream_t s);
// ---- adjoint of the 3D viscous solve (3D_V) ----
// τ = 2·Mus·ε̇(V), the converged value of compute_τ! (the exact viscous operator's stresses)
cudaError_t launch_tau_exact(const Geom& g, const Fields64& f, const Num& n, cudaStream_t s);
// ∂J/∂log μ into fwd.grad, from the forward solution (fwd) and the adjoint solution (adj)
cudaError_t launch_grad_logmu(const Geom& g, const Fields64& fwd, const Fields64& adj, const Num& n, cudaStream_t s);
// one physical step's ∂J/∂log μ term of the visco-elastic operator (3D_VE_PERF) from the
// forward and adjoint stresses, written (add = false) or added (add = true) to fwd.grad
cudaError_t launch_grad_logmu_ve(const Geom& g, const Fields64& fwd, const Fields64& adj, bool add, cudaStream_t s);
// single-pass 3D kernel: V update of iteration n from `cur`, then Pt/τ of n+1, into `nxt`
// `err` is a device flag the kernel sets if one of its bounded staging waits timed out;
// `direct` selects the variant that reads its inputs from global memory without staging.
cudaError_t launch_fused3(int variant, const Geom& g, const Fields64& cur, const Fields64& nxt, const Num& n,
                          bool store_divV, int* err, cudaStream_t s,
                          bool direct);
inline bool variant_fused(int v) { return variant_is3d(v) && !variant_damped(v); }

// ---- z-marching compute_Pt_τ! with TMA-staged planes (pts_zstage.cu): 3D_VE, 3D_VE_PERF,
// 3D_V. `tile` selects a tile configuration (zstage_tile_info), `kz` the z-planes per
// thread block; `err` is set if one of the kernel's bounded waits gave up.
int zstage_num_configs();
bool zstage_tile_info(int tile, int* ty, int* ring);
cudaError_t launch_Pt_tau_zs(int variant, int tile, const Geom& g, const Fields64& f, const Num& n, int kz,
                             bool store_divV, int* err, cudaStream_t s);

// Message returned by pts_last_error(NULL) (for entry points without a context).
void set_global_error(const char* msg);

// ---- mixed precision (3D explicit-index variants) ----
// FP32 fields of the inner sweeps: the correction δ of the ten iterated fields (the six
// stresses carried as u = δτ - w), the sources of the current FP64 iterate (aP, aV, and
// w = aτ/(D - 1) in the aτ arrays; pts_kernels32.cu), and FP32 copies of the
// coefficients. Same unified layout and extents as the FP64 fields.
struct Mixed32 {
    float *dPt, *dVx, *dVy, *dVz, *dtxx, *dtyy, *dtzz, *dtxy, *dtxz, *dtyz;
    float *aP, *atxx, *atyy, *atzz, *atxy, *atxz, *atyz, *aVx, *aVy, *aVz;
    float2* GM;    // Gdτ and Mus interleaved: one 8-byte load gives both at a point
    float* dtRho;
    float* u2[6];  // the stress corrections of the second buffer set (one-pass sweeps), or null
};
// FP32 inner sweep (pts_kernels32.cu): δ-form compute_Pt_τ! and compute_V! + bc.
cudaError_t launch_corr_A32(int variant, const Geom& g, const Mixed32& m, const Num& n, cudaStream_t s);
cudaError_t launch_corr_B32(int variant, const Geom& g, const Mixed32& m, const Num& n, cudaStream_t s);
// The δ-form compute_Pt_τ! as a z-marching kernel with TMA-staged planes (same arithmetic as
// launch_corr_A32); `tile` < zstage32_num_configs(), `kz` planes per block (0: 32).
cudaError_t launch_corr_A32_zs(int variant, int tile, const Geom& g, const Mixed32& m, const Num& n, int kz, int* err,
                               cudaStream_t s);
int zstage32_num_configs();
// compute_V! + bc as a z-marching kernel with TMA-staged planes (pts_zvbc.cuh): FP64 (same
// bits as launch_V_bc, without momentum sources or adjoint folding) and the FP32 δ-form sweep
// (same arithmetic as launch_corr_B32). `tile` < zvbc_num_configs() / zvbc32_num_configs().
cudaError_t launch_V_bc_zs(int variant, int tile, const Geom& g, const Fields64& f, const Num& n, int kz, int* err,
                           cudaStream_t s);
cudaError_t launch_corr_B32_zs(int variant, int tile, const Geom& g, const Mixed32& m, const Num& n, int kz, int* err,
                               cudaStream_t s);
int zvbc_num_configs();
int zvbc32_num_configs();
// compute_V! + bc of one FP32 sweep and compute_Pt_τ! of the next in one z-marching pass,
// from the corrections in `m` into the other buffer set `out` (its ten δ arrays); the same
// arithmetic as launch_corr_B32_zs followed by launch_corr_A32_zs. `tile` <
// zfused32_num_configs(), `kz` planes per block (0: 64).
cudaError_t launch_corr_BA32_zs(int variant, int tile, const Geom& g, const Mixed32& m, const Mixed32& out,
                                const Num& n, int kz, int* err, cudaStream_t s);
int zfused32_num_configs();
// compute_Pt_τ! (2D: V2D, VE2D, VE2D_PERF) as a y-marching kernel with TMA-staged tiles; the
// same bits as launch_Pt_tau. `tile` < ystage_num_configs(), `ky` rows per block (0: 128).
cudaError_t launch_Pt_tau_ys(int variant, int tile, const Geom& g, const Fields64& f, const Num& n, int ky,
                             bool store_divV, int* err, cudaStream_t s);
int ystage_num_configs();
bool zstage32_tile_info(int tile, int* ty, int* ring);
// FP64 outer step (pts_kernels64.cu): fold X += δ and clear δ; residual sources of X
// (aP = ∇·V, aτ = constitutive residual, aV = momentum residual R) with the check
// partials and its finaliser; FP32 copies of the coefficients.
cudaError_t launch_fold(const Geom& g, const Fields64& f, const Mixed32& m, cudaStream_t s);
cudaError_t launch_sources(int variant, const Geom& g, const Fields64& f, const Mixed32& m, const Num& n,
                           double* partials, int nblocks_cap, CheckResult* result, cudaStream_t s);
cudaError_t launch_coef32(const Geom& g, const Fields64& f, const Mixed32& m, cudaStream_t s);

// ---- batched 2D sweep (pts_batch.cu host side, kernels in pts_kernels64.cu) ----
// One instance: its geometry and numerics, where its fields start in every arena, and
// the first of its TX x TY tiles in the flattened tile list.
struct BInst {
    Geom g;
    Num n;
    int64_t off;
    int tile0, ntx, nty;
    double lenRx, lenRy, lenDiv, ly;
    double Gd, dR;     // the instance's uniform Gdτ and dτ_Rho (Musτ .= μs0)
    int64_t iter_last; // its PT loop runs while iter <= iter_last (iterMax)
    // visco-elastic sweep only: the norm_Rx scale lx, the instance's check cadence and its
    // number of physical steps
    double lx;
    int nout, nt;
};
struct BState {
    int* converged;   // per instance: 1 its PT loop has ended on the tolerance, 2 frozen on NaN
    int64_t* iters;   // per instance: PT iterations done
    double* err;      // per instance: err of the last check
    double* partials; // per tile: 8 partial sums/extrema of the check
    int* nactive;     // instances still iterating
    int* act;         // active list rebuilt at each check: K, T, first tile[K+1], instance[K] (2n+3 ints)
    int* nan_flag;
};
// Per-instance state of the batched visco-elastic sweep (k2_batch_ve). The instance's
// status lives in BState::converged: 0 iterating, 1 finished with its last step converged,
// 2 frozen on NaN, 3 finished with its last step stopped by iterMax. BState::iters holds
// its total PT iterations (ittot).
constexpr int kBatchMaxSteps = 64;
struct BStateVE {
    int64_t* start;       // global iteration count at which the current step began
    int* steps;           // physical steps finished
    int64_t* step_iters;  // PT iterations of each finished step, kBatchMaxSteps per instance
    int* assign;          // 1: a step has just ended and the next begins (τ_o ← τ pending)
    int64_t* next_event;  // [0]: next global iteration count at which an instance checks or ends a step
};
constexpr int kBatchTileShapes = 4;
inline void batch_tile_dims(int tile, int* tx, int* ty) {
    static const int d[kBatchTileShapes][2] = {{32, 4}, {32, 8}, {64, 4}, {32, 16}};
    *tx = d[tile][0];
    *ty = d[tile][1];
}
cudaError_t launch_batch(int tile, const BInst* d_inst, int ntiles, int ninst,
                         const Fields64& F, const BState& st, int nout, int64_t iter_last, double eps, cudaStream_t s);
cudaError_t launch_batch_ve(int tile, const BInst* d_inst, int ntiles, int ninst, const Fields64& F,
                            const BState& st, const BStateVE& sv, int64_t iter_cap, double eps, cudaStream_t s);
// Mus of one instance of the visco-elastic aspect-ratio sweep: musi in nsub circles of
// radius 1 centred at ((isub-1)*ly + ly/2, ly/2), mus0 elsewhere
cudaError_t launch_init_ve_param(const Geom& g, const Fields64& f, const Num& n, int nsub, double mus0, double musi,
                                 cudaStream_t s);
// ICs of one sweep instance: Mus/ρg = inclusion (radius2) ? (musi, rhogi) : (1, 0), pure shear ebg
cudaError_t launch_init_sweep(const Geom& g, const Fields64& f, const Num& n, double musi, double radius2,
                              double rhogi, double ebg, cudaStream_t s);

}  // namespace pts
