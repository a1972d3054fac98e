// pts_kernels64.cu -- FP64 stencil kernels of the PT iteration (all variants).
//
// Compiled with --fmad=false: no multiply-add is contracted, and every expression below
// is written in the reference's left-to-right order, so each kernel reproduces the
// reference's Float64 arithmetic bit for bit (the fixtures in tests/golden pin this).
// IEEE division and sqrt are the CUDA defaults (-prec-div=true, -prec-sqrt=true).
//
// Kernels here are the straightforward one-thread-per-point forms (two launches per PT
// iteration: compute_Pt_τ! and compute_V! + bc); the 3D visco-elastic hot path also has
// the single-pass z-streaming kernel in pts_fused3d.cuh and the z-staged compute_Pt_τ! in
// pts_zstage.cu.
#include <cooperative_groups.h>

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdlib>

#include "pts_internal.h"
#include "pts_expr64.cuh"

namespace pts {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ expression helpers

// The stress expressions (gr_of, tau_n, tau_s, tau_n_den, dsc) live in pts_expr64.cuh,
// shared with the z-staged kernels of pts_zstage.cu.
using namespace expr;

// ------------------------------------------------------------------ 3D kernels

// compute_P! + compute_τ! (roles) == compute_Pt_τ! (perf), one thread per cell (i,j,k).
// Arrays the kernel only reads (V, Gdτ, Mus, τ_o) go through the read-only data path.
template <bool EL, bool PERF>
__global__ void __launch_bounds__(256) k3_Pt_tau(Geom g, Fields64 f, Num n, int roles, int store_divV) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny || k >= nz) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    const double dvx = __ldg(&f.Vx[c + sx]) - __ldg(&f.Vx[c]);
    const double dvy = __ldg(&f.Vy[c + sy]) - __ldg(&f.Vy[c]);
    const double dvz = __ldg(&f.Vz[c + sz]) - __ldg(&f.Vz[c]);
    const double Gc = __ldg(&f.Gdt[c]);
    if (roles & ROLE_P) {
        if (PERF) {
            f.Pt[c] = f.Pt[c] - n.r * Gc * ((n._dx * dvx + n._dy * dvy) + n._dz * dvz);
        } else {
            const double dv = (dvx / n.dx + dvy / n.dy) + dvz / n.dz;
            if (store_divV) f.divV[c] = dv;
            f.Pt[c] = f.Pt[c] - n.r * Gc * dv;
        }
    }
    if (!(roles & ROLE_TAU)) return;
    const double Mc = __ldg(&f.Mus[c]);
    const double gdt = n.gdt;
    const bool nx_ = j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2;
    const bool ny_ = i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2;
    const bool nz_ = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
    if (nx_ || ny_ || nz_) {
        const double Gr = EL ? gr_of(Gc, gdt) : 0.0;
        const double den = EL ? ((1.0 + Gc / Mc) + Gr) : (1.0 + Gc / Mc);
        if (nx_) f.txx[c] = tau_n_den<EL, PERF>(f.txx[c], EL ? __ldg(&f.txx_o[c]) : 0.0, Gc, Gr, den, n.dx, n._dx, dvx);
        if (ny_) f.tyy[c] = tau_n_den<EL, PERF>(f.tyy[c], EL ? __ldg(&f.tyy_o[c]) : 0.0, Gc, Gr, den, n.dy, n._dy, dvy);
        if (nz_) f.tzz[c] = tau_n_den<EL, PERF>(f.tzz[c], EL ? __ldg(&f.tzz_o[c]) : 0.0, Gc, Gr, den, n.dz, n._dz, dvz);
    }
    // τxy on edge (x-face i, y-face j, cell k): i in [1,nx-1], j in [1,ny-1], k in [1,nz-2]
    if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2) {
        const double ag = (((__ldg(&f.Gdt[c - sx - sy]) + __ldg(&f.Gdt[c - sy])) + __ldg(&f.Gdt[c - sx])) + Gc) * 0.25;
        const double am = (((__ldg(&f.Mus[c - sx - sy]) + __ldg(&f.Mus[c - sy])) + __ldg(&f.Mus[c - sx])) + Mc) * 0.25;
        f.txy[c] = tau_s<EL, PERF>(f.txy[c], EL ? __ldg(&f.txy_o[c]) : 0.0, ag, am, gdt, n.dy, n._dy, __ldg(&f.Vx[c]) - __ldg(&f.Vx[c - sy]),
                                   n.dx, n._dx, __ldg(&f.Vy[c]) - __ldg(&f.Vy[c - sx]));
    }
    // τxz on edge (x-face i, cell j, z-face k): i in [1,nx-1], j in [1,ny-2], k in [1,nz-1]
    if (i >= 1 && j >= 1 && j <= ny - 2 && k >= 1) {
        const double ag = (((__ldg(&f.Gdt[c - sx - sz]) + __ldg(&f.Gdt[c - sz])) + __ldg(&f.Gdt[c - sx])) + Gc) * 0.25;
        const double am = (((__ldg(&f.Mus[c - sx - sz]) + __ldg(&f.Mus[c - sz])) + __ldg(&f.Mus[c - sx])) + Mc) * 0.25;
        f.txz[c] = tau_s<EL, PERF>(f.txz[c], EL ? __ldg(&f.txz_o[c]) : 0.0, ag, am, gdt, n.dz, n._dz, __ldg(&f.Vx[c]) - __ldg(&f.Vx[c - sz]),
                                   n.dx, n._dx, __ldg(&f.Vz[c]) - __ldg(&f.Vz[c - sx]));
    }
    // τyz on edge (cell i, y-face j, z-face k): i in [1,nx-2], j in [1,ny-1], k in [1,nz-1]
    if (i >= 1 && i <= nx - 2 && j >= 1 && k >= 1) {
        const double ag = (((__ldg(&f.Gdt[c - sy - sz]) + __ldg(&f.Gdt[c - sz])) + __ldg(&f.Gdt[c - sy])) + Gc) * 0.25;
        const double am = (((__ldg(&f.Mus[c - sy - sz]) + __ldg(&f.Mus[c - sz])) + __ldg(&f.Mus[c - sy])) + Mc) * 0.25;
        f.tyz[c] = tau_s<EL, PERF>(f.tyz[c], EL ? __ldg(&f.tyz_o[c]) : 0.0, ag, am, gdt, n.dz, n._dz, __ldg(&f.Vy[c]) - __ldg(&f.Vy[c - sz]),
                                   n.dy, n._dy, __ldg(&f.Vz[c]) - __ldg(&f.Vz[c - sy]));
    }
}

// Momentum residuals at interior faces (compute_Res!, Stokes3D_ve_perf.jl:92-94;
// compute_dV!/compute_Res!, Stokes3D_ve_multixpu.jl:80-82,94-96).
template <bool PERF>
__device__ __forceinline__ double res3_x(const Fields64& f, const Num& n, idx_t c, idx_t sx, idx_t sy,
                                         idx_t sz) {
    return ((dsc<PERF>(__ldg(&f.txx[c]) - __ldg(&f.txx[c - sx]), n.dx, n._dx) + dsc<PERF>(__ldg(&f.txy[c + sy]) - __ldg(&f.txy[c]), n.dy, n._dy)) +
            dsc<PERF>(__ldg(&f.txz[c + sz]) - __ldg(&f.txz[c]), n.dz, n._dz)) -
           dsc<PERF>(__ldg(&f.Pt[c]) - __ldg(&f.Pt[c - sx]), n.dx, n._dx);
}
template <bool PERF>
__device__ __forceinline__ double res3_y(const Fields64& f, const Num& n, idx_t c, idx_t sx, idx_t sy,
                                         idx_t sz) {
    return ((dsc<PERF>(__ldg(&f.tyy[c]) - __ldg(&f.tyy[c - sy]), n.dy, n._dy) + dsc<PERF>(__ldg(&f.txy[c + sx]) - __ldg(&f.txy[c]), n.dx, n._dx)) +
            dsc<PERF>(__ldg(&f.tyz[c + sz]) - __ldg(&f.tyz[c]), n.dz, n._dz)) -
           dsc<PERF>(__ldg(&f.Pt[c]) - __ldg(&f.Pt[c - sy]), n.dy, n._dy);
}
template <bool PERF>
__device__ __forceinline__ double res3_z(const Fields64& f, const Num& n, idx_t c, idx_t sx, idx_t sy,
                                         idx_t sz) {
    return ((dsc<PERF>(__ldg(&f.tzz[c]) - __ldg(&f.tzz[c - sz]), n.dz, n._dz) + dsc<PERF>(__ldg(&f.txz[c + sx]) - __ldg(&f.txz[c]), n.dx, n._dx)) +
            dsc<PERF>(__ldg(&f.tyz[c + sy]) - __ldg(&f.tyz[c]), n.dy, n._dy)) -
           dsc<PERF>(__ldg(&f.Pt[c]) - __ldg(&f.Pt[c - sz]), n.dz, n._dz);
}

// Residual of the transposed system at an interior face (adjoint mode of 3D_V): the face's
// own residual plus those of the free-slip ghost faces that copy it -- the transpose of the
// copy. A ghost's stencil is the interior one; where it reaches a stress point that does
// not exist the array holds zero (compute_τ! never writes outside its ranges). Summed in a
// fixed order: own, ghosts below/above along the first tangential axis, along the second,
// then the corner ghosts. AX = 0, 1, 2 for Vx (tangential y, z), Vy (x, z), Vz (x, y).
template <int AX>
__device__ __forceinline__ double res3_fold(const Geom& g, const Fields64& f, const Num& n, int i, int j, int k) {
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    auto R_at = [&](int ii, int jj, int kk) -> double {
        const idx_t cc = gidx32(g, ii, jj, kk);
        if (AX == 0) return res3_x<true>(f, n, cc, sx, sy, sz);
        if (AX == 1) return res3_y<true>(f, n, cc, sx, sy, sz);
        return res3_z<true>(f, n, cc, sx, sy, sz);
    };
    // tangential coordinates (a, b) and their interior bounds [1, ahi], [1, bhi]
    const int a = (AX == 0) ? j : i, b = (AX == 2) ? j : k;
    const int ahi = (AX == 0) ? g.ny - 2 : g.nx - 2, bhi = (AX == 2) ? g.ny - 2 : g.nz - 2;
    auto at = [&](int aa, int bb) -> double {
        if (AX == 0) return R_at(i, aa, bb);
        if (AX == 1) return R_at(aa, j, bb);
        return R_at(aa, bb, k);
    };
    const int ga0 = (a == 1) ? 0 : -1, ga1 = (a == ahi) ? ahi + 1 : -1;
    const int gb0 = (b == 1) ? 0 : -1, gb1 = (b == bhi) ? bhi + 1 : -1;
    double R = at(a, b);
    if (ga0 >= 0) R = R + at(ga0, b);
    if (ga1 >= 0) R = R + at(ga1, b);
    if (gb0 >= 0) R = R + at(a, gb0);
    if (gb1 >= 0) R = R + at(a, gb1);
    if (ga0 >= 0 && gb0 >= 0) R = R + at(ga0, gb0);
    if (ga0 >= 0 && gb1 >= 0) R = R + at(ga0, gb1);
    if (ga1 >= 0 && gb0 >= 0) R = R + at(ga1, gb0);
    if (ga1 >= 0 && gb1 >= 0) R = R + at(ga1, gb1);
    return R;
}

// Free-slip copies folded into the update: a face whose tangential indices are the first
// or last interior ones also writes its value onto the adjacent boundary faces. The
// reference's bc_x!/bc_y!/bc_z! calls copy whole planes in sequence
// (Stokes3D_ve_perf.jl:202-207), which leaves every boundary face equal to the face at
// its tangential indices clamped into the interior; writing from the source face gives
// exactly that, with no face read after another thread wrote it.
__device__ __forceinline__ void bc_copies(double* A, idx_t c, double v, int a, int alo, int ahi, idx_t sa, int b,
                                          int blo, int bhi, idx_t sb) {
    const int da = (a == alo) ? -1 : 0, ua = (a == ahi) ? 1 : 0;
    const int db = (b == blo) ? -1 : 0, ub = (b == bhi) ? 1 : 0;
    if (da) A[c - sa] = v;
    if (ua) A[c + sa] = v;
    if (db) A[c - sb] = v;
    if (ub) A[c + sb] = v;
    if (da && db) A[c - sa - sb] = v;
    if (da && ub) A[c - sa + sb] = v;
    if (ua && db) A[c + sa - sb] = v;
    if (ua && ub) A[c + sa + sb] = v;
}

// compute_V! (perf: Stokes3D_ve_perf.jl:83-88; roles: compute_dV! + compute_V!,
// Stokes3D_ve_multixpu.jl:79-91) with the six bc copies, one thread per face point. With
// SRC the momentum sources F join the residual: V += (R + F)*@av(dτ_Rho). With ADJ
// (adjoint mode, explicit-index form only) the residual is the folded one and the ghosts
// are not written (they stay zero).
template <bool PERF, bool SRC = false, bool ADJ = false>
__device__ __forceinline__ void v_bc3_point(const Geom& g, const Fields64& f, const Num& n, int i, int j, int k,
                                            int update) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    // Vx: source faces j in [1,ny-2], k in [1,nz-2]; updated for i in [1,nx-1]
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
        double v = f.Vx[c];
        if (update && i >= 1 && i <= nx - 1) {
            const double R0 = ADJ ? res3_fold<0>(g, f, n, i, j, k) : res3_x<PERF>(f, n, c, sx, sy, sz);
            const double R = SRC ? R0 + __ldg(&f.Fx[c]) : R0;
            v = v + R * ((__ldg(&f.dtRho[c - sx]) + __ldg(&f.dtRho[c])) * 0.5);
            f.Vx[c] = v;
        }
        if (!ADJ) bc_copies(f.Vx, c, v, j, 1, ny - 2, sy, k, 1, nz - 2, sz);
    }
    // Vy: source faces i in [1,nx-2], k in [1,nz-2]; updated for j in [1,ny-1]
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) {
        double v = f.Vy[c];
        if (update && j >= 1 && j <= ny - 1) {
            const double R0 = ADJ ? res3_fold<1>(g, f, n, i, j, k) : res3_y<PERF>(f, n, c, sx, sy, sz);
            const double R = SRC ? R0 + __ldg(&f.Fy[c]) : R0;
            v = v + R * ((__ldg(&f.dtRho[c - sy]) + __ldg(&f.dtRho[c])) * 0.5);
            f.Vy[c] = v;
        }
        if (!ADJ) bc_copies(f.Vy, c, v, i, 1, nx - 2, sx, k, 1, nz - 2, sz);
    }
    // Vz: source faces i in [1,nx-2], j in [1,ny-2]; updated for k in [1,nz-1]
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
        double v = f.Vz[c];
        if (update && k >= 1 && k <= nz - 1) {
            const double R0 = ADJ ? res3_fold<2>(g, f, n, i, j, k) : res3_z<PERF>(f, n, c, sx, sy, sz);
            const double R = SRC ? R0 + __ldg(&f.Fz[c]) : R0;
            v = v + R * ((__ldg(&f.dtRho[c - sz]) + __ldg(&f.dtRho[c])) * 0.5);
            f.Vz[c] = v;
        }
        if (!ADJ) bc_copies(f.Vz, c, v, i, 1, nx - 2, sx, j, 1, ny - 2, sy);
    }
}

template <bool PERF, bool SRC = false, bool ADJ = false>
__global__ void __launch_bounds__(256) k3_V_bc(Geom g, Fields64 f, Num n, int update) {
    v_bc3_point<PERF, SRC, ADJ>(g, f, n, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y,
                                blockIdx.z, update);
}

// The same update on the face planes k0 .. k0 + gridDim.z - 1 only: the boundary and inner
// regions of @hide_communication (Stokes3D_ve_multixpu.jl:230-239). A face update reads V
// only at its own point and writes bc copies only next to the domain's first and last
// interior planes, so disjoint plane ranges may run concurrently, in any order.
template <bool PERF>
__global__ void __launch_bounds__(256) k3_V_bc_planes(Geom g, Fields64 f, Num n, int k0) {
    v_bc3_point<PERF>(g, f, n, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y,
                      k0 + (int)blockIdx.z, 1);
}

// compute_dV! alone (Stokes3D_ve_multixpu.jl:79-84): dV = R*@av_xi(dτ_Rho) at interior faces
// (R + F with SRC).
template <bool PERF, bool SRC = false>
__global__ void k3_dV(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
        f.dVx[c] = (SRC ? res3_x<PERF>(f, n, c, sx, sy, sz) + f.Fx[c] : res3_x<PERF>(f, n, c, sx, sy, sz)) *
                   ((f.dtRho[c - sx] + f.dtRho[c]) * 0.5);
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2)
        f.dVy[c] = (SRC ? res3_y<PERF>(f, n, c, sx, sy, sz) + f.Fy[c] : res3_y<PERF>(f, n, c, sx, sy, sz)) *
                   ((f.dtRho[c - sy] + f.dtRho[c]) * 0.5);
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1)
        f.dVz[c] = (SRC ? res3_z<PERF>(f, n, c, sx, sy, sz) + f.Fz[c] : res3_z<PERF>(f, n, c, sx, sy, sz)) *
                   ((f.dtRho[c - sz] + f.dtRho[c]) * 0.5);
}

// compute_V! alone (Stokes3D_ve_multixpu.jl:86-91): @inn(V) = @inn(V) + @all(dV).
__global__ void k3_add_dV(Geom g, Fields64 f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) f.Vx[c] = f.Vx[c] + f.dVx[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2) f.Vy[c] = f.Vy[c] + f.dVy[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1) f.Vz[c] = f.Vz[c] + f.dVz[c];
}

// ------------------------------------------------------------------ 3D damped scheme (viscous)
//
// scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl on one rank. Unified positions as
// in 2D: dτPt on the cells; dτVx and dVxdτ (held in dVx) on the x-faces of Rx, and so on.

// compute_timesteps! (Stokes3D0_multixpu.jl:37-43), one thread per face/cell point
__global__ void __launch_bounds__(256) k3d_timesteps(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    const double t = 1.0 / 6.1 / (1.0 + n.beta_n) / n.Vsc * n.min_dxy2;
    if (i < nx && j < ny && k < nz) f.dtPt[c] = 6.1 * (1.0 + n.beta_n) / n.Ptsc / n.max_nxy * f.Must[c];
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)  // @av_xi(Musτ)
        f.dtVx[c] = t / ((f.Must[c - sx] + f.Must[c]) * 0.5);
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2)  // @av_yi(Musτ)
        f.dtVy[c] = t / ((f.Must[c - sy] + f.Must[c]) * 0.5);
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1)  // @av_zi(Musτ)
        f.dtVz[c] = t / ((f.Must[c - sz] + f.Must[c]) * 0.5);
}

// compute_P! (Stokes3D0_multixpu.jl:45-49) and compute_τ! (:51-59):
//   τxx = 2@inn_yz(Mus)*(@d_xi(Vx)/dx - 1/3*∇V + β_n*∇V),  τxy = 2@av_xyi(Mus)*(0.5*(@d_yi(Vx)/dy + @d_xi(Vy)/dx))
// With ROLE_TAU alone ∇V is read back from the field compute_P! stored.
__global__ void __launch_bounds__(256) k3d_Pt_tau(Geom g, Fields64 f, Num n, int roles, int store_divV) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny || k >= nz) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    const double dvx = __ldg(&f.Vx[c + sx]) - __ldg(&f.Vx[c]);
    const double dvy = __ldg(&f.Vy[c + sy]) - __ldg(&f.Vy[c]);
    const double dvz = __ldg(&f.Vz[c + sz]) - __ldg(&f.Vz[c]);
    double dv;
    if (roles & ROLE_P) {
        dv = (dvx / n.dx + dvy / n.dy) + dvz / n.dz;
        if (store_divV) f.divV[c] = dv;
        f.Pt[c] = f.Pt[c] - __ldg(&f.dtPt[c]) * dv;
    } else {
        dv = f.divV[c];
    }
    if (!(roles & ROLE_TAU)) return;
    const double Mc = __ldg(&f.Mus[c]);
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
        f.txx[c] = 2.0 * Mc * (dvx / n.dx - 1.0 / 3.0 * dv + n.beta_n * dv);
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
        f.tyy[c] = 2.0 * Mc * (dvy / n.dy - 1.0 / 3.0 * dv + n.beta_n * dv);
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
        f.tzz[c] = 2.0 * Mc * (dvz / n.dz - 1.0 / 3.0 * dv + n.beta_n * dv);
    if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2) {  // τxy edge
        const double am = (((__ldg(&f.Mus[c - sx - sy]) + __ldg(&f.Mus[c - sy])) + __ldg(&f.Mus[c - sx])) + Mc) * 0.25;
        f.txy[c] = 2.0 * am * (0.5 * ((__ldg(&f.Vx[c]) - __ldg(&f.Vx[c - sy])) / n.dy + (__ldg(&f.Vy[c]) - __ldg(&f.Vy[c - sx])) / n.dx));
    }
    if (i >= 1 && j >= 1 && j <= ny - 2 && k >= 1) {  // τxz edge
        const double am = (((__ldg(&f.Mus[c - sx - sz]) + __ldg(&f.Mus[c - sz])) + __ldg(&f.Mus[c - sx])) + Mc) * 0.25;
        f.txz[c] = 2.0 * am * (0.5 * ((__ldg(&f.Vx[c]) - __ldg(&f.Vx[c - sz])) / n.dz + (__ldg(&f.Vz[c]) - __ldg(&f.Vz[c - sx])) / n.dx));
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && k >= 1) {  // τyz edge
        const double am = (((__ldg(&f.Mus[c - sy - sz]) + __ldg(&f.Mus[c - sz])) + __ldg(&f.Mus[c - sy])) + Mc) * 0.25;
        f.tyz[c] = 2.0 * am * (0.5 * ((__ldg(&f.Vy[c]) - __ldg(&f.Vy[c - sz])) / n.dz + (__ldg(&f.Vz[c]) - __ldg(&f.Vz[c - sy])) / n.dy));
    }
}

// compute_dV! + compute_V! + the six bc copies (Stokes3D0_multixpu.jl:61-76,186-193):
//   dVxdτ = dampX*dVxdτ + Rx,  @inn(Vx) = @inn(Vx) + dτVx*dVxdτ.  update = 0: copies only.
__global__ void __launch_bounds__(256) k3d_V_bc(Geom g, Fields64 f, Num n, int update) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
        double v = f.Vx[c];
        if (update && i >= 1 && i <= nx - 1) {
            const double r = n.dampX * f.dVx[c] + res3_x<false>(f, n, c, sx, sy, sz);
            f.dVx[c] = r;
            v = v + __ldg(&f.dtVx[c]) * r;
            f.Vx[c] = v;
        }
        bc_copies(f.Vx, c, v, j, 1, ny - 2, sy, k, 1, nz - 2, sz);
    }
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) {
        double v = f.Vy[c];
        if (update && j >= 1 && j <= ny - 1) {
            const double r = n.dampY * f.dVy[c] + res3_y<false>(f, n, c, sx, sy, sz);
            f.dVy[c] = r;
            v = v + __ldg(&f.dtVy[c]) * r;
            f.Vy[c] = v;
        }
        bc_copies(f.Vy, c, v, i, 1, nx - 2, sx, k, 1, nz - 2, sz);
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
        double v = f.Vz[c];
        if (update && k >= 1 && k <= nz - 1) {
            const double r = n.dampZ * f.dVz[c] + res3_z<false>(f, n, c, sx, sy, sz);
            f.dVz[c] = r;
            v = v + __ldg(&f.dtVz[c]) * r;
            f.Vz[c] = v;
        }
        bc_copies(f.Vz, c, v, i, 1, nx - 2, sx, j, 1, ny - 2, sy);
    }
}

// compute_dV! alone (Stokes3D0_multixpu.jl:61-69): R and the damped rates.
__global__ void k3d_dV(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
        const double R = res3_x<false>(f, n, c, sx, sy, sz);
        f.Rx[c] = R;
        f.dVx[c] = n.dampX * f.dVx[c] + R;
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2) {
        const double R = res3_y<false>(f, n, c, sx, sy, sz);
        f.Ry[c] = R;
        f.dVy[c] = n.dampY * f.dVy[c] + R;
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1) {
        const double R = res3_z<false>(f, n, c, sx, sy, sz);
        f.Rz[c] = R;
        f.dVz[c] = n.dampZ * f.dVz[c] + R;
    }
}

// compute_V! alone (Stokes3D0_multixpu.jl:71-76): @inn(V) = @inn(V) + dτV*dVdτ
__global__ void k3d_add_dV(Geom g, Fields64 f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) f.Vx[c] = f.Vx[c] + f.dtVx[c] * f.dVx[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2) f.Vy[c] = f.Vy[c] + f.dtVy[c] * f.dVy[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1) f.Vz[c] = f.Vz[c] + f.dtVz[c] * f.dVz[c];
}

// ------------------------------------------------------------------ 2D kernels

// compute_P! + compute_τ! for the three 2D scripts:
//   V2D        Stokes2D.jl:33-44      VE2D  Stokes2D_ve.jl:42-55     VE2D_PERF  Stokes2D_ve_perf.jl:47-53
// (the body is a device function so the batched sweep kernel runs the same code per point)
template <int VAR>
__device__ __forceinline__ void pt_tau_2d(const Geom& g, const Fields64& f, const Num& n, int i, int j, int roles,
                                          int store_divV) {
    const int nx = g.nx, ny = g.ny;
    if (i >= nx || j >= ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    const double dvx = f.Vx[c + sx] - f.Vx[c];
    const double dvy = f.Vy[c + sy] - f.Vy[c];
    const double Gc = f.Gdt[c];
    if (roles & ROLE_P) {
        if (VAR == VE2D_PERF) {
            f.Pt[c] = f.Pt[c] - n.r * Gc * (n._dx * dvx + n._dy * dvy);
        } else {
            const double dv = dvx / n.dx + dvy / n.dy;
            if (store_divV) f.divV[c] = dv;
            f.Pt[c] = f.Pt[c] - n.r * Gc * dv;
        }
    }
    if (!(roles & ROLE_TAU)) return;
    const double Mc = f.Mus[c];
    if (VAR == V2D) {
        f.txx[c] = (f.txx[c] + ((2.0 * Gc) * dvx) / n.dx) / (Gc / Mc + 1.0);
        f.tyy[c] = (f.tyy[c] + ((2.0 * Gc) * dvy) / n.dy) / (Gc / Mc + 1.0);
    } else {
        const double Gr = gr_of(Gc, n.gdt);
        const double ex = (VAR == VE2D_PERF) ? n._dx * dvx : dvx / n.dx;
        const double ey = (VAR == VE2D_PERF) ? n._dy * dvy : dvy / n.dy;
        f.txx[c] = ((f.txx[c] + f.txx_o[c] * Gr) + (2.0 * Gc) * ex) / ((1.0 + Gc / Mc) + Gr);
        f.tyy[c] = ((f.tyy[c] + f.tyy_o[c] * Gr) + (2.0 * Gc) * ey) / ((1.0 + Gc / Mc) + Gr);
    }
    // τxy on the vertex (x-face i, y-face j): i in [1,nx-1], j in [1,ny-1]
    if (i >= 1 && j >= 1) {
        const double ag = (((f.Gdt[c - sx - sy] + f.Gdt[c - sy]) + f.Gdt[c - sx]) + Gc) * 0.25;
        const double am = (((f.Mus[c - sx - sy] + f.Mus[c - sy]) + f.Mus[c - sx]) + Mc) * 0.25;
        const double d1 = f.Vx[c] - f.Vx[c - sy];  // @d_yi(Vx)
        const double d2 = f.Vy[c] - f.Vy[c - sx];  // @d_xi(Vy)
        if (VAR == V2D) {
            f.txy[c] = (f.txy[c] + (2.0 * ag) * (0.5 * (d1 / n.dy + d2 / n.dx))) / (ag / am + 1.0);
        } else if (VAR == VE2D) {
            const double Gr = gr_of(ag, n.gdt);
            f.txy[c] = ((f.txy[c] + f.txy_o[c] * Gr) + (2.0 * ag) * (0.5 * (d1 / n.dy + d2 / n.dx))) /
                       ((1.0 + ag / am) + Gr);
        } else {
            const double Gr = gr_of(ag, n.gdt);
            f.txy[c] = ((f.txy[c] + f.txy_o[c] * Gr) + ((2.0 * ag) * 0.5) * (n._dy * d1 + n._dx * d2)) /
                       ((1.0 + ag / am) + Gr);
        }
    }
}

template <int VAR>
__global__ void __launch_bounds__(256) k2_Pt_tau(Geom g, Fields64 f, Num n, int roles, int store_divV) {
    pt_tau_2d<VAR>(g, f, n, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y, roles,
                   store_divV);
}

template <bool PERF>
__device__ __forceinline__ double res2_x(const Fields64& f, const Num& n, idx_t c, idx_t sx, idx_t sy) {
    return (dsc<PERF>(f.txx[c] - f.txx[c - sx], n.dx, n._dx) + dsc<PERF>(f.txy[c + sy] - f.txy[c], n.dy, n._dy)) -
           dsc<PERF>(f.Pt[c] - f.Pt[c - sx], n.dx, n._dx);
}
// With RHOG the buoyancy term of Stokes2D_param.jl:59: Ry -= @av_yi(ρg).
template <bool PERF, bool RHOG = false>
__device__ __forceinline__ double res2_y(const Fields64& f, const Num& n, idx_t c, idx_t sx, idx_t sy) {
    const double R = (dsc<PERF>(f.tyy[c] - f.tyy[c - sy], n.dy, n._dy) + dsc<PERF>(f.txy[c + sx] - f.txy[c], n.dx, n._dx)) -
                     dsc<PERF>(f.Pt[c] - f.Pt[c - sy], n.dy, n._dy);
    if (RHOG) return R - (f.rhog[c - sy] + f.rhog[c]) * 0.5;
    return R;
}

// compute_V! (+ compute_dV!) with bc_y!(Vx), bc_x!(Vy) (Stokes2D.jl:46-58,133-134;
// Stokes2D_ve_perf.jl:55-59,151-152).
template <int VAR, bool RHOG = false>
__device__ __forceinline__ void v_bc_2d(const Geom& g, const Fields64& f, const Num& n, int i, int j, int update) {
    constexpr bool PERF = (VAR == VE2D_PERF);
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    if (j >= 1 && j <= ny - 2) {  // Vx source faces (bc_y!)
        double v = f.Vx[c];
        if (update && i >= 1 && i <= nx - 1) {
            v = v + res2_x<PERF>(f, n, c, sx, sy) * ((f.dtRho[c - sx] + f.dtRho[c]) * 0.5);
            f.Vx[c] = v;
        }
        if (j == 1) f.Vx[c - sy] = v;
        if (j == ny - 2) f.Vx[c + sy] = v;
    }
    if (i >= 1 && i <= nx - 2) {  // Vy source faces (bc_x!)
        double v = f.Vy[c];
        if (update && j >= 1 && j <= ny - 1) {
            v = v + res2_y<PERF, RHOG>(f, n, c, sx, sy) * ((f.dtRho[c - sy] + f.dtRho[c]) * 0.5);
            f.Vy[c] = v;
        }
        if (i == 1) f.Vy[c - sx] = v;
        if (i == nx - 2) f.Vy[c + sx] = v;
    }
}

template <int VAR>
__global__ void __launch_bounds__(256) k2_V_bc(Geom g, Fields64 f, Num n, int update) {
    v_bc_2d<VAR>(g, f, n, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y, update);
}

// compute_dV! alone; Stokes2D.jl:46-52 also stores Rx, Ry.
template <int VAR>
__global__ void k2_dV(Geom g, Fields64 f, Num n) {
    constexpr bool PERF = (VAR == VE2D_PERF);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) {
        const double R = res2_x<PERF>(f, n, c, sx, sy);
        if (VAR == V2D) f.Rx[c] = R;
        f.dVx[c] = R * ((f.dtRho[c - sx] + f.dtRho[c]) * 0.5);
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) {
        const double R = res2_y<PERF>(f, n, c, sx, sy);
        if (VAR == V2D) f.Ry[c] = R;
        f.dVy[c] = R * ((f.dtRho[c - sy] + f.dtRho[c]) * 0.5);
    }
}

__global__ void k2_add_dV(Geom g, Fields64 f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) f.Vx[c] = f.Vx[c] + f.dVx[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) f.Vy[c] = f.Vy[c] + f.dVy[c];
}

// ------------------------------------------------------------------ 2D damped scheme
//
// scripts/previous_damp/Stokes2D0.jl (viscous) and Stokes2D_ve0.jl (Maxwell VE). Unified
// positions: dτPt on the cells; dτVx and the damped rate dVxdτ (held in dVx) on the x-faces
// of Rx (i in [1,nx-1], j in [1,ny-2]); dτVy, dVydτ (dVy) on the y-faces of Ry.

// compute_timesteps! (Stokes2D_ve0.jl:27-32, Stokes2D0.jl:26-31)
__global__ void __launch_bounds__(256) k2d_timesteps(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    if (i < nx && j < ny) f.dtPt[c] = 4.1 * (1.0 + n.beta_n) / n.Ptsc / n.max_nxy * f.Must[c];
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2)  // @av_xi(Musτ)
        f.dtVx[c] = 1.0 / 4.1 / n.Vsc * n.min_dxy2 / ((f.Must[c - sx] + f.Must[c]) * 0.5) / (1.0 + n.beta_n);
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1)  // @av_yi(Musτ)
        f.dtVy[c] = 1.0 / 4.1 / n.Vsc * n.min_dxy2 / ((f.Must[c - sy] + f.Must[c]) * 0.5) / (1.0 + n.beta_n);
}

// compute_P! (Stokes2D_ve0.jl:41-45): ∇V, Pt = Pt - dτPt*∇V; then compute_τ! with the
// numerical compressibility β_n: viscous (Stokes2D0.jl:39-44)
//   τxx = 2Mus*(d_xa(Vx)/dx - 1/3*∇V + β_n*∇V),  τxy = 2@av(Mus)*(0.5*(d_yi(Vx)/dy + d_xi(Vy)/dx))
// Maxwell (Stokes2D_ve0.jl:47-54), Xsi = Mus/(G*dt):
//   τxx = τxx_o*Xsi/(Xsi+1) + 2Mus/(Xsi+1)*(...),  τxy likewise with @av(Mus)
// With ROLE_TAU alone ∇V is read back from the field compute_P! stored.
template <bool EL>
__global__ void __launch_bounds__(256) k2d_Pt_tau(Geom g, Fields64 f, Num n, int roles, int store_divV) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    const double dvx = f.Vx[c + sx] - f.Vx[c];
    const double dvy = f.Vy[c + sy] - f.Vy[c];
    double dv;
    if (roles & ROLE_P) {
        dv = dvx / n.dx + dvy / n.dy;
        if (store_divV) f.divV[c] = dv;
        f.Pt[c] = f.Pt[c] - f.dtPt[c] * dv;
    } else {
        dv = f.divV[c];
    }
    if (!(roles & ROLE_TAU)) return;
    const double Mc = f.Mus[c];
    const double ex = dvx / n.dx - 1.0 / 3.0 * dv + n.beta_n * dv;
    const double ey = dvy / n.dy - 1.0 / 3.0 * dv + n.beta_n * dv;
    if (EL) {
        const double X = Mc / n.gdt;
        f.txx[c] = f.txx_o[c] * X / (X + 1.0) + 2.0 * Mc / (X + 1.0) * ex;
        f.tyy[c] = f.tyy_o[c] * X / (X + 1.0) + 2.0 * Mc / (X + 1.0) * ey;
    } else {
        f.txx[c] = 2.0 * Mc * ex;
        f.tyy[c] = 2.0 * Mc * ey;
    }
    if (i >= 1 && j >= 1) {  // τxy on the vertex (x-face i, y-face j)
        const double am = (((f.Mus[c - sx - sy] + f.Mus[c - sy]) + f.Mus[c - sx]) + Mc) * 0.25;
        const double exy = 0.5 * ((f.Vx[c] - f.Vx[c - sy]) / n.dy + (f.Vy[c] - f.Vy[c - sx]) / n.dx);
        if (EL) {
            const double X = am / n.gdt;
            f.txy[c] = f.txy_o[c] * X / (X + 1.0) + 2.0 * am / (X + 1.0) * exy;
        } else {
            f.txy[c] = 2.0 * am * exy;
        }
    }
}

// compute_dV! + compute_V! + bc_y!(Vx), bc_x!(Vy) (Stokes2D_ve0.jl:56-68,156-157):
//   dVxdτ = dampX*dVxdτ + Rx,  @inn(Vx) = @inn(Vx) + dτVx*dVxdτ
// With update = 0 only the free-slip copies.
__global__ void __launch_bounds__(256) k2d_V_bc(Geom g, Fields64 f, Num n, int update) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    if (j >= 1 && j <= ny - 2) {  // Vx source faces (bc_y!)
        double v = f.Vx[c];
        if (update && i >= 1 && i <= nx - 1) {
            const double r = n.dampX * f.dVx[c] + res2_x<false>(f, n, c, sx, sy);
            f.dVx[c] = r;
            v = v + __ldg(&f.dtVx[c]) * r;
            f.Vx[c] = v;
        }
        if (j == 1) f.Vx[c - sy] = v;
        if (j == ny - 2) f.Vx[c + sy] = v;
    }
    if (i >= 1 && i <= nx - 2) {  // Vy source faces (bc_x!)
        double v = f.Vy[c];
        if (update && j >= 1 && j <= ny - 1) {
            const double r = n.dampY * f.dVy[c] + res2_y<false>(f, n, c, sx, sy);
            f.dVy[c] = r;
            v = v + __ldg(&f.dtVy[c]) * r;
            f.Vy[c] = v;
        }
        if (i == 1) f.Vy[c - sx] = v;
        if (i == nx - 2) f.Vy[c + sx] = v;
    }
}

// compute_dV! alone (Stokes2D_ve0.jl:56-62): Rx, Ry and the damped rates.
__global__ void k2d_dV(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    const idx_t sx = 1, sy = g.px;
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) {
        const double R = res2_x<false>(f, n, c, sx, sy);
        f.Rx[c] = R;
        f.dVx[c] = n.dampX * f.dVx[c] + R;
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) {
        const double R = res2_y<false>(f, n, c, sx, sy);
        f.Ry[c] = R;
        f.dVy[c] = n.dampY * f.dVy[c] + R;
    }
}

// compute_V! alone (Stokes2D_ve0.jl:64-68): @inn(V) = @inn(V) + dτV*dVdτ
__global__ void k2d_add_dV(Geom g, Fields64 f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) f.Vx[c] = f.Vx[c] + f.dtVx[c] * f.dVx[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) f.Vy[c] = f.Vy[c] + f.dtVy[c] * f.dVy[c];
}

// ------------------------------------------------------------------ convergence check

struct Acc {
    double s[4];   // Σ Rx², Σ Ry², Σ Rz², Σ ∇V²
    double vmin, vmax, pmin, pmax;
};

__device__ __forceinline__ void acc_init(Acc& a) {
    a.s[0] = a.s[1] = a.s[2] = a.s[3] = 0.0;
    a.vmin = a.pmin = DBL_MAX;
    a.vmax = a.pmax = -DBL_MAX;
}

// Deterministic block reduction (fixed shuffle tree, then fixed cross-warp order).
__device__ void acc_block_store(Acc& a, double* out) {
    for (int o = 16; o > 0; o >>= 1) {
        for (int q = 0; q < 4; ++q) a.s[q] += __shfl_down_sync(kFull, a.s[q], o);
        a.vmin = fmin(a.vmin, __shfl_down_sync(kFull, a.vmin, o));
        a.vmax = fmax(a.vmax, __shfl_down_sync(kFull, a.vmax, o));
        a.pmin = fmin(a.pmin, __shfl_down_sync(kFull, a.pmin, o));
        a.pmax = fmax(a.pmax, __shfl_down_sync(kFull, a.pmax, o));
    }
    __shared__ double sm[32][kCheckSlots];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nw = (nthr + 31) >> 5;
    if (lane == 0) {
        sm[warp][0] = a.s[0]; sm[warp][1] = a.s[1]; sm[warp][2] = a.s[2]; sm[warp][3] = a.s[3];
        sm[warp][4] = a.vmin; sm[warp][5] = a.vmax; sm[warp][6] = a.pmin; sm[warp][7] = a.pmax;
    }
    __syncthreads();
    if (tid == 0) {
        double r[kCheckSlots];
        for (int q = 0; q < kCheckSlots; ++q) r[q] = sm[0][q];
        for (int w = 1; w < nw; ++w) {
            for (int q = 0; q < 4; ++q) r[q] += sm[w][q];
            r[4] = fmin(r[4], sm[w][4]); r[5] = fmax(r[5], sm[w][5]);
            r[6] = fmin(r[6], sm[w][6]); r[7] = fmax(r[7], sm[w][7]);
        }
        const int64_t b = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
        for (int q = 0; q < kCheckSlots; ++q) out[b * kCheckSlots + q] = r[q];
    }
}

// 3D check: compute_Res! (perf: ∇V from the current V) / stored ∇V (roles), the residual
// arrays (R + F with SRC, folded with ADJ) and the per-block partial norms and extrema.
// Blocks stride over z.
template <bool PERF, bool SRC = false, bool ADJ = false>
__global__ void __launch_bounds__(256) k3_check(Geom g, Fields64 f, Num n, double* partials) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    Acc a;
    acc_init(a);
    if (i <= nx && j < ny) {
        for (int k = blockIdx.z; k < nz; k += gridDim.z) {
            const idx_t c = gidx32(g, i, j, k);
            const double vx = f.Vx[c];
            a.vmin = fmin(a.vmin, vx);
            a.vmax = fmax(a.vmax, vx);
            if (i < nx) {
                const double p = f.Pt[c];
                a.pmin = fmin(a.pmin, p);
                a.pmax = fmax(a.pmax, p);
                double dv;
                if (PERF) {
                    dv = (n._dx * (f.Vx[c + sx] - f.Vx[c]) + n._dy * (f.Vy[c + sy] - f.Vy[c])) +
                         n._dz * (f.Vz[c + sz] - f.Vz[c]);
                    f.divV[c] = dv;
                } else {
                    dv = f.divV[c];
                }
                a.s[3] += dv * dv;
            }
            if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
                const double R0 = ADJ ? res3_fold<0>(g, f, n, i, j, k) : res3_x<PERF>(f, n, c, sx, sy, sz);
                const double R = SRC ? R0 + f.Fx[c] : R0;
                f.Rx[c] = R;
                a.s[0] += R * R;
            }
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2) {
                const double R0 = ADJ ? res3_fold<1>(g, f, n, i, j, k) : res3_y<PERF>(f, n, c, sx, sy, sz);
                const double R = SRC ? R0 + f.Fy[c] : R0;
                f.Ry[c] = R;
                a.s[1] += R * R;
            }
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1) {
                const double R0 = ADJ ? res3_fold<2>(g, f, n, i, j, k) : res3_z<PERF>(f, n, c, sx, sy, sz);
                const double R = SRC ? R0 + f.Fz[c] : R0;
                f.Rz[c] = R;
                a.s[2] += R * R;
            }
        }
    }
    acc_block_store(a, partials);
}

template <int VAR>
__global__ void __launch_bounds__(256) k2_check(Geom g, Fields64 f, Num n, double* partials) {
    constexpr bool PERF = (VAR == VE2D_PERF);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny;
    const idx_t sx = 1, sy = g.px;
    Acc a;
    acc_init(a);
    if (i <= nx && j < ny) {
        const idx_t c = gidx32(g, i, j, 0);
        const double vx = f.Vx[c];
        a.vmin = vx;
        a.vmax = vx;
        if (i < nx) {
            a.pmin = a.pmax = f.Pt[c];
            double dv;
            if (PERF) {
                dv = n._dx * (f.Vx[c + sx] - f.Vx[c]) + n._dy * (f.Vy[c + sy] - f.Vy[c]);
                f.divV[c] = dv;
            } else {
                dv = f.divV[c];
            }
            a.s[3] = dv * dv;
        }
        if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) {
            const double R = res2_x<PERF>(f, n, c, sx, sy);
            f.Rx[c] = R;
            a.s[0] = R * R;
        }
        if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) {
            const double R = res2_y<PERF>(f, n, c, sx, sy);
            f.Ry[c] = R;
            a.s[1] = R * R;
        }
    }
    acc_block_store(a, partials);
}

// Finaliser: fixed-order sum of the block partials, then the norms of the check
// (Stokes3D_ve_perf.jl:213-218): norm_R = norm(R)/(Pmax-Pmin)*lx/sqrt(length(R)).
__global__ void k_check_finalize(const double* partials, int nblocks, double4 sc, double lenRx, double lenRy,
                                 double lenRz, double lenDiv, int ndim, CheckResult* out) {
    __shared__ double sm[256][kCheckSlots];
    const int t = threadIdx.x;
    double r[kCheckSlots] = {0.0, 0.0, 0.0, 0.0, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    for (int b = t; b < nblocks; b += blockDim.x) {
        const double* p = partials + (int64_t)b * kCheckSlots;
        for (int q = 0; q < 4; ++q) r[q] += p[q];
        r[4] = fmin(r[4], p[4]); r[5] = fmax(r[5], p[5]);
        r[6] = fmin(r[6], p[6]); r[7] = fmax(r[7], p[7]);
    }
    for (int q = 0; q < kCheckSlots; ++q) sm[t][q] = r[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) {
            for (int q = 0; q < 4; ++q) sm[t][q] += sm[t + s][q];
            sm[t][4] = fmin(sm[t][4], sm[t + s][4]); sm[t][5] = fmax(sm[t][5], sm[t + s][5]);
            sm[t][6] = fmin(sm[t][6], sm[t + s][6]); sm[t][7] = fmax(sm[t][7], sm[t + s][7]);
        }
        __syncthreads();
    }
    if (t == 0) {
        const double dP = sm[0][7] - sm[0][6], dV = sm[0][5] - sm[0][4];
        CheckResult c;
        c.nRx = sqrt(sm[0][0]) / dP * sc.x / sqrt(lenRx);
        c.nRy = sqrt(sm[0][1]) / dP * sc.y / sqrt(lenRy);
        c.nRz = (ndim == 3) ? sqrt(sm[0][2]) / dP * sc.z / sqrt(lenRz) : 0.0;
        c.ndiv = sqrt(sm[0][3]) / dV * sc.w / sqrt(lenDiv);
        c.vmin = sm[0][4]; c.vmax = sm[0][5]; c.pmin = sm[0][6]; c.pmax = sm[0][7];
        c.sRx = sm[0][0]; c.sRy = sm[0][1]; c.sRz = sm[0][2]; c.sdiv = sm[0][3];
        const bool bad = isnan(c.nRx) || isnan(c.nRy) || isnan(c.nRz) || isnan(c.ndiv);
        c.err = bad ? NAN : fmax(fmax(c.nRx, c.nRy), fmax(c.nRz, c.ndiv));
        c.flag_nan = bad ? 1.0 : 0.0;
        *out = c;
    }
}

// ------------------------------------------------------------------ adjoint of the 3D viscous solve
//
// The forward 3D_V iterate converges to R = D·τ(B V) − ∇P = 0, ∇·(B V) = 0 with τ = 2μ ε̇,
// B the free-slip extension (ghosts copy their interior faces). For a misfit J(V), with λ the
// solution of the transposed system (adjoint mode: ghosts zero, ghost residuals folded onto
// the faces they copy),
//   ∂J/∂μ_c = −[2 Σ_n ε̇_n(V) ε̇_n(λ) + Σ_{edges e around c} ε̇_s(V) ε̇_s(λ)]
// (normal rates where compute_τ! updates them, shear rates on the interior edges, each edge
// averaging 4 cells): λᵀ ∂R/∂μ_c, as τ is linear in μ and W = diag(1 normal, 2 shear).

// Shear strain rates in the explicit-index (·_dx) form of the 3D_V kernels.
__device__ __forceinline__ double rate_xy(const Fields64& f, const Num& n, idx_t e, idx_t sx, idx_t sy) {
    return 0.5 * (n._dy * (f.Vx[e] - f.Vx[e - sy]) + n._dx * (f.Vy[e] - f.Vy[e - sx]));
}
__device__ __forceinline__ double rate_xz(const Fields64& f, const Num& n, idx_t e, idx_t sx, idx_t sz) {
    return 0.5 * (n._dz * (f.Vx[e] - f.Vx[e - sz]) + n._dx * (f.Vz[e] - f.Vz[e - sx]));
}
__device__ __forceinline__ double rate_yz(const Fields64& f, const Num& n, idx_t e, idx_t sy, idx_t sz) {
    return 0.5 * (n._dz * (f.Vy[e] - f.Vy[e - sz]) + n._dy * (f.Vz[e] - f.Vz[e - sy]));
}

// τ = 2·Mus·ε̇(V) on the points compute_τ! updates (the fixed point of the viscous update).
__global__ void __launch_bounds__(256) k3_tau_exact(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    const double Mc = f.Mus[c];
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) f.txx[c] = 2.0 * Mc * (n._dx * (f.Vx[c + sx] - f.Vx[c]));
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) f.tyy[c] = 2.0 * Mc * (n._dy * (f.Vy[c + sy] - f.Vy[c]));
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) f.tzz[c] = 2.0 * Mc * (n._dz * (f.Vz[c + sz] - f.Vz[c]));
    if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2) {
        const double am = (((f.Mus[c - sx - sy] + f.Mus[c - sy]) + f.Mus[c - sx]) + Mc) * 0.25;
        f.txy[c] = 2.0 * am * rate_xy(f, n, c, sx, sy);
    }
    if (i >= 1 && j >= 1 && j <= ny - 2 && k >= 1) {
        const double am = (((f.Mus[c - sx - sz] + f.Mus[c - sz]) + f.Mus[c - sx]) + Mc) * 0.25;
        f.txz[c] = 2.0 * am * rate_xz(f, n, c, sx, sz);
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && k >= 1) {
        const double am = (((f.Mus[c - sy - sz] + f.Mus[c - sz]) + f.Mus[c - sy]) + Mc) * 0.25;
        f.tyz[c] = 2.0 * am * rate_yz(f, n, c, sy, sz);
    }
}

// ∂J/∂log μ_c = μ_c ∂J/∂μ_c at every cell, from the forward fields f and the adjoint fields a
// (same geometry), written to f.grad. The edge sums run in a fixed order.
__global__ void __launch_bounds__(256) k3_grad_logmu(Geom g, Fields64 f, Fields64 a, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    double nrm = 0.0, shr = 0.0;
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
        nrm = nrm + (n._dx * (f.Vx[c + sx] - f.Vx[c])) * (n._dx * (a.Vx[c + sx] - a.Vx[c]));
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
        nrm = nrm + (n._dy * (f.Vy[c + sy] - f.Vy[c])) * (n._dy * (a.Vy[c + sy] - a.Vy[c]));
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
        nrm = nrm + (n._dz * (f.Vz[c + sz] - f.Vz[c])) * (n._dz * (a.Vz[c + sz] - a.Vz[c]));
    // xy edges (x-face i', y-face j', cell k): i' in {i, i+1} ∩ [1,nx-1], j' in {j, j+1} ∩ [1,ny-1]
    if (k >= 1 && k <= nz - 2)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                const int ie = i + di, je = j + dj;
                if (ie < 1 || ie > nx - 1 || je < 1 || je > ny - 1) continue;
                const idx_t e = c + di * sx + dj * sy;
                shr = shr + rate_xy(f, n, e, sx, sy) * rate_xy(a, n, e, sx, sy);
            }
    // xz edges (x-face i', cell j, z-face k')
    if (j >= 1 && j <= ny - 2)
        for (int dk = 0; dk < 2; ++dk)
            for (int di = 0; di < 2; ++di) {
                const int ie = i + di, ke = k + dk;
                if (ie < 1 || ie > nx - 1 || ke < 1 || ke > nz - 1) continue;
                const idx_t e = c + di * sx + dk * sz;
                shr = shr + rate_xz(f, n, e, sx, sz) * rate_xz(a, n, e, sx, sz);
            }
    // yz edges (cell i, y-face j', z-face k')
    if (i >= 1 && i <= nx - 2)
        for (int dk = 0; dk < 2; ++dk)
            for (int dj = 0; dj < 2; ++dj) {
                const int je = j + dj, ke = k + dk;
                if (je < 1 || je > ny - 1 || ke < 1 || ke > nz - 1) continue;
                const idx_t e = c + dj * sy + dk * sz;
                shr = shr + rate_yz(f, n, e, sy, sz) * rate_yz(a, n, e, sy, sz);
            }
    f.grad[c] = -(f.Mus[c] * (2.0 * nrm + shr));
}

// One physical step's term of ∂J/∂log μ for the visco-elastic operator (3D_VE_PERF), from the
// forward step's converged stresses τ (f) and the adjoint step's stresses τa (a). A converged
// VE step has τ = η(2ε̇ + τ_o/(G dt)), η = 1/(1/μ + 1/(G dt)) (μ̄ on the shear edges); its
// stress multiplier is W·τa/(2η), and the μ-derivative of the constraint gives
//   ∂J/∂log μ_c += −[Σ_n τa_n τ_n/(2 μ_c) + μ_c Σ_{edges e around c} τa_e τ_e/(4 μ̄_e²)].
// ADD accumulates into f.grad (the steps of a time loop), otherwise it overwrites.
template <bool ADD>
__global__ void __launch_bounds__(256) k3_grad_logmu_ve(Geom g, Fields64 f, Fields64 a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    const double Mc = f.Mus[c];
    double nrm = 0.0, shr = 0.0;
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) nrm = nrm + a.txx[c] * f.txx[c];
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) nrm = nrm + a.tyy[c] * f.tyy[c];
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) nrm = nrm + a.tzz[c] * f.tzz[c];
    auto mbar = [&](idx_t e, idx_t s1, idx_t s2) {
        return (((f.Mus[e - s1 - s2] + f.Mus[e - s2]) + f.Mus[e - s1]) + f.Mus[e]) * 0.25;
    };
    if (k >= 1 && k <= nz - 2)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                const int ie = i + di, je = j + dj;
                if (ie < 1 || ie > nx - 1 || je < 1 || je > ny - 1) continue;
                const idx_t e = c + di * sx + dj * sy;
                const double m = mbar(e, sx, sy);
                shr = shr + a.txy[e] * f.txy[e] / (m * m);
            }
    if (j >= 1 && j <= ny - 2)
        for (int dk = 0; dk < 2; ++dk)
            for (int di = 0; di < 2; ++di) {
                const int ie = i + di, ke = k + dk;
                if (ie < 1 || ie > nx - 1 || ke < 1 || ke > nz - 1) continue;
                const idx_t e = c + di * sx + dk * sz;
                const double m = mbar(e, sx, sz);
                shr = shr + a.txz[e] * f.txz[e] / (m * m);
            }
    if (i >= 1 && i <= nx - 2)
        for (int dk = 0; dk < 2; ++dk)
            for (int dj = 0; dj < 2; ++dj) {
                const int je = j + dj, ke = k + dk;
                if (je < 1 || je > ny - 1 || ke < 1 || ke > nz - 1) continue;
                const idx_t e = c + dj * sy + dk * sz;
                const double m = mbar(e, sy, sz);
                shr = shr + a.tyz[e] * f.tyz[e] / (m * m);
            }
    const double t = -(nrm / (2.0 * Mc) + Mc * (shr * 0.25));
    f.grad[c] = ADD ? f.grad[c] + t : t;
}

// ------------------------------------------------------------------ batched 2D sweep (persistent)

// Block reduction of one Acc into out[0..7] (fixed order, as acc_block_store).
__device__ void acc_block_store_to(Acc& a, double* out) {
    for (int o = 16; o > 0; o >>= 1) {
        for (int q = 0; q < 4; ++q) a.s[q] += __shfl_down_sync(kFull, a.s[q], o);
        a.vmin = fmin(a.vmin, __shfl_down_sync(kFull, a.vmin, o));
        a.vmax = fmax(a.vmax, __shfl_down_sync(kFull, a.vmax, o));
        a.pmin = fmin(a.pmin, __shfl_down_sync(kFull, a.pmin, o));
        a.pmax = fmax(a.pmax, __shfl_down_sync(kFull, a.pmax, o));
    }
    __shared__ double sm[32][kCheckSlots];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    if ((tid & 31) == 0) {
        const int w = tid >> 5;
        sm[w][0] = a.s[0]; sm[w][1] = a.s[1]; sm[w][2] = a.s[2]; sm[w][3] = a.s[3];
        sm[w][4] = a.vmin; sm[w][5] = a.vmax; sm[w][6] = a.pmin; sm[w][7] = a.pmax;
    }
    __syncthreads();
    if (tid == 0) {
        double r[kCheckSlots];
        for (int q = 0; q < kCheckSlots; ++q) r[q] = sm[0][q];
        for (int w = 1; w < nw; ++w) {
            for (int q = 0; q < 4; ++q) r[q] += sm[w][q];
            r[4] = fmin(r[4], sm[w][4]); r[5] = fmax(r[5], sm[w][5]);
            r[6] = fmin(r[6], sm[w][6]); r[7] = fmax(r[7], sm[w][7]);
        }
        for (int q = 0; q < kCheckSlots; ++q) out[q] = r[q];
    }
    __syncthreads();
}

// The arrays of the sweep (one arena per field, instances back to back).
struct SweepF {
    double *Pt, *Vx, *Vy, *txx, *tyy, *txy, *Mus, *divV, *Rx, *Ry, *rhog;
};
__device__ __forceinline__ SweepF sweep_at(const SweepF& F, int64_t off) {
    return {F.Pt + off,  F.Vx + off,   F.Vy + off, F.txx + off, F.tyy + off, F.txy + off,
            F.Mus + off, F.divV + off, F.Rx + off, F.Ry + off,  F.rhog + off};
}

// What a tile of the sweep needs of its instance, loaded into registers when a block's walk
// enters the instance.
// The subexpressions that depend on the instance only (1/Gdτ, @av(Gdτ), 1/@av(Gdτ),
// @av_xi(dτ_Rho)) are formed here once, with the reference's operations, so every point
// uses the same bits it would compute itself.
struct SweepP {
    int nx, ny, px, py, ntx, tile0;
    int64_t off, cap;
    double dx, dy, r, G;  // G = Gdτ (uniform per instance)
    double invG;          // 1.0/Gdτ
    double ag, invag;     // @av(Gdτ) = (((G+G)+G)+G)*0.25 and 1.0/@av(Gdτ)
    double aR;            // @av_xi(dτ_Rho) = @av_yi(dτ_Rho) = (R+R)*0.5, R = dτ_Rho
};

__device__ __forceinline__ SweepP sweep_params(const BInst& I, int64_t iter_last) {
    SweepP P;
    P.nx = I.g.nx; P.ny = I.g.ny; P.px = I.g.px; P.py = I.g.py; P.ntx = I.ntx; P.tile0 = I.tile0;
    P.off = I.off;
    P.cap = I.iter_last < iter_last ? I.iter_last : iter_last;
    P.dx = I.n.dx; P.dy = I.n.dy; P.r = I.n.r; P.G = I.Gd;
    P.invG = 1.0 / P.G;
    P.ag = (((P.G + P.G) + P.G) + P.G) * 0.25;
    P.invag = 1.0 / P.ag;
    P.aR = (I.dR + I.dR) * 0.5;
    return P;
}

// compute_P! + compute_τ! of the sweep script (Stokes2D_param.jl:42-55) with its uniform
// iteration parameters (Musτ .= μs0, :190-192): Gdτ is one number G per instance, so
// @av(Gdτ) is formed from it in the reference's order and no Gdτ array is read. Every load
// is issued before the first store (the fields are distinct arrays), so a point costs one
// round trip to memory rather than one per store.
// The arithmetic of the sweep's compute_P! + compute_τ! at one point, on operand values
// (shared by the direct and the staged walks, so both give the same bits).
struct SweepA {
    double dv, pt, txx, tyy, txy;
};
__device__ __forceinline__ SweepA pt_tau_core(const SweepP& P, bool edge, double vx0, double vx1, double vy0, double vy1,
                                              double pt, double Mc, double sxx, double syy, double m11, double m01,
                                              double m10, double vxs, double vys, double sxy) {
    SweepA o;
    const double G = P.G;
    const double dvx = vx1 - vx0, dvy = vy1 - vy0;
    o.dv = dvx / P.dx + dvy / P.dy;
    // x/2.0 is written x*0.5: both are the correctly rounded x/2, the same bits for every x
    const double mu = 1.0 / (P.invG + 1.0 / Mc);  // @μ_veτ
    o.pt = pt - P.r * G * o.dv;
    o.txx = 2.0 * mu * (dvx / P.dx + (sxx / G) * 0.5);
    o.tyy = 2.0 * mu * (dvy / P.dy + (syy / G) * 0.5);
    o.txy = 0.0;
    if (edge) {
        const double am = (((m11 + m01) + m10) + Mc) * 0.25;
        const double mua = 1.0 / (P.invag + 1.0 / am);  // @μ_veτ_av
        const double d1 = vx0 - vxs;                      // @d_yi(Vx)
        const double d2 = vy0 - vys;                      // @d_xi(Vy)
        o.txy = 2.0 * mua * (0.5 * (d1 / P.dy + d2 / P.dx) + (sxy / P.ag) * 0.5);
    }
    return o;
}

__device__ __forceinline__ void pt_tau_sweep(const SweepF& f, const SweepP& P, int i, int j, bool store_divV) {
    if (i >= P.nx || j >= P.ny) return;
    const idx_t sx = 1, sy = P.px;
    const idx_t c = i + sy * j;
    const bool edge = (i >= 1 && j >= 1);
    const double vx0 = f.Vx[c], vx1 = f.Vx[c + sx], vy0 = f.Vy[c], vy1 = f.Vy[c + sy];
    const double pt = f.Pt[c], Mc = f.Mus[c], sxx = f.txx[c], syy = f.tyy[c];
    double m11 = 0.0, m01 = 0.0, m10 = 0.0, vxs = 0.0, vys = 0.0, sxy = 0.0;
    if (edge) {
        m11 = f.Mus[c - sx - sy];
        m01 = f.Mus[c - sy];
        m10 = f.Mus[c - sx];
        vxs = f.Vx[c - sy];
        vys = f.Vy[c - sx];
        sxy = f.txy[c];
    }
    const SweepA o = pt_tau_core(P, edge, vx0, vx1, vy0, vy1, pt, Mc, sxx, syy, m11, m01, m10, vxs, vys, sxy);
    if (store_divV) f.divV[c] = o.dv;
    f.Pt[c] = o.pt;
    f.txx[c] = o.txx;
    f.tyy[c] = o.tyy;
    if (edge) f.txy[c] = o.txy;
}

// Rx, Ry of compute_dV! (Stokes2D_param.jl:58-59), Ry with the buoyancy term -@av_yi(ρg)
__device__ __forceinline__ double res_x_core(const SweepP& P, double xx, double xx_m, double xy_p, double xy, double pt,
                                             double pt_m) {
    return ((xx - xx_m) / P.dx + (xy_p - xy) / P.dy) - (pt - pt_m) / P.dx;
}
__device__ __forceinline__ double res_y_core(const SweepP& P, double yy, double yy_m, double xy_p, double xy, double pt,
                                             double pt_m, double rg_m, double rg) {
    const double R = ((yy - yy_m) / P.dy + (xy_p - xy) / P.dx) - (pt - pt_m) / P.dy;
    return R - (rg_m + rg) * 0.5;
}
__device__ __forceinline__ double res_sweep_x(const SweepF& f, const SweepP& P, idx_t c, idx_t sy) {
    return res_x_core(P, f.txx[c], f.txx[c - 1], f.txy[c + sy], f.txy[c], f.Pt[c], f.Pt[c - 1]);
}
__device__ __forceinline__ double res_sweep_y(const SweepF& f, const SweepP& P, idx_t c, idx_t sy) {
    return res_y_core(P, f.tyy[c], f.tyy[c - sy], f.txy[c + 1], f.txy[c], f.Pt[c], f.Pt[c - sy], f.rhog[c - sy],
                      f.rhog[c]);
}

// compute_dV! + compute_V! + bc_y!(Vx), bc_x!(Vy) of the sweep script (Stokes2D_param.jl:57-81,
// 198-200) with the uniform dτ_Rho R: @av_xi(dτ_Rho) = (R + R)*0.5. Loads first, as above.
// The update and the free-slip copies of one face point, from its operands (shared by the
// direct and the staged walks).
__device__ __forceinline__ void v_bc_apply(const SweepF& f, const SweepP& P, int i, int j, idx_t c, bool fx, bool ux,
                                           bool fy, bool uy, double vx, double vy, double Rx, double Ry) {
    const idx_t sx = 1, sy = P.px;
    const double aR = P.aR;
    if (fx) {
        if (ux) {
            vx = vx + Rx * aR;
            f.Vx[c] = vx;
        }
        if (j == 1) f.Vx[c - sy] = vx;
        if (j == P.ny - 2) f.Vx[c + sy] = vx;
    }
    if (fy) {
        if (uy) {
            vy = vy + Ry * aR;
            f.Vy[c] = vy;
        }
        if (i == 1) f.Vy[c - sx] = vy;
        if (i == P.nx - 2) f.Vy[c + sx] = vy;
    }
}

__device__ __forceinline__ void v_bc_sweep(const SweepF& f, const SweepP& P, int i, int j) {
    const int nx = P.nx, ny = P.ny;
    if (i > nx || j > ny) return;
    const idx_t sy = P.px;
    const idx_t c = i + sy * j;
    const bool fx = (j >= 1 && j <= ny - 2), ux = fx && (i >= 1 && i <= nx - 1);
    const bool fy = (i >= 1 && i <= nx - 2), uy = fy && (j >= 1 && j <= ny - 1);
    double vx = 0.0, vy = 0.0, Rx = 0.0, Ry = 0.0;
    if (fx) vx = f.Vx[c];
    if (fy) vy = f.Vy[c];
    if (ux) Rx = res_sweep_x(f, P, c, sy);
    if (uy) Ry = res_sweep_y(f, P, c, sy);
    v_bc_apply(f, P, i, j, c, fx, ux, fy, uy, vx, vy, Rx, Ry);
}

// Active list of the sweep (built by block 0): act[0] = K instances still iterating,
// act[1] = T their tiles, act[2 .. 2+K] = first virtual tile of each (act[2+K] = T),
// act[3+n .. 3+n+K) = their instance ids, in instance order.
__device__ void build_active_list(const BInst* __restrict__ inst, int ninst, const BState& st, int64_t iter,
                                  int64_t iter_last, int* s_cnt) {
    const int nt = blockDim.x * blockDim.y, tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int per = (ninst + nt - 1) / nt, b0 = tid * per, b1 = min(ninst, b0 + per);
    int k = 0, t = 0;
    auto active = [&](int b) {
        const int64_t cap = inst[b].iter_last < iter_last ? inst[b].iter_last : iter_last;
        return *(volatile const int*)&st.converged[b] == 0 && iter <= cap;
    };
    for (int b = b0; b < b1; ++b)
        if (active(b)) { ++k; t += inst[b].ntx * inst[b].nty; }
    s_cnt[2 * tid] = k;
    s_cnt[2 * tid + 1] = t;
    __syncthreads();
    if (tid == 0) {  // exclusive scan over the threads' chunks (instance order)
        int K = 0, T = 0;
        for (int u = 0; u < nt; ++u) {
            const int dk = s_cnt[2 * u], dt = s_cnt[2 * u + 1];
            s_cnt[2 * u] = K;
            s_cnt[2 * u + 1] = T;
            K += dk;
            T += dt;
        }
        st.act[0] = K;
        st.act[1] = T;
        st.act[2 + K] = T;
    }
    __syncthreads();
    k = s_cnt[2 * tid];
    t = s_cnt[2 * tid + 1];
    for (int b = b0; b < b1; ++b)
        if (active(b)) {
            st.act[2 + k] = t;
            st.act[3 + ninst + k] = b;
            ++k;
            t += inst[b].ntx * inst[b].nty;
        }
    __syncthreads();
}

// All instances of a sweep iterate in lockstep inside one cooperative launch. Each block
// walks a contiguous chunk of the active instances' TX x TY tiles (the active list is
// rebuilt after every check, when instances converge). Per PT iteration: compute_P! +
// compute_τ!, grid barrier, compute_dV! + compute_V! + bc_y!/bc_x!, grid barrier
// (Stokes2D_param.jl:195-200). Every nout iterations each instance's check
// (Stokes2D_param.jl:203-210 with a single tolerance, norms scaled by ly) is reduced in a
// fixed order from per-tile partials, and an instance whose err <= eps (or NaN) is frozen
// -- its `while err > ε` loop ended. An instance also ends after its iteration iter_last
// (`iter <= iterMax`, with the launch-wide iter_last as a ceiling); until the next rebuild
// its tiles are skipped. nactive counts the instances still iterating; it changes only
// before a grid barrier, so every block reads the same value at the top of the loop and
// they all leave together.
constexpr int kListSmem = 1024;  // active lists up to this many instances are walked from shared memory
// Resident threads per SM the sweep kernel is compiled for (bounds its registers per thread).
#ifndef PTS_SWEEP_THREADS_PER_SM
#define PTS_SWEEP_THREADS_PER_SM 1024
#endif
// tiles ahead of the one being computed whose first lines are requested into L2
#ifndef PTS_SWEEP_PREFETCH
#define PTS_SWEEP_PREFETCH 1
#endif

template <int TX, int TY>
__global__ void __launch_bounds__(TX* TY, PTS_SWEEP_THREADS_PER_SM / (TX * TY)) k2_batch(const BInst* __restrict__ inst, int ntiles, int ninst, SweepF F,
                                                   BState st, int nout, int64_t iter_last, double eps) {
    (void)ntiles;
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    __shared__ int s_first[kListSmem + 1];
    __shared__ int s_id[kListSmem];
    __shared__ int s_cnt[2 * TX * TY];
    __shared__ int s_KT[2];
    const int* g_first = st.act + 2;
    const int* g_id = st.act + 3 + ninst;
    int K = 0, T = 0;
    bool in_smem = false;
    // the active list of this epoch into shared memory (when it fits)
    auto load_list = [&]() {
        if (tid == 0) {
            s_KT[0] = *(volatile int*)&st.act[0];
            s_KT[1] = *(volatile int*)&st.act[1];
        }
        __syncthreads();
        K = s_KT[0];
        T = s_KT[1];
        in_smem = K <= kListSmem;
        if (in_smem) {
            for (int u = tid; u <= K; u += TX * TY) s_first[u] = ((volatile const int*)g_first)[u];
            for (int u = tid; u < K; u += TX * TY) s_id[u] = ((volatile const int*)g_id)[u];
        }
        __syncthreads();
    };
    auto first_at = [&](int k) { return in_smem ? s_first[k] : ((volatile const int*)g_first)[k]; };
    auto id_at = [&](int k) { return in_smem ? s_id[k] : ((volatile const int*)g_id)[k]; };
    // body(P, b, t, i, j) for every point of this block's chunk of the active tiles; pre(P, i, j)
    // is called first with the point of the block's next tile when that tile belongs to the
    // same instance, so its cache lines can be requested while this tile computes
    auto walk = [&](auto&& body, auto&& pre) {
        const int chunk = (T + (int)gridDim.x - 1) / (int)gridDim.x;
        const int v0 = (int)blockIdx.x * chunk, v1 = min(T, v0 + chunk);
        if (v0 >= v1) return;
        int lo = 0, hi = K - 1;  // last k with first_at(k) <= v0
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (first_at(mid) <= v0) lo = mid;
            else hi = mid - 1;
        }
        int k = lo, b = id_at(k), f0 = first_at(k), f1 = first_at(k + 1);
        SweepP P = sweep_params(inst[b], iter_last);
        // tile coordinates (qx, qy) of q = v - f0, advanced by one tile per step: integer
        // divisions only where the walk enters an instance or a prefetch wraps a tile row
        int qx = (v0 - f0) % P.ntx, qy = (v0 - f0) / P.ntx;
        for (int v = v0; v < v1; ++v) {
            if (v >= f1) {
                do { ++k; f0 = f1; f1 = first_at(k + 1); } while (v >= f1);
                b = id_at(k);
                P = sweep_params(inst[b], iter_last);
                qx = (v - f0) % P.ntx;
                qy = (v - f0) / P.ntx;
            }
            const int q = v - f0;
#pragma unroll
            for (int d = 1; d <= PTS_SWEEP_PREFETCH; ++d)
                if (v + d < v1 && v + d < f1 && (d == PTS_SWEEP_PREFETCH || v == v0)) {
                    int nx_ = qx + d, ny_ = qy;
                    if (nx_ >= P.ntx) {
                        nx_ = (q + d) % P.ntx;
                        ny_ = (q + d) / P.ntx;
                    }
                    pre(P, nx_ * TX + tx, ny_ * TY + ty);
                }
            body(P, b, P.tile0 + q, qx * TX + tx, qy * TY + ty);
            if (++qx == P.ntx) {
                qx = 0;
                ++qy;
            }
        }
    };
    // L2 prefetches of the lines a point's stencil reads first, at an address clamped into the
    // instance's own padded arrays (always a valid address)
    auto pf = [](const double* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); };
    auto preA = [&](const SweepP& P, int i, int j) {
        const SweepF f = sweep_at(F, P.off);
        const int jc = min(j, P.ny);
        const idx_t c = min(i, P.nx) + P.px * jc;
        pf(f.Vx + c); pf(f.Vy + c); pf(f.Pt + c); pf(f.Mus + c);
        pf(f.txx + c); pf(f.tyy + c); pf(f.txy + c);
        if (jc < P.ny) pf(f.Vy + c + P.px);
    };
    auto preB = [&](const SweepP& P, int i, int j) {
        const SweepF f = sweep_at(F, P.off);
        const int jc = min(j, P.ny);
        const idx_t c = min(i, P.nx) + P.px * jc;
        pf(f.Vx + c); pf(f.Vy + c); pf(f.Pt + c); pf(f.rhog + c);
        pf(f.txx + c); pf(f.tyy + c); pf(f.txy + c);
        if (jc < P.ny) pf(f.txy + c + P.px);
    };
    auto no_pre = [](const SweepP&, int, int) {};
    if (blockIdx.x == 0) build_active_list(inst, ninst, st, 0, iter_last, s_cnt);
    grid.sync();
    load_list();
    int64_t iter = 0;
    for (;;) {
        if (*(volatile int*)st.nactive == 0 || iter > iter_last) break;
        const bool chk = ((iter + 1) % nout == 0);
        walk([&](const SweepP& P, int, int, int i, int j) {
            if (iter <= P.cap) pt_tau_sweep(sweep_at(F, P.off), P, i, j, chk);
        }, preA);
        grid.sync();
        walk([&](const SweepP& P, int, int, int i, int j) {
            if (iter <= P.cap) v_bc_sweep(sweep_at(F, P.off), P, i, j);
        }, preB);
        // an instance doing its last allowed iteration leaves the active count here
        for (int b = blockIdx.x * TX * TY + tid; b < ninst; b += gridDim.x * TX * TY) {
            const int64_t cap = inst[b].iter_last < iter_last ? inst[b].iter_last : iter_last;
            if (!st.converged[b] && iter == cap) atomicSub(st.nactive, 1);
        }
        grid.sync();
        ++iter;
        if (!chk) continue;
        // per-tile partials of the check (instances that did this iteration)
        walk([&](const SweepP& P, int, int t, int i, int j) {
            if (iter > P.cap + 1) return;
            const int nx = P.nx, ny = P.ny;
            const SweepF f = sweep_at(F, P.off);
            Acc a;
            acc_init(a);
            const idx_t sy = P.px;
            const idx_t c = i + sy * j;
            if (i < nx && j <= ny) {
                const double vy = f.Vy[c];
                a.vmin = vy;
                a.vmax = vy;
            }
            if (i < nx && j < ny) {
                a.pmin = a.pmax = f.Pt[c];
                const double dv = f.divV[c];
                a.s[3] = dv * dv;
            }
            if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) {
                const double R = res_sweep_x(f, P, c, sy);
                f.Rx[c] = R;
                a.s[0] = R * R;
            }
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) {
                const double R = res_sweep_y(f, P, c, sy);
                f.Ry[c] = R;
                a.s[1] = R * R;
            }
            acc_block_store_to(a, st.partials + (int64_t)t * kCheckSlots);
        }, no_pre);
        grid.sync();
        // per-instance finalisation: one block per instance, fixed-order reduction
        __shared__ double red[TX * TY][kCheckSlots];
        for (int b = blockIdx.x; b < ninst; b += gridDim.x) {
            const BInst& I = inst[b];
            const int64_t cap = I.iter_last < iter_last ? I.iter_last : iter_last;
            if (st.converged[b] || iter > cap + 1) continue;
            const int nt = I.ntx * I.nty;
            double r[kCheckSlots] = {0.0, 0.0, 0.0, 0.0, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
            for (int u = tid; u < nt; u += TX * TY) {
                const double* p = st.partials + (int64_t)(I.tile0 + u) * kCheckSlots;
                for (int w = 0; w < 4; ++w) r[w] += p[w];
                r[4] = fmin(r[4], p[4]); r[5] = fmax(r[5], p[5]);
                r[6] = fmin(r[6], p[6]); r[7] = fmax(r[7], p[7]);
            }
            for (int w = 0; w < kCheckSlots; ++w) red[tid][w] = r[w];
            __syncthreads();
            for (int s = (TX * TY) / 2; s > 0; s >>= 1) {
                if (tid < s) {
                    for (int w = 0; w < 4; ++w) red[tid][w] += red[tid + s][w];
                    red[tid][4] = fmin(red[tid][4], red[tid + s][4]); red[tid][5] = fmax(red[tid][5], red[tid + s][5]);
                    red[tid][6] = fmin(red[tid][6], red[tid + s][6]); red[tid][7] = fmax(red[tid][7], red[tid + s][7]);
                }
                __syncthreads();
            }
            if (tid == 0) {
                const double dP = red[0][7] - red[0][6], dV = red[0][5] - red[0][4];
                const double nRx = sqrt(red[0][0]) / dP * I.ly / sqrt(I.lenRx);
                const double nRy = sqrt(red[0][1]) / dP * I.ly / sqrt(I.lenRy);
                const double nDv = sqrt(red[0][3]) / dV * I.ly / sqrt(I.lenDiv);
                const bool bad = isnan(nRx) || isnan(nRy) || isnan(nDv);
                const double err = bad ? NAN : fmax(fmax(nRx, nRy), nDv);
                st.err[b] = err;
                st.iters[b] = iter;
                if (bad) atomicExch(st.nan_flag, 1);
                if (!(err > eps)) {
                    st.converged[b] = bad ? 2 : 1;                 // 2: frozen on NaN
                    if (iter <= cap) atomicSub(st.nactive, 1);  // else already left at its cap
                }
            }
            __syncthreads();
        }
        grid.sync();
        if (blockIdx.x == 0) build_active_list(inst, ninst, st, iter, iter_last, s_cnt);
        grid.sync();
        load_list();
    }
    // instances whose loop ended on iterMax: iterations done = iter_last + 1
    for (int b = blockIdx.x * TX * TY + tid; b < ninst; b += gridDim.x * TX * TY) {
        const int64_t cap = inst[b].iter_last < iter_last ? inst[b].iter_last : iter_last;
        if (!st.converged[b]) st.iters[b] = iter < cap + 1 ? iter : cap + 1;
    }
}

// ------------------------------------------------------------------ batched 2D visco-elastic sweep
//
// scripts/Stokes2D_ve_param.jl (the aspect-ratio study) for many instances at once, as its
// driver scripts/runme_Stokes2D_aspect_ratio.jl sweeps FACT x NSUB x RESOL with one Julia
// process per instance. Each instance keeps the script's own numerics: the role kernels
// compute_P!, compute_τ!, compute_dV! + compute_V! + bc (the per-point functions of the 2D
// visco-elastic contexts, pt_tau_2d<VE2D> and v_bc_2d<VE2D>, so every instance computes
// the bits a context would), local-max iteration parameters, a check every nout of its own
// iterations with norm_Rx scaled by lx and norm_Ry, norm_∇V by ly (:170-177), and nt
// physical steps, each starting with assign_τ! and ending when err <= ε or after iterMax
// (:152-186).

// Mus of an instance (:133-141): μs0, and μsi where
//   ((ix-1)*dx + 0.5*dx - 0.5*ly - (isub-1)*ly)^2 + ((iy-1)*dy + 0.5*dy - 0.5*ly)^2 < 1
// for some isub in 1..nsub, in the script's operation order.
__global__ void k2_init_ve_param(Geom g, Fields64 f, Num n, int nsub, double mus0, double musi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const double Y = ((double)j * n.dy + 0.5 * n.dy) - 0.5 * n.ly;
    double mu = mus0;
    for (int s = 1; s <= nsub; ++s) {
        const double X = (((double)i * n.dx + 0.5 * n.dx) - 0.5 * n.ly) - (double)(s - 1) * n.ly;
        if (X * X + Y * Y < 1.0) mu = musi;
    }
    f.Mus[gidx32(g, i, j, 0)] = mu;
}

// The fields of one instance: every arena advanced to the instance's first element.
__device__ __forceinline__ Fields64 ve_at(const Fields64& F, int64_t off) {
    Fields64 f = F;
    f.Pt = F.Pt + off; f.Vx = F.Vx + off; f.Vy = F.Vy + off;
    f.txx = F.txx + off; f.tyy = F.tyy + off; f.txy = F.txy + off;
    f.txx_o = F.txx_o + off; f.tyy_o = F.tyy_o + off; f.txy_o = F.txy_o + off;
    f.Mus = F.Mus + off; f.Gdt = F.Gdt + off; f.dtRho = F.dtRho + off;
    f.divV = F.divV + off; f.Rx = F.Rx + off; f.Ry = F.Ry + off;
    return f;
}

// Block 0: the list of instances still iterating (as build_active_list) and the next global
// iteration count at which one of them checks (a multiple of its nout within its step) or
// ends its step (iterMax + 1 iterations); clears the pending assign_τ! flags.
__device__ void build_list_ve(const BInst* __restrict__ inst, int ninst, const BState& st, const BStateVE& sv,
                              int64_t iter, int* s_cnt, long long* s_min) {
    const int nt = blockDim.x * blockDim.y, tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int per = (ninst + nt - 1) / nt, b0 = tid * per, b1 = min(ninst, b0 + per);
    int k = 0, t = 0;
    long long ev = LLONG_MAX;
    for (int b = b0; b < b1; ++b) {
        sv.assign[b] = 0;
        if (*(volatile const int*)&st.converged[b] != 0) continue;
        ++k;
        t += inst[b].ntx * inst[b].nty;
        const int64_t s0 = *(volatile const int64_t*)&sv.start[b], it = iter - s0, nout = inst[b].nout;
        const int64_t nc = s0 + (it / nout + 1) * nout, ne = s0 + inst[b].iter_last + 1;
        ev = min(ev, (long long)(nc < ne ? nc : ne));
    }
    s_cnt[2 * tid] = k;
    s_cnt[2 * tid + 1] = t;
    for (int o = 16; o > 0; o >>= 1) ev = min(ev, __shfl_down_sync(kFull, ev, o));
    if ((tid & 31) == 0) s_min[tid >> 5] = ev;
    __syncthreads();
    if (tid == 0) {
        int K = 0, T = 0;
        for (int u = 0; u < nt; ++u) {
            const int dk = s_cnt[2 * u], dt = s_cnt[2 * u + 1];
            s_cnt[2 * u] = K;
            s_cnt[2 * u + 1] = T;
            K += dk;
            T += dt;
        }
        st.act[0] = K;
        st.act[1] = T;
        st.act[2 + K] = T;
        long long m = LLONG_MAX;
        for (int w = 0; w < (nt + 31) / 32; ++w) m = min(m, s_min[w]);
        *(volatile long long*)sv.next_event = m;
    }
    __syncthreads();
    k = s_cnt[2 * tid];
    t = s_cnt[2 * tid + 1];
    for (int b = b0; b < b1; ++b)
        if (*(volatile const int*)&st.converged[b] == 0) {
            st.act[2 + k] = t;
            st.act[3 + ninst + k] = b;
            ++k;
            t += inst[b].ntx * inst[b].nty;
        }
    __syncthreads();
}

// All instances in one cooperative launch, in lockstep on a global iteration count. Per PT
// iteration: compute_P! + compute_τ!, grid barrier, compute_dV! + compute_V! + bc, grid
// barrier. At an event (some instance has done a multiple of its nout iterations in its
// current step, or iterMax + 1 of them): the check of those instances from per-tile
// partials, per-instance step bookkeeping, assign_τ! (τ_o ← τ) for the instances that begin
// a new step, a rebuilt list of the instances still iterating and the next event. ∇V is
// stored on event iterations only: the check is its only reader, and an instance's last
// iteration is always an event.
template <int TX, int TY>
__global__ void __launch_bounds__(TX* TY, PTS_SWEEP_THREADS_PER_SM / (TX * TY))
    k2_batch_ve(const BInst* __restrict__ inst, int ninst, Fields64 F, BState st, BStateVE sv, int64_t iter_cap,
                double eps) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    constexpr int NT = TX * TY;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    __shared__ int s_first[kListSmem + 1];
    __shared__ int s_id[kListSmem];
    __shared__ int s_cnt[2 * NT];
    __shared__ int s_KT[2];
    __shared__ long long s_min[NT / 32];
    __shared__ double red[NT][kCheckSlots];
    const int* g_first = st.act + 2;
    const int* g_id = st.act + 3 + ninst;
    int K = 0, T = 0;
    bool in_smem = false;
    auto load_list = [&]() {
        if (tid == 0) {
            s_KT[0] = *(volatile int*)&st.act[0];
            s_KT[1] = *(volatile int*)&st.act[1];
        }
        __syncthreads();
        K = s_KT[0];
        T = s_KT[1];
        in_smem = K <= kListSmem;
        if (in_smem) {
            for (int u = tid; u <= K; u += NT) s_first[u] = ((volatile const int*)g_first)[u];
            for (int u = tid; u < K; u += NT) s_id[u] = ((volatile const int*)g_id)[u];
        }
        __syncthreads();
    };
    auto first_at = [&](int k) { return in_smem ? s_first[k] : ((volatile const int*)g_first)[k]; };
    auto id_at = [&](int k) { return in_smem ? s_id[k] : ((volatile const int*)g_id)[k]; };
    // enter(b) when the walk enters instance b, then body(b, t, i, j) for every point of this
    // block's chunk of the active tiles (t: the tile's index in the flattened tile list)
    auto walk = [&](auto&& enter, auto&& body) {
        const int chunk = (T + (int)gridDim.x - 1) / (int)gridDim.x;
        const int v0 = (int)blockIdx.x * chunk, v1 = min(T, v0 + chunk);
        if (v0 >= v1) return;
        int lo = 0, hi = K - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (first_at(mid) <= v0) lo = mid;
            else hi = mid - 1;
        }
        int k = lo, b = id_at(k), f0 = first_at(k), f1 = first_at(k + 1);
        int ntx = inst[b].ntx, tile0 = inst[b].tile0;
        int qx = (v0 - f0) % ntx, qy = (v0 - f0) / ntx;
        enter(b);
        for (int v = v0; v < v1; ++v) {
            if (v >= f1) {
                do { ++k; f0 = f1; f1 = first_at(k + 1); } while (v >= f1);
                b = id_at(k);
                ntx = inst[b].ntx;
                tile0 = inst[b].tile0;
                qx = (v - f0) % ntx;
                qy = (v - f0) / ntx;
                enter(b);
            }
            body(b, tile0 + (v - f0), qx * TX + tx, qy * TY + ty);
            if (++qx == ntx) {
                qx = 0;
                ++qy;
            }
        }
    };
    // what the stencils need of the instance the walk is in
    Geom gI{};
    Num nI{};
    int64_t offI = 0;
    bool chkI = false, asgI = false;  // the instance checks at this event / begins a new step
    int64_t iter = 0;                 // PT iterations done, counted globally
    auto enter = [&](int b) {
        const BInst& I = inst[b];
        gI = I.g;
        nI.dx = I.n.dx; nI.dy = I.n.dy; nI._dx = I.n._dx; nI._dy = I.n._dy;
        nI.r = I.n.r; nI.gdt = I.n.gdt;
        offI = I.off;
        chkI = ((iter - *(volatile const int64_t*)&sv.start[b]) % I.nout) == 0;
        asgI = *(volatile const int*)&sv.assign[b] != 0;
    };

    if (blockIdx.x == 0) {
        for (int b = tid; b < ninst; b += NT) st.err[b] = 2.0 * eps;  // err = 2ε of every step
        __syncthreads();
        build_list_ve(inst, ninst, st, sv, 0, s_cnt, s_min);
    }
    grid.sync();
    load_list();
    for (;;) {
        if (*(volatile int*)st.nactive == 0 || iter >= iter_cap) break;
        const int64_t ev = *(volatile long long*)sv.next_event;
        const int sdv = (iter + 1 == ev) ? 1 : 0;
        walk(enter, [&](int, int, int i, int j) {
            pt_tau_2d<VE2D>(gI, ve_at(F, offI), nI, i, j, ROLE_P | ROLE_TAU, sdv);
        });
        grid.sync();
        walk(enter, [&](int, int, int i, int j) { v_bc_2d<VE2D>(gI, ve_at(F, offI), nI, i, j, 1); });
        grid.sync();
        ++iter;
        if (iter != ev) continue;
        // per-tile partials of the check (compute_Res! + the reductions of :170-177) of the
        // instances with a multiple of nout iterations in their current step
        walk(enter, [&](int, int t, int i, int j) {
            if (!chkI) return;  // uniform over the block (one tile)
            const int nx = gI.nx, ny = gI.ny;
            const Fields64 f = ve_at(F, offI);
            Acc a;
            acc_init(a);
            if (i <= nx && j < ny) {
                const idx_t sy = gI.px, c = i + sy * j;
                const double vx = f.Vx[c];
                a.vmin = vx;
                a.vmax = vx;
                if (i < nx) {
                    a.pmin = a.pmax = f.Pt[c];
                    const double dv = f.divV[c];
                    a.s[3] = dv * dv;
                }
                if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) {
                    const double R = res2_x<false>(f, nI, c, 1, sy);
                    f.Rx[c] = R;
                    a.s[0] = R * R;
                }
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) {
                    const double R = res2_y<false>(f, nI, c, 1, sy);
                    f.Ry[c] = R;
                    a.s[1] = R * R;
                }
            }
            acc_block_store_to(a, st.partials + (int64_t)t * kCheckSlots);
        });
        grid.sync();
        // per instance (one block each): norms, then the step's end (err <= ε, or iterMax + 1
        // iterations done) with the next step's start or the instance's end
        for (int b = blockIdx.x; b < ninst; b += gridDim.x) {
            if (st.converged[b] != 0) continue;
            const BInst& I = inst[b];
            const int64_t it = iter - sv.start[b];
            const bool chk = (it % I.nout) == 0, endmax = it == I.iter_last + 1;
            if (!chk && !endmax) continue;
            if (chk) {
                const int nt = I.ntx * I.nty;
                double r[kCheckSlots] = {0.0, 0.0, 0.0, 0.0, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
                for (int u = tid; u < nt; u += NT) {
                    const double* p = st.partials + (int64_t)(I.tile0 + u) * kCheckSlots;
                    for (int w = 0; w < 4; ++w) r[w] += p[w];
                    r[4] = fmin(r[4], p[4]); r[5] = fmax(r[5], p[5]);
                    r[6] = fmin(r[6], p[6]); r[7] = fmax(r[7], p[7]);
                }
                for (int w = 0; w < kCheckSlots; ++w) red[tid][w] = r[w];
                __syncthreads();
                for (int s = NT / 2; s > 0; s >>= 1) {
                    if (tid < s) {
                        for (int w = 0; w < 4; ++w) red[tid][w] += red[tid + s][w];
                        red[tid][4] = fmin(red[tid][4], red[tid + s][4]); red[tid][5] = fmax(red[tid][5], red[tid + s][5]);
                        red[tid][6] = fmin(red[tid][6], red[tid + s][6]); red[tid][7] = fmax(red[tid][7], red[tid + s][7]);
                    }
                    __syncthreads();
                }
            }
            if (tid == 0) {
                double err = st.err[b];
                if (chk) {
                    const double dP = red[0][7] - red[0][6], dV = red[0][5] - red[0][4];
                    const double nRx = sqrt(red[0][0]) / dP * I.lx / sqrt(I.lenRx);
                    const double nRy = sqrt(red[0][1]) / dP * I.ly / sqrt(I.lenRy);
                    const double nDv = sqrt(red[0][3]) / dV * I.ly / sqrt(I.lenDiv);
                    const bool bad = isnan(nRx) || isnan(nRy) || isnan(nDv);
                    err = bad ? NAN : fmax(fmax(nRx, nRy), fmax(0.0, nDv));
                    st.err[b] = err;
                }
                if (isnan(err)) {  // the script stops with error("NaN"): this instance freezes
                    st.converged[b] = 2;
                    atomicExch(st.nan_flag, 1);
                    atomicSub(st.nactive, 1);
                } else if (endmax || !(err > eps)) {
                    const int s = sv.steps[b];
                    if (s < kBatchMaxSteps) sv.step_iters[(int64_t)b * kBatchMaxSteps + s] = it;
                    st.iters[b] += it;  // ittot += iter
                    sv.steps[b] = s + 1;
                    if (s + 1 >= I.nt) {
                        st.converged[b] = !(err > eps) ? 1 : 3;
                        atomicSub(st.nactive, 1);
                    } else {  // next step: err = 2ε; iter = 0; assign_τ!
                        st.err[b] = 2.0 * eps;
                        sv.start[b] = iter;
                        sv.assign[b] = 1;
                    }
                }
            }
            __syncthreads();
        }
        grid.sync();
        // assign_τ! (τ_o ← τ) of the instances that begin a new step
        walk(enter, [&](int, int, int i, int j) {
            if (!asgI || i > gI.nx || j > gI.ny) return;
            const Fields64 f = ve_at(F, offI);
            const idx_t c = i + (idx_t)gI.px * j;
            f.txx_o[c] = f.txx[c];
            f.tyy_o[c] = f.tyy[c];
            f.txy_o[c] = f.txy[c];
        });
        grid.sync();
        if (blockIdx.x == 0) build_list_ve(inst, ninst, st, sv, iter, s_cnt, s_min);
        grid.sync();
        load_list();
    }
}

// ------------------------------------------------------------------ mixed precision: FP64 outer step

// X += δ for the ten iterated fields, then the corrections are cleared (elementwise over
// the padded arrays). The sweeps carry the stress corrections as u = δτ - w (w in the aτ
// arrays, see k3_sources), so δτ = u + w.
__global__ void k_fold(int64_t n, Fields64 f, Mixed32 m) {
    double* X[10] = {f.Pt, f.Vx, f.Vy, f.Vz, f.txx, f.tyy, f.tzz, f.txy, f.txz, f.tyz};
    float* D[10] = {m.dPt, m.dVx, m.dVy, m.dVz, m.dtxx, m.dtyy, m.dtzz, m.dtxy, m.dtxz, m.dtyz};
    const float* W[6] = {m.atxx, m.atyy, m.atzz, m.atxy, m.atxz, m.atyz};
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            X[q][e] = X[q][e] + (double)D[q][e];
            D[q][e] = 0.0f;
        }
#pragma unroll
        for (int q = 4; q < 10; ++q) {
            X[q][e] = X[q][e] + ((double)D[q][e] + (double)W[q - 4][e]);
            D[q][e] = 0.0f;
        }
    }
}

// Residual sources of the FP64 iterate for the FP32 sweeps, and the convergence check of
// that iterate (compute_Res! + norms, Stokes3D_ve_perf.jl:90-96,210-218) in one pass:
//   aP = ∇·V (the check's ∇V), R (the check's Rx, Ry, Rz, FP64, for k3_srcw),
//   w = aτ/(D - 1) into the aτ arrays, where aτ = τ_o*Gr + 2Gdτ*ε̇(V) - τ*(D - 1) is the
//   constitutive residual (zero when τ satisfies its PT update) and D = 1 + Gdτ/Mus + Gr.
// With the stress corrections carried as u = δτ - w the sweeps' stress update
// δτ' = (δτ + aτ + 2Gdτ*ε̇(δV))/D becomes u' = (u + 2Gdτ*ε̇(δV))/D exactly: no stress
// source is read by the sweeps, and w joins the momentum source instead (k3_srcw).
template <bool EL>
__global__ void __launch_bounds__(256) k3_sources(Geom g, Fields64 f, Mixed32 m, Num n, double* partials) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    Acc a;
    acc_init(a);
    if (i <= nx && j < ny) {
        for (int k = blockIdx.z; k < nz; k += gridDim.z) {
            const idx_t c = gidx32(g, i, j, k);
            const double vx = f.Vx[c];
            a.vmin = fmin(a.vmin, vx);
            a.vmax = fmax(a.vmax, vx);
            if (i < nx) {
                const double p = f.Pt[c];
                a.pmin = fmin(a.pmin, p);
                a.pmax = fmax(a.pmax, p);
                const double dvx = f.Vx[c + sx] - vx, dvy = f.Vy[c + sy] - f.Vy[c], dvz = f.Vz[c + sz] - f.Vz[c];
                const double dv = (n._dx * dvx + n._dy * dvy) + n._dz * dvz;
                f.divV[c] = dv;
                m.aP[c] = (float)dv;
                a.s[3] += dv * dv;
                const double Gc = f.Gdt[c], Mc = f.Mus[c];
                const double Gr = EL ? gr_of(Gc, n.gdt) : 0.0;
                const double Dm = Gc / Mc + Gr;  // D - 1
                auto a_n = [&](const double* t, const double* to, double e) {
                    return (((EL ? to[c] * Gr : 0.0) + (2.0 * Gc) * e) - t[c] * Dm) / Dm;
                };
                if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) m.atxx[c] = (float)a_n(f.txx, f.txx_o, n._dx * dvx);
                if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) m.atyy[c] = (float)a_n(f.tyy, f.tyy_o, n._dy * dvy);
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) m.atzz[c] = (float)a_n(f.tzz, f.tzz_o, n._dz * dvz);
            }
            if (i < nx) {
                auto a_s = [&](const double* t, const double* to, idx_t o1, idx_t o2, double s) {
                    const double ag = (((f.Gdt[c - o1 - o2] + f.Gdt[c - o2]) + f.Gdt[c - o1]) + f.Gdt[c]) * 0.25;
                    const double am = (((f.Mus[c - o1 - o2] + f.Mus[c - o2]) + f.Mus[c - o1]) + f.Mus[c]) * 0.25;
                    const double Gr = EL ? gr_of(ag, n.gdt) : 0.0;
                    const double dm = ag / am + Gr;
                    return (((EL ? to[c] * Gr : 0.0) + (2.0 * ag) * (0.5 * s)) - t[c] * dm) / dm;
                };
                if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2)
                    m.atxy[c] = (float)a_s(f.txy, f.txy_o, sx, sy,
                                           n._dy * (f.Vx[c] - f.Vx[c - sy]) + n._dx * (f.Vy[c] - f.Vy[c - sx]));
                if (i >= 1 && j >= 1 && j <= ny - 2 && k >= 1)
                    m.atxz[c] = (float)a_s(f.txz, f.txz_o, sx, sz,
                                           n._dz * (f.Vx[c] - f.Vx[c - sz]) + n._dx * (f.Vz[c] - f.Vz[c - sx]));
                if (i >= 1 && i <= nx - 2 && j >= 1 && k >= 1)
                    m.atyz[c] = (float)a_s(f.tyz, f.tyz_o, sy, sz,
                                           n._dz * (f.Vy[c] - f.Vy[c - sz]) + n._dy * (f.Vz[c] - f.Vz[c - sy]));
            }
            if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
                const double R = res3_x<true>(f, n, c, sx, sy, sz);
                f.Rx[c] = R;
                a.s[0] += R * R;
            }
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2) {
                const double R = res3_y<true>(f, n, c, sx, sy, sz);
                f.Ry[c] = R;
                a.s[1] += R * R;
            }
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1) {
                const double R = res3_z<true>(f, n, c, sx, sy, sz);
                f.Rz[c] = R;
                a.s[2] += R * R;
            }
        }
    }
    acc_block_store(a, partials);
}

// Momentum sources and the sweeps' starting stress corrections, after k3_sources:
//   aV = R(τ, Pt) of the FP64 iterate + the stress part of R applied to w (FP64 sums of the
//   FP32 w, so the sweeps and the fold see the same w), and u = -w (δτ = 0).
// One thread per unified face point.
__global__ void __launch_bounds__(256) k3_srcw(Geom g, Fields64 f, Mixed32 m, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    auto W = [&](const float* w, idx_t o) -> double { return (double)w[o]; };
    if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
        m.aVx[c] = (float)(f.Rx[c] + ((n._dx * (W(m.atxx, c) - W(m.atxx, c - sx)) + n._dy * (W(m.atxy, c + sy) - W(m.atxy, c))) +
                                      n._dz * (W(m.atxz, c + sz) - W(m.atxz, c))));
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2)
        m.aVy[c] = (float)(f.Ry[c] + ((n._dy * (W(m.atyy, c) - W(m.atyy, c - sy)) + n._dx * (W(m.atxy, c + sx) - W(m.atxy, c))) +
                                      n._dz * (W(m.atyz, c + sz) - W(m.atyz, c))));
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1)
        m.aVz[c] = (float)(f.Rz[c] + ((n._dz * (W(m.atzz, c) - W(m.atzz, c - sz)) + n._dx * (W(m.atxz, c + sx) - W(m.atxz, c))) +
                                      n._dy * (W(m.atyz, c + sy) - W(m.atyz, c))));
    const float* W6[6] = {m.atxx, m.atyy, m.atzz, m.atxy, m.atxz, m.atyz};
    float* U6[6] = {m.dtxx, m.dtyy, m.dtzz, m.dtxy, m.dtxz, m.dtyz};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float u = -W6[q][c];
        U6[q][c] = u;
        if (m.u2[q]) m.u2[q][c] = u;  // the points the one-pass sweeps never update stay -w in both sets
    }
}

__global__ void k_coef32(int64_t n, const double* Gdt, const double* Mus, const double* dtRho, float2* GM32,
                         float* R32) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        GM32[e] = make_float2((float)Gdt[e], (float)Mus[e]);
        R32[e] = (float)dtRho[e];
    }
}

// ------------------------------------------------------------------ set-up kernels

// Initial conditions (Stokes3D_ve_perf.jl:164-172; Stokes3D_ve_multixpu.jl:174-178 builds
// the staggered coordinates through ImplicitGlobalGrid's x_g, which for one rank is
// (ix-1)*dx - 0.5*dx; Stokes2D.jl:106-114 for 2D). One thread per unified point.
template <bool D3, bool IGG>
__global__ void k_init_inclusion(Geom g, Fields64 f, Num n, double mus0, double musi, double radius2, double ebg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const double X = ((double)i * n.dx + 0.5 * n.dx) - 0.5 * n.lx;
    const double Y = ((double)j * n.dy + 0.5 * n.dy) - 0.5 * n.ly;
    if (i < nx && j < ny && k < (D3 ? nz : 1)) {
        double rad2 = X * X + Y * Y;
        if (D3) {
            const double Z = ((double)(k + n.zoff) * n.dz + 0.5 * n.dz) - 0.5 * n.lz;
            rad2 = rad2 + Z * Z;
        }
        f.Mus[c] = (rad2 < radius2) ? musi : mus0;
    }
    const double xv = IGG ? ((((double)i * n.dx + (-0.5 * n.dx)) + 0.5 * n.dx) - 0.5 * n.lx)
                          : ((double)i * n.dx - 0.5 * n.lx);
    if (j < ny && k < (D3 ? nz : 1)) f.Vx[c] = (-ebg) * xv;
    if (D3) {
        const double zv = IGG ? ((((double)(k + n.zoff) * n.dz + (-0.5 * n.dz)) + 0.5 * n.dz) - 0.5 * n.lz)
                              : ((double)(k + n.zoff) * n.dz - 0.5 * n.lz);
        if (i < nx && j < ny) f.Vz[c] = ebg * zv;
    } else {
        if (i < nx) f.Vy[c] = ebg * ((double)j * n.dy - 0.5 * n.ly);
    }
}

// create_inclusions! (Stokes2D_param.jl:83-99) for a list of circles (2D) or spheres (3D),
// each with its own squared radius and viscosity: at each cell centre
//   x = (ix-1)*dx + 0.5*dx - 0.5*lx   (y, z alike; inclusion centres in the same centred frame)
//   rad2 = (x - Xi)^2 + (y - Yi)^2 [+ (z - Zi)^2],  inside when rad2 < r2,
// Mus = the viscosity of the first inclusion the cell is inside, else mus0 (the reference's
// loop breaks at the first hit). Velocities get the pure-shear ICs of k_init_inclusion.
template <bool D3, bool IGG>
__global__ void k_init_inclusions(Geom g, Fields64 f, Num n, const pts_inclusion* __restrict__ inc, int count,
                                  double mus0, double ebg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    if (i < nx && j < ny && k < (D3 ? nz : 1)) {
        const double X = ((double)i * n.dx + 0.5 * n.dx) - 0.5 * n.lx;
        const double Y = ((double)j * n.dy + 0.5 * n.dy) - 0.5 * n.ly;
        const double Z = D3 ? ((double)(k + n.zoff) * n.dz + 0.5 * n.dz) - 0.5 * n.lz : 0.0;
        double mu = mus0;
        for (int q = 0; q < count; ++q) {
            const double ax = X - __ldg(&inc[q].x), ay = Y - __ldg(&inc[q].y);
            double rad2 = ax * ax + ay * ay;
            if (D3) {
                const double az = Z - __ldg(&inc[q].z);
                rad2 = rad2 + az * az;
            }
            if (rad2 < __ldg(&inc[q].r2)) {
                mu = __ldg(&inc[q].mus);
                break;
            }
        }
        f.Mus[c] = mu;
    }
    const double xv = IGG ? ((((double)i * n.dx + (-0.5 * n.dx)) + 0.5 * n.dx) - 0.5 * n.lx)
                          : ((double)i * n.dx - 0.5 * n.lx);
    if (j < ny && k < (D3 ? nz : 1)) f.Vx[c] = (-ebg) * xv;
    if (D3) {
        const double zv = IGG ? ((((double)(k + n.zoff) * n.dz + (-0.5 * n.dz)) + 0.5 * n.dz) - 0.5 * n.lz)
                              : ((double)(k + n.zoff) * n.dz - 0.5 * n.lz);
        if (i < nx && j < ny) f.Vz[c] = ebg * zv;
    } else {
        if (i < nx) f.Vy[c] = ebg * ((double)j * n.dy - 0.5 * n.ly);
    }
}

// ICs of one batched-sweep instance (Stokes2D_param.jl:176-181 with one centred inclusion;
// the box lx x ly of Stokes2D_ve_param.jl:99-102): the same operations as the oracle.
__global__ void k2_init_sweep(Geom g, Fields64 f, Num n, double musi, double radius2, double rhogi, double ebg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nx || j > g.ny) return;
    const idx_t c = gidx32(g, i, j, 0);
    if (i < g.nx && j < g.ny) {
        const double X = ((double)i * n.dx + 0.5 * n.dx) - 0.5 * n.lx;
        const double Y = ((double)j * n.dy + 0.5 * n.dy) - 0.5 * n.ly;
        const bool in = (X * X + Y * Y) < radius2;
        f.Mus[c] = in ? musi : 1.0;
        f.rhog[c] = in ? rhogi : 0.0;
    }
    if (j < g.ny) f.Vx[c] = (-ebg) * ((double)i * n.dx - 0.5 * n.lx);
    if (i < g.nx) f.Vy[c] = ebg * ((double)j * n.dy - 0.5 * n.ly);
}

// smooth! (Stokes3D_ve_perf.jl:24-27; 2D Stokes2D.jl:17-20) on the interior cells.
template <bool D3>
__global__ void k_smooth(Geom g, double* __restrict__ dst, const double* __restrict__ A, double coef) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i < 1 || j < 1 || i > g.nx - 2 || j > g.ny - 2) return;
    if (D3 && (k < 1 || k > g.nz - 2)) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sy = g.px, sz = (idx_t)g.pxy;
    const double a = A[c];
    const double d2x = (A[c + 1] - a) - (a - A[c - 1]);
    const double d2y = (A[c + sy] - a) - (a - A[c - sy]);
    double s = d2x + d2y;
    if (D3) s = s + ((A[c + sz] - a) - (a - A[c - sz]));
    dst[c] = a + coef * s;
}

// compute_maxloc! + bc_x!/bc_y!/bc_z! on Musτ (Stokes3D_ve_perf.jl:29-32,178-182): the
// boundary copies leave each boundary cell equal to the local max at its clamped index.
template <bool D3>
__global__ void k_maxloc(Geom g, double* __restrict__ must, const double* __restrict__ A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const int ci = min(max(i, 1), g.nx - 2), cj = min(max(j, 1), g.ny - 2);
    const int ck = D3 ? min(max(k, 1), g.nz - 2) : 0;
    const idx_t c = gidx32(g, ci, cj, ck);
    const idx_t sy = g.px, sz = (idx_t)g.pxy;
    double m = fmax(fmax(fmax(fmax(A[c - 1], A[c + 1]), A[c]), A[c - sy]), A[c + sy]);
    if (D3) m = fmax(fmax(m, A[c - sz]), A[c + sz]);
    must[gidx32(g, i, j, k)] = m;
}

// compute_iter_params! (Stokes3D_ve_perf.jl:34-39; viscous Stokes2D.jl:27-31).
template <bool EL>
__global__ void k_iter_params(Geom g, Fields64 f, Num n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const double mu_eff = EL ? 1.0 / (1.0 / f.Must[c] + 1.0 / n.gdt) : f.Must[c];
    const double dtr = n.Vpdt * n.max_l / n.Re / mu_eff;
    f.dtRho[c] = dtr;
    f.Gdt[c] = (n.Vpdt * n.Vpdt) / dtr / (n.r + 2.0);
}

inline dim3 blk() { return dim3(32, 8, 1); }
inline dim3 grid_cells(const Geom& g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }
inline dim3 grid_faces(const Geom& g, bool d3) {
    return dim3((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, d3 ? g.nz + 1 : 1);
}

}  // namespace

// ------------------------------------------------------------------ launchers

// Block of the 3D compute_Pt_τ! kernel: x-y tile with a short z-extent.
#ifndef PTS_PT_BX
#define PTS_PT_BX 32
#define PTS_PT_BY 8
#define PTS_PT_BZ 1
#endif
inline dim3 blk_pt() { return dim3(PTS_PT_BX, PTS_PT_BY, PTS_PT_BZ); }
inline dim3 grid_pt(const Geom& g) {
    return dim3((g.nx + PTS_PT_BX - 1) / PTS_PT_BX, (g.ny + PTS_PT_BY - 1) / PTS_PT_BY, (g.nz + PTS_PT_BZ - 1) / PTS_PT_BZ);
}

cudaError_t launch_Pt_tau(int v, const Geom& g, const Fields64& f, const Num& n, int roles, bool store_divV,
                          cudaStream_t s) {
    const int sd = store_divV ? 1 : 0;
    switch (v) {
        case VE3D: k3_Pt_tau<true, false><<<grid_pt(g), blk_pt(), 0, s>>>(g, f, n, roles, sd); break;
        case VE3D_PERF: k3_Pt_tau<true, true><<<grid_pt(g), blk_pt(), 0, s>>>(g, f, n, roles, sd); break;
        case V3D: k3_Pt_tau<false, true><<<grid_pt(g), blk_pt(), 0, s>>>(g, f, n, roles, sd); break;
        case V3D_DAMP: k3d_Pt_tau<<<grid_pt(g), blk_pt(), 0, s>>>(g, f, n, roles, sd); break;
        case V2D: k2_Pt_tau<V2D><<<grid_cells(g), blk(), 0, s>>>(g, f, n, roles, sd); break;
        case VE2D: k2_Pt_tau<VE2D><<<grid_cells(g), blk(), 0, s>>>(g, f, n, roles, sd); break;
        case VE2D_PERF: k2_Pt_tau<VE2D_PERF><<<grid_cells(g), blk(), 0, s>>>(g, f, n, roles, sd); break;
        case V2D_DAMP: k2d_Pt_tau<false><<<grid_cells(g), blk(), 0, s>>>(g, f, n, roles, sd); break;
        case VE2D_DAMP: k2d_Pt_tau<true><<<grid_cells(g), blk(), 0, s>>>(g, f, n, roles, sd); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_V_bc(int v, const Geom& g, const Fields64& f, const Num& n, bool update, cudaStream_t s) {
    const int u = update ? 1 : 0;
    switch (v) {
        case VE3D: k3_V_bc<false><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n, u); break;
        case V3D_DAMP: k3d_V_bc<<<grid_faces(g, true), blk(), 0, s>>>(g, f, n, u); break;
        case VE3D_PERF:
        case V3D:
            if (n.adjoint) {
                if (f.Fx) k3_V_bc<true, true, true><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n, u);
                else k3_V_bc<true, false, true><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n, u);
            } else if (f.Fx) {
                k3_V_bc<true, true><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n, u);
            } else {
                k3_V_bc<true><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n, u);
            }
            break;
        case V2D: k2_V_bc<V2D><<<grid_faces(g, false), blk(), 0, s>>>(g, f, n, u); break;
        case VE2D: k2_V_bc<VE2D><<<grid_faces(g, false), blk(), 0, s>>>(g, f, n, u); break;
        case VE2D_PERF: k2_V_bc<VE2D_PERF><<<grid_faces(g, false), blk(), 0, s>>>(g, f, n, u); break;
        case V2D_DAMP:
        case VE2D_DAMP: k2d_V_bc<<<grid_faces(g, false), blk(), 0, s>>>(g, f, n, u); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_V_bc_planes(int v, const Geom& g, const Fields64& f, const Num& n, int k0, int k1,
                               cudaStream_t s) {
    if (k0 < 0 || k1 > g.nz + 1 || k0 > k1) return cudaErrorInvalidValue;
    if (k1 == k0) return cudaSuccess;
    dim3 gr = grid_faces(g, true);
    gr.z = (unsigned)(k1 - k0);
    switch (v) {
        case VE3D: k3_V_bc_planes<false><<<gr, blk(), 0, s>>>(g, f, n, k0); break;
        case VE3D_PERF:
        case V3D: k3_V_bc_planes<true><<<gr, blk(), 0, s>>>(g, f, n, k0); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dV(int v, const Geom& g, const Fields64& f, const Num& n, cudaStream_t s) {
    switch (v) {
        case VE3D: k3_dV<false><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n); break;
        case V3D_DAMP: k3d_dV<<<grid_faces(g, true), blk(), 0, s>>>(g, f, n); break;
        case VE3D_PERF:
        case V3D:
            if (f.Fx) k3_dV<true, true><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n);
            else k3_dV<true><<<grid_faces(g, true), blk(), 0, s>>>(g, f, n);
            break;
        case V2D: k2_dV<V2D><<<grid_faces(g, false), blk(), 0, s>>>(g, f, n); break;
        case VE2D: k2_dV<VE2D><<<grid_faces(g, false), blk(), 0, s>>>(g, f, n); break;
        case VE2D_PERF: k2_dV<VE2D_PERF><<<grid_faces(g, false), blk(), 0, s>>>(g, f, n); break;
        case V2D_DAMP:
        case VE2D_DAMP: k2d_dV<<<grid_faces(g, false), blk(), 0, s>>>(g, f, n); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_add_dV(int v, const Geom& g, const Fields64& f, cudaStream_t s) {
    if (v == V3D_DAMP) k3d_add_dV<<<grid_faces(g, true), blk(), 0, s>>>(g, f);
    else if (variant_is3d(v)) k3_add_dV<<<grid_faces(g, true), blk(), 0, s>>>(g, f);
    else if (variant_damped(v)) k2d_add_dV<<<grid_faces(g, false), blk(), 0, s>>>(g, f);
    else k2_add_dV<<<grid_faces(g, false), blk(), 0, s>>>(g, f);
    return cudaGetLastError();
}

// z-blocks of the 3D check/sources passes (each thread walks nz/PTS_CHECK_GZ planes)
#ifndef PTS_CHECK_GZ
#define PTS_CHECK_GZ 32
#endif
static dim3 check_grid(int v, const Geom& g) {
    if (variant_is3d(v)) return dim3((g.nx + 1 + 31) / 32, (g.ny + 7) / 8, g.nz < PTS_CHECK_GZ ? g.nz : PTS_CHECK_GZ);
    return dim3((g.nx + 1 + 31) / 32, (g.ny + 7) / 8, 1);
}

int check_num_blocks(int v, const Geom& g) {
    const dim3 gr = check_grid(v, g);
    return (int)(gr.x * gr.y * gr.z);
}

cudaError_t launch_check(int v, const Geom& g, const Fields64& f, const Num& n, double* partials, int nblocks_cap,
                         CheckResult* result, cudaStream_t s) {
    const dim3 gr = check_grid(v, g);
    const int nb = (int)(gr.x * gr.y * gr.z);
    if (nb > nblocks_cap) return cudaErrorInvalidValue;
    switch (v) {
        case VE3D:
        case V3D_DAMP: k3_check<false><<<gr, blk(), 0, s>>>(g, f, n, partials); break;
        case VE3D_PERF:
        case V3D:
            if (n.adjoint) {
                if (f.Fx) k3_check<true, true, true><<<gr, blk(), 0, s>>>(g, f, n, partials);
                else k3_check<true, false, true><<<gr, blk(), 0, s>>>(g, f, n, partials);
            } else if (f.Fx) {
                k3_check<true, true><<<gr, blk(), 0, s>>>(g, f, n, partials);
            } else {
                k3_check<true><<<gr, blk(), 0, s>>>(g, f, n, partials);
            }
            break;
        case V2D: k2_check<V2D><<<gr, blk(), 0, s>>>(g, f, n, partials); break;
        case VE2D: k2_check<VE2D><<<gr, blk(), 0, s>>>(g, f, n, partials); break;
        case VE2D_PERF: k2_check<VE2D_PERF><<<gr, blk(), 0, s>>>(g, f, n, partials); break;
        // the damped check is Stokes2D.jl's: ∇V stored by compute_P!, R of the current τ, Pt
        case V2D_DAMP:
        case VE2D_DAMP: k2_check<V2D><<<gr, blk(), 0, s>>>(g, f, n, partials); break;
        default: return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const bool d3 = variant_is3d(v);
    const double nx = g.nx, ny = g.ny, nz = d3 ? g.nz : 1;
    const double lenRx = d3 ? (nx - 1) * (ny - 2) * (nz - 2) : (nx - 1) * (ny - 2);
    const double lenRy = d3 ? (nx - 2) * (ny - 1) * (nz - 2) : (nx - 2) * (ny - 1);
    const double lenRz = d3 ? (nx - 2) * (ny - 2) * (nz - 1) : 1.0;
    const double lenDiv = nx * ny * nz;
    k_check_finalize<<<1, 256, 0, s>>>(partials, nb, make_double4(n.nsc[0], n.nsc[1], n.nsc[2], n.nsc[3]), lenRx, lenRy, lenRz, lenDiv, d3 ? 3 : 2, result);
    return cudaGetLastError();
}

cudaError_t launch_init_sweep(const Geom& g, const Fields64& f, const Num& n, double musi, double radius2,
                              double rhogi, double ebg, cudaStream_t s) {
    k2_init_sweep<<<grid_faces(g, false), blk(), 0, s>>>(g, f, n, musi, radius2, rhogi, ebg);
    return cudaGetLastError();
}

template <int TX, int TY>
static cudaError_t launch_batch_t(const BInst* d_inst, int ntiles, int ninst, const Fields64& F64, BState st,
                                  int nout, int64_t iter_last, double eps, cudaStream_t s) {
    SweepF F{F64.Pt, F64.Vx, F64.Vy, F64.txx, F64.tyy, F64.txy, F64.Mus, F64.divV, F64.Rx, F64.Ry, F64.rhog};
    int per_sm = 0, dev = 0, nsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2_batch<TX, TY>, TX * TY, 0);
    if (e != cudaSuccess) return e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    int grid = per_sm * nsm;  // every block co-resident, as grid.sync() requires
    const int want = ntiles > ninst ? ntiles : ninst;
    if (grid > want) grid = want;
    if (grid < 1) return cudaErrorInvalidConfiguration;
    void* args[] = {(void*)&d_inst, (void*)&ntiles,    (void*)&ninst, (void*)&F,
                    (void*)&st,     (void*)&nout,      (void*)&iter_last, (void*)&eps};
    return cudaLaunchCooperativeKernel((const void*)k2_batch<TX, TY>, dim3(grid), dim3(TX, TY), args, 0, s);
}

cudaError_t launch_batch(int tile, const BInst* d_inst, int ntiles, int ninst,
                         const Fields64& F, const BState& st, int nout, int64_t iter_last, double eps, cudaStream_t s) {
    switch (tile) {
        case 0: return launch_batch_t<32, 4>(d_inst, ntiles, ninst, F, st, nout, iter_last, eps, s);
        case 1: return launch_batch_t<32, 8>(d_inst, ntiles, ninst, F, st, nout, iter_last, eps, s);
        case 2: return launch_batch_t<64, 4>(d_inst, ntiles, ninst, F, st, nout, iter_last, eps, s);
        case 3: return launch_batch_t<32, 16>(d_inst, ntiles, ninst, F, st, nout, iter_last, eps, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int TX, int TY>
static cudaError_t launch_batch_ve_t(const BInst* d_inst, int ntiles, int ninst, const Fields64& F, BState st,
                                     BStateVE sv, int64_t iter_cap, double eps, cudaStream_t s) {
    int per_sm = 0, dev = 0, nsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2_batch_ve<TX, TY>, TX * TY, 0);
    if (e != cudaSuccess) return e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    int grid = per_sm * nsm;  // every block co-resident, as grid.sync() requires
    const int want = ntiles > ninst ? ntiles : ninst;
    if (grid > want) grid = want;
    if (grid < 1) return cudaErrorInvalidConfiguration;
    Fields64 Fv = F;
    void* args[] = {(void*)&d_inst, (void*)&ninst, (void*)&Fv, (void*)&st, (void*)&sv, (void*)&iter_cap, (void*)&eps};
    return cudaLaunchCooperativeKernel((const void*)k2_batch_ve<TX, TY>, dim3(grid), dim3(TX, TY), args, 0, s);
}

cudaError_t launch_batch_ve(int tile, const BInst* d_inst, int ntiles, int ninst, const Fields64& F,
                            const BState& st, const BStateVE& sv, int64_t iter_cap, double eps, cudaStream_t s) {
    switch (tile) {
        case 0: return launch_batch_ve_t<32, 4>(d_inst, ntiles, ninst, F, st, sv, iter_cap, eps, s);
        case 1: return launch_batch_ve_t<32, 8>(d_inst, ntiles, ninst, F, st, sv, iter_cap, eps, s);
        case 2: return launch_batch_ve_t<64, 4>(d_inst, ntiles, ninst, F, st, sv, iter_cap, eps, s);
        case 3: return launch_batch_ve_t<32, 16>(d_inst, ntiles, ninst, F, st, sv, iter_cap, eps, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_init_ve_param(const Geom& g, const Fields64& f, const Num& n, int nsub, double mus0, double musi,
                                 cudaStream_t s) {
    k2_init_ve_param<<<grid_cells(g), blk(), 0, s>>>(g, f, n, nsub, mus0, musi);
    return cudaGetLastError();
}

cudaError_t launch_fold(const Geom& g, const Fields64& f, const Mixed32& m, cudaStream_t s) {
    k_fold<<<148 * 8, 256, 0, s>>>(g.n, f, m);
    return cudaGetLastError();
}

cudaError_t launch_sources(int v, const Geom& g, const Fields64& f, const Mixed32& m, const Num& n, double* partials,
                           int nblocks_cap, CheckResult* result, cudaStream_t s) {
    const dim3 gr = check_grid(v, g);
    const int nb = (int)(gr.x * gr.y * gr.z);
    if (nb > nblocks_cap) return cudaErrorInvalidValue;
    if (v == VE3D_PERF) k3_sources<true><<<gr, blk(), 0, s>>>(g, f, m, n, partials);
    else if (v == V3D) k3_sources<false><<<gr, blk(), 0, s>>>(g, f, m, n, partials);
    else return cudaErrorInvalidValue;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const double nx = g.nx, ny = g.ny, nz = g.nz;
    k_check_finalize<<<1, 256, 0, s>>>(partials, nb, make_double4(n.nsc[0], n.nsc[1], n.nsc[2], n.nsc[3]), (nx - 1) * (ny - 2) * (nz - 2), (nx - 2) * (ny - 1) * (nz - 2),
                                       (nx - 2) * (ny - 2) * (nz - 1), nx * ny * nz, 3, result);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k3_srcw<<<grid_faces(g, true), blk(), 0, s>>>(g, f, m, n);
    return cudaGetLastError();
}

cudaError_t launch_coef32(const Geom& g, const Fields64& f, const Mixed32& m, cudaStream_t s) {
    k_coef32<<<148 * 8, 256, 0, s>>>(g.n, f.Gdt, f.Mus, f.dtRho, m.GM, m.dtRho);
    return cudaGetLastError();
}

cudaError_t launch_init_inclusion(int v, const Geom& g, const Fields64& f, const Num& n, double mus0, double musi,
                                  double radius2, double ebg, cudaStream_t s) {
    const bool d3 = variant_is3d(v);
    const dim3 gr = grid_faces(g, d3);
    // the multi-XPU scripts build their ICs through ImplicitGlobalGrid's x_g
    if (v == VE3D || v == V3D_DAMP) k_init_inclusion<true, true><<<gr, blk(), 0, s>>>(g, f, n, mus0, musi, radius2, ebg);
    else if (d3) k_init_inclusion<true, false><<<gr, blk(), 0, s>>>(g, f, n, mus0, musi, radius2, ebg);
    else k_init_inclusion<false, false><<<gr, blk(), 0, s>>>(g, f, n, mus0, musi, radius2, ebg);
    return cudaGetLastError();
}

cudaError_t launch_init_inclusions(int v, const Geom& g, const Fields64& f, const Num& n, const pts_inclusion* d_inc,
                                   int count, double mus0, double ebg, cudaStream_t s) {
    const bool d3 = variant_is3d(v);
    const dim3 gr = grid_faces(g, d3);
    if (v == VE3D || v == V3D_DAMP) k_init_inclusions<true, true><<<gr, blk(), 0, s>>>(g, f, n, d_inc, count, mus0, ebg);
    else if (d3) k_init_inclusions<true, false><<<gr, blk(), 0, s>>>(g, f, n, d_inc, count, mus0, ebg);
    else k_init_inclusions<false, false><<<gr, blk(), 0, s>>>(g, f, n, d_inc, count, mus0, ebg);
    return cudaGetLastError();
}

cudaError_t launch_smooth(int v, const Geom& g, double* dst, const double* src, double fact, cudaStream_t s) {
    if (variant_is3d(v)) k_smooth<true><<<grid_cells(g), blk(), 0, s>>>(g, dst, src, 1.0 / 6.1 / fact);
    else k_smooth<false><<<grid_cells(g), blk(), 0, s>>>(g, dst, src, 1.0 / 4.1 / fact);
    return cudaGetLastError();
}

cudaError_t launch_maxloc(int v, const Geom& g, double* must, const double* mus, cudaStream_t s) {
    if (variant_is3d(v)) k_maxloc<true><<<grid_cells(g), blk(), 0, s>>>(g, must, mus);
    else k_maxloc<false><<<grid_cells(g), blk(), 0, s>>>(g, must, mus);
    return cudaGetLastError();
}

cudaError_t launch_iter_params(int v, const Geom& g, const Fields64& f, const Num& n, cudaStream_t s) {
    if (v == V3D_DAMP) k3d_timesteps<<<grid_faces(g, true), blk(), 0, s>>>(g, f, n);
    else if (variant_damped(v)) k2d_timesteps<<<grid_faces(g, false), blk(), 0, s>>>(g, f, n);
    else if (variant_elastic(v)) k_iter_params<true><<<grid_cells(g), blk(), 0, s>>>(g, f, n);
    else k_iter_params<false><<<grid_cells(g), blk(), 0, s>>>(g, f, n);
    return cudaGetLastError();
}

cudaError_t launch_tau_exact(const Geom& g, const Fields64& f, const Num& n, cudaStream_t s) {
    k3_tau_exact<<<grid_cells(g), blk(), 0, s>>>(g, f, n);
    return cudaGetLastError();
}

cudaError_t launch_grad_logmu(const Geom& g, const Fields64& fwd, const Fields64& adj, const Num& n, cudaStream_t s) {
    if (!fwd.grad) return cudaErrorInvalidValue;
    k3_grad_logmu<<<grid_cells(g), blk(), 0, s>>>(g, fwd, adj, n);
    return cudaGetLastError();
}

cudaError_t launch_grad_logmu_ve(const Geom& g, const Fields64& fwd, const Fields64& adj, bool add, cudaStream_t s) {
    if (!fwd.grad) return cudaErrorInvalidValue;
    if (add) k3_grad_logmu_ve<true><<<grid_cells(g), blk(), 0, s>>>(g, fwd, adj);
    else k3_grad_logmu_ve<false><<<grid_cells(g), blk(), 0, s>>>(g, fwd, adj);
    return cudaGetLastError();
}

}  // namespace pts

// ------------------------------------------------------------------ single-pass 3D (FP64)
#include "pts_fused3d.cuh"

namespace pts {

static Fused3Args<double> fused_args(const Fields64& cur, const Fields64& nxt, int* err) {
    Fused3Args<double> a{};
    const double* g1[] = {cur.txx, cur.tyy, cur.tzz, cur.txy, cur.txz, cur.tyz, cur.Pt, cur.dtRho};
    for (int q = 0; q < 8; ++q) a.g1[q] = g1[q];
    a.g2[0] = cur.Vx; a.g2[1] = cur.Vy; a.g2[2] = cur.Vz;
    a.g3[0] = cur.Gdt; a.g3[1] = cur.Mus;
    const double* g4[] = {cur.txx_o, cur.tyy_o, cur.tzz_o, cur.txy_o, cur.txz_o, cur.tyz_o};
    for (int q = 0; q < 6; ++q) a.g4[q] = g4[q];
    a.Vx2 = nxt.Vx; a.Vy2 = nxt.Vy; a.Vz2 = nxt.Vz;
    a.txx2 = nxt.txx; a.tyy2 = nxt.tyy; a.tzz2 = nxt.tzz; a.txy2 = nxt.txy; a.txz2 = nxt.txz; a.tyz2 = nxt.tyz;
    a.Pt2 = nxt.Pt;
    a.divV = cur.divV;
    a.err = err;
    return a;
}

// z-planes per CTA: enough CTAs for ~8 waves at one resident CTA per SM, long z runs to
// amortise the two recomputed boundary planes of each chunk.
int fused3_zchunk(const Geom& g) {
    const int tiles = ((g.nx + 1 + fused3::TX - 1) / fused3::TX) * ((g.ny + 1 + fused3::TY - 1) / fused3::TY);
    int zch = g.nz + 1;
    while (zch > 16 && (int64_t)tiles * ((g.nz + 1 + zch - 1) / zch) < 148 * 8) zch = (zch + 1) / 2;
    return zch;
}

#ifndef PTS_DIRECT_ZCH
#define PTS_DIRECT_ZCH 16
#endif
template <typename T, bool EL, bool PERF, bool CORR>
cudaError_t launch_fused3_t(const Geom& g, const Fused3Args<T>& a, const NumT<T>& n, bool store_divV, cudaStream_t s,
                            bool direct) {
    using C = fused3::Cfg<T, EL, CORR>;
    if (direct) {
        // short z-chunks: many independent blocks; each chunk recomputes one extra B plane
        const int zch = PTS_DIRECT_ZCH;
        const dim3 grid((g.nx + 1 + fused3::TX - 1) / fused3::TX, (g.ny + 1 + fused3::TY - 1) / fused3::TY,
                        (g.nz + 1 + zch - 1) / zch);
        k3_fused_direct<T, EL, PERF, CORR><<<grid, dim3(fused3::TX, fused3::TY, 1), 0, s>>>(g, a, n, zch,
                                                                                          store_divV ? 1 : 0);
        return cudaGetLastError();
    }
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k3_fused_BA<T, EL, PERF, CORR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)C::smem_bytes);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int zch = fused3_zchunk(g);
    const dim3 grid((g.nx + 1 + fused3::TX - 1) / fused3::TX, (g.ny + 1 + fused3::TY - 1) / fused3::TY,
                    (g.nz + 1 + zch - 1) / zch);
    k3_fused_BA<T, EL, PERF, CORR><<<grid, dim3(fused3::TX, fused3::TY, 1), C::smem_bytes, s>>>(g, a, n, zch,
                                                                                              store_divV ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_fused3(int v, const Geom& g, const Fields64& cur, const Fields64& nxt, const Num& nm,
                          bool store_divV, int* err, cudaStream_t s, bool direct) {
    const Fused3Args<double> a = fused_args(cur, nxt, err);
    NumT<double> n{nm.dx, nm.dy, nm.dz, nm._dx, nm._dy, nm._dz, nm.r, nm.gdt, 2.0, 0.5, 1.0, 0.25,
                   nm.gdt == 1.0 ? 1 : 0};
    switch (v) {
        case VE3D_PERF: return launch_fused3_t<double, true, true, false>(g, a, n, store_divV, s, direct);
        case V3D: return launch_fused3_t<double, false, true, false>(g, a, n, store_divV, s, direct);
        case VE3D: return launch_fused3_t<double, true, false, false>(g, a, n, store_divV, s, direct);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pts
