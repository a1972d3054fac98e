// ptstokes_oracle.cpp -- CPU restatement (C++17 + OpenMP, FP64) of the reference's
// pseudo-transient Stokes stencil kernels.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity oracle: it is built and called
// by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, and only
// as the checker. The product (libptstokes.so) never links or calls it.
//
// Every function restates one kernel of PTsolvers/PseudoTransientStokes.jl index
// for index, with Julia's 1-based column-major indexing kept literally (the A(i,j,k)
// accessors below subtract 1) so a reader can lay each line beside the reference.
// Floating point follows Julia's left-to-right evaluation of `a + b + c` and
// `a*b/c`; the build uses -ffp-contract=off so no multiply-add is fused, which is
// what Julia/LLVM does for these scripts on the Threads backend.
//
// The ParallelStencil FiniteDifferences macros (@d_xa, @d_xi, @av, @av_xi,
// @av_xyi, @d2_xi, @maxloc, @inn, @all) are not vendored in the reference; they are
// restated here from their published definitions in ParallelStencil.jl
// (FiniteDifferences2D / FiniteDifferences3D): "a" = along the whole extent,
// "i" = on the inner points of the other dimensions (index + 1).
// Each @parallel statement `@all(A) = ...` / `@inn(A) = ...` is guarded by the
// extent of its left-hand side, exactly as @parallel generates it.
#include <cstdint>
#include <cmath>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// A field as the reference holds it: Float64 column-major, extents n1 x n2 x n3
// (n3 = 1 in 2D).
struct oarr {
    double* p;
    int64_t n1, n2, n3;
};

}  // extern "C"

namespace {

struct F2 {
    double* p; int64_t n1, n2;
    F2(const oarr& a) : p(a.p), n1(a.n1), n2(a.n2) {}
    inline double& operator()(int64_t i, int64_t j) const { return p[(i - 1) + n1 * (j - 1)]; }
};
struct F3 {
    double* p; int64_t n1, n2, n3;
    F3(const oarr& a) : p(a.p), n1(a.n1), n2(a.n2), n3(a.n3) {}
    inline double& operator()(int64_t i, int64_t j, int64_t k) const {
        return p[(i - 1) + n1 * ((j - 1) + n2 * (k - 1))];
    }
};

}  // namespace

extern "C" {

// ---------------------------------------------------------------- generic helpers

// assign_τ! / `Mus2 .= Mus` / `Musτ .= Mus`: elementwise copy over the whole array
// (Stokes2D_ve.jl:35-40, Stokes3D_ve_perf.jl:41-49).
void ora_copy(oarr dst, oarr src) {
    const int64_t n = dst.n1 * dst.n2 * dst.n3;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) dst.p[i] = src.p[i];
}

// compute_iter_params! viscous (Stokes2D.jl:27-31, Stokes2D_param.jl:36-40):
//   dτ_Rho = Vpdτ*max_lxy/Re/Musτ ;  Gdτ = Vpdτ^2/dτ_Rho/(r+2.0)
void ora_iter_params_v(oarr dtRho, oarr Gdt, oarr Must, double Vpdt, double Re, double r, double max_l) {
    const int64_t n = dtRho.n1 * dtRho.n2 * dtRho.n3;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        dtRho.p[i] = Vpdt * max_l / Re / Must.p[i];
        Gdt.p[i] = (Vpdt * Vpdt) / dtRho.p[i] / (r + 2.0);
    }
}

// compute_iter_params! visco-elastic (Stokes2D_ve.jl:28-33, Stokes2D_ve_perf.jl:29-34,
// Stokes3D_ve_perf.jl:34-39):
//   μ_eff = 1.0/(1.0/Musτ + 1.0/(G*dt)); dτ_Rho = Vpdτ*max_l/Re/μ_eff; Gdτ = Vpdτ^2/dτ_Rho/(r+2)
void ora_iter_params_ve(oarr dtRho, oarr Gdt, oarr Must, double Vpdt, double G, double dt,
                        double Re, double r, double max_l) {
    const int64_t n = dtRho.n1 * dtRho.n2 * dtRho.n3;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double mu_eff = 1.0 / (1.0 / Must.p[i] + 1.0 / (G * dt));
        dtRho.p[i] = Vpdt * max_l / Re / mu_eff;
        Gdt.p[i] = (Vpdt * Vpdt) / dtRho.p[i] / (r + 2.0);
    }
}

// ---------------------------------------------------------------- 2D set-up kernels

// smooth! (Stokes2D.jl:17-20): @inn(A2) = @inn(A) + 1.0/4.1/fact*(@d2_xi(A) + @d2_yi(A))
void ora2_smooth(oarr A2_, oarr A_, double fact) {
    F2 A2(A2_), A(A_);
    const double c = 1.0 / 4.1 / fact;
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= A2.n2 - 2; ++iy)
        for (int64_t ix = 1; ix <= A2.n1 - 2; ++ix) {
            const int64_t i = ix + 1, j = iy + 1;
            const double d2x = (A(i + 1, j) - A(i, j)) - (A(i, j) - A(i - 1, j));
            const double d2y = (A(i, j + 1) - A(i, j)) - (A(i, j) - A(i, j - 1));
            A2(i, j) = A(i, j) + c * (d2x + d2y);
        }
}

// compute_maxloc! (Stokes2D.jl:22-25): @inn(B) = @maxloc(A), the max over the point and
// its four axis neighbours.
void ora2_maxloc(oarr B_, oarr A_) {
    F2 B(B_), A(A_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= B.n2 - 2; ++iy)
        for (int64_t ix = 1; ix <= B.n1 - 2; ++ix) {
            const int64_t i = ix + 1, j = iy + 1;
            B(i, j) = std::max(std::max(std::max(std::max(A(i - 1, j), A(i + 1, j)), A(i, j)), A(i, j - 1)),
                               A(i, j + 1));
        }
}

// bc_x! / bc_y! (Stokes2D.jl:60-70): free-slip copy of the first/last interior line.
void ora2_bc_x(oarr A_) {
    F2 A(A_);
    for (int64_t iy = 1; iy <= A.n2; ++iy) {
        A(1, iy) = A(2, iy);
        A(A.n1, iy) = A(A.n1 - 1, iy);
    }
}
void ora2_bc_y(oarr A_) {
    F2 A(A_);
    for (int64_t ix = 1; ix <= A.n1; ++ix) {
        A(ix, 1) = A(ix, 2);
        A(ix, A.n2) = A(ix, A.n2 - 1);
    }
}

// ---------------------------------------------------------------- 2D viscous (Stokes2D.jl)

// compute_P! (Stokes2D.jl:33-37, Stokes2D_ve.jl:42-46):
//   @all(∇V) = @d_xa(Vx)/dx + @d_ya(Vy)/dy ; @all(Pt) = @all(Pt) - r*@all(Gdτ)*@all(∇V)
void ora2_compute_P(oarr divV_, oarr Pt_, oarr Vx_, oarr Vy_, oarr Gdt_, double r, double dx, double dy) {
    F2 divV(divV_), Pt(Pt_), Vx(Vx_), Vy(Vy_), Gdt(Gdt_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Pt.n2; ++iy)
        for (int64_t ix = 1; ix <= Pt.n1; ++ix) {
            divV(ix, iy) = (Vx(ix + 1, iy) - Vx(ix, iy)) / dx + (Vy(ix, iy + 1) - Vy(ix, iy)) / dy;
            Pt(ix, iy) = Pt(ix, iy) - r * Gdt(ix, iy) * divV(ix, iy);
        }
}

// compute_τ! viscous (Stokes2D.jl:39-44)
void ora2v_compute_tau(oarr txx_, oarr tyy_, oarr txy_, oarr Vx_, oarr Vy_, oarr Mus_, oarr Gdt_,
                       double dx, double dy) {
    F2 txx(txx_), tyy(tyy_), txy(txy_), Vx(Vx_), Vy(Vy_), Mus(Mus_), Gdt(Gdt_);
    const int64_t nx = txx.n1, ny = txx.n2;
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= ny; ++iy)
        for (int64_t ix = 1; ix <= nx; ++ix) {
            txx(ix, iy) = (txx(ix, iy) + 2.0 * Gdt(ix, iy) * (Vx(ix + 1, iy) - Vx(ix, iy)) / dx) /
                          (Gdt(ix, iy) / Mus(ix, iy) + 1.0);
            tyy(ix, iy) = (tyy(ix, iy) + 2.0 * Gdt(ix, iy) * (Vy(ix, iy + 1) - Vy(ix, iy)) / dy) /
                          (Gdt(ix, iy) / Mus(ix, iy) + 1.0);
            if (ix <= txy.n1 && iy <= txy.n2) {
                const double avG = (Gdt(ix, iy) + Gdt(ix + 1, iy) + Gdt(ix, iy + 1) + Gdt(ix + 1, iy + 1)) * 0.25;
                const double avM = (Mus(ix, iy) + Mus(ix + 1, iy) + Mus(ix, iy + 1) + Mus(ix + 1, iy + 1)) * 0.25;
                txy(ix, iy) = (txy(ix, iy) + 2.0 * avG *
                                                 (0.5 * ((Vx(ix + 1, iy + 1) - Vx(ix + 1, iy)) / dy +
                                                         (Vy(ix + 1, iy + 1) - Vy(ix, iy + 1)) / dx))) /
                              (avG / avM + 1.0);
            }
        }
}

// compute_dV! viscous (Stokes2D.jl:46-52): stores Rx, Ry and dV = @av_xi(dτ_Rho)*R.
void ora2v_compute_dV(oarr Rx_, oarr Ry_, oarr dVx_, oarr dVy_, oarr Pt_, oarr txx_, oarr tyy_, oarr txy_,
                      oarr dtRho_, double dx, double dy) {
    F2 Rx(Rx_), Ry(Ry_), dVx(dVx_), dVy(dVy_), Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_), dtR(dtRho_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Ry.n2; ++iy)
        for (int64_t ix = 1; ix <= Rx.n1; ++ix) {
            if (ix <= Rx.n1 && iy <= Rx.n2) {
                Rx(ix, iy) = (txx(ix + 1, iy + 1) - txx(ix, iy + 1)) / dx + (txy(ix, iy + 1) - txy(ix, iy)) / dy -
                             (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1)) / dx;
                dVx(ix, iy) = (dtR(ix, iy + 1) + dtR(ix + 1, iy + 1)) * 0.5 * Rx(ix, iy);
            }
            if (ix <= Ry.n1 && iy <= Ry.n2) {
                Ry(ix, iy) = (tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) / dy + (txy(ix + 1, iy) - txy(ix, iy)) / dx -
                             (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy)) / dy;
                dVy(ix, iy) = (dtR(ix + 1, iy) + dtR(ix + 1, iy + 1)) * 0.5 * Ry(ix, iy);
            }
        }
}

// compute_V! (Stokes2D.jl:54-58): @inn(Vx) = @inn(Vx) + @all(dVx) ; same for Vy.
void ora2_compute_V(oarr Vx_, oarr Vy_, oarr dVx_, oarr dVy_) {
    F2 Vx(Vx_), Vy(Vy_), dVx(dVx_), dVy(dVy_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= std::max(dVx.n2, dVy.n2); ++iy)
        for (int64_t ix = 1; ix <= std::max(dVx.n1, dVy.n1); ++ix) {
            if (ix <= dVx.n1 && iy <= dVx.n2) Vx(ix + 1, iy + 1) = Vx(ix + 1, iy + 1) + dVx(ix, iy);
            if (ix <= dVy.n1 && iy <= dVy.n2) Vy(ix + 1, iy + 1) = Vy(ix + 1, iy + 1) + dVy(ix, iy);
        }
}

// ---------------------------------------------------------------- 2D visco-elastic (Stokes2D_ve.jl)

// compute_τ! VE (Stokes2D_ve.jl:48-55), Gr = @all(Gdτ)/(G*dt), av_Gr = @av(Gdτ)/(G*dt)
void ora2ve_compute_tau(oarr txx_, oarr tyy_, oarr txy_, oarr txxo_, oarr tyyo_, oarr txyo_, oarr Gdt_,
                        oarr Vx_, oarr Vy_, oarr Mus_, double G, double dt, double dx, double dy) {
    F2 txx(txx_), tyy(tyy_), txy(txy_), txxo(txxo_), tyyo(tyyo_), txyo(txyo_), Gdt(Gdt_), Vx(Vx_), Vy(Vy_),
        Mus(Mus_);
    const int64_t nx = txx.n1, ny = txx.n2;
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= ny; ++iy)
        for (int64_t ix = 1; ix <= nx; ++ix) {
            const double Gr = Gdt(ix, iy) / (G * dt);
            txx(ix, iy) = (txx(ix, iy) + txxo(ix, iy) * Gr + 2.0 * Gdt(ix, iy) * ((Vx(ix + 1, iy) - Vx(ix, iy)) / dx)) /
                          (1.0 + Gdt(ix, iy) / Mus(ix, iy) + Gr);
            tyy(ix, iy) = (tyy(ix, iy) + tyyo(ix, iy) * Gr + 2.0 * Gdt(ix, iy) * ((Vy(ix, iy + 1) - Vy(ix, iy)) / dy)) /
                          (1.0 + Gdt(ix, iy) / Mus(ix, iy) + Gr);
            if (ix <= txy.n1 && iy <= txy.n2) {
                const double avG = (Gdt(ix, iy) + Gdt(ix + 1, iy) + Gdt(ix, iy + 1) + Gdt(ix + 1, iy + 1)) * 0.25;
                const double avM = (Mus(ix, iy) + Mus(ix + 1, iy) + Mus(ix, iy + 1) + Mus(ix + 1, iy + 1)) * 0.25;
                const double avGr = avG / (G * dt);
                txy(ix, iy) = (txy(ix, iy) + txyo(ix, iy) * avGr +
                               2.0 * avG *
                                   (0.5 * ((Vx(ix + 1, iy + 1) - Vx(ix + 1, iy)) / dy +
                                           (Vy(ix + 1, iy + 1) - Vy(ix, iy + 1)) / dx))) /
                              (1.0 + avG / avM + avGr);
            }
        }
}

// compute_dV! VE (Stokes2D_ve.jl:57-61):
//   @all(dVx) = (@d_xi(τxx)/dx + @d_ya(τxy)/dy - @d_xi(Pt)/dx)*@av_xi(dτ_Rho)
void ora2ve_compute_dV(oarr dVx_, oarr dVy_, oarr Pt_, oarr txx_, oarr tyy_, oarr txy_, oarr dtRho_,
                       double dx, double dy) {
    F2 dVx(dVx_), dVy(dVy_), Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_), dtR(dtRho_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= dVy.n2; ++iy)
        for (int64_t ix = 1; ix <= dVx.n1; ++ix) {
            if (ix <= dVx.n1 && iy <= dVx.n2)
                dVx(ix, iy) = ((txx(ix + 1, iy + 1) - txx(ix, iy + 1)) / dx + (txy(ix, iy + 1) - txy(ix, iy)) / dy -
                               (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1)) / dx) *
                              ((dtR(ix, iy + 1) + dtR(ix + 1, iy + 1)) * 0.5);
            if (ix <= dVy.n1 && iy <= dVy.n2)
                dVy(ix, iy) = ((tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) / dy + (txy(ix + 1, iy) - txy(ix, iy)) / dx -
                               (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy)) / dy) *
                              ((dtR(ix + 1, iy) + dtR(ix + 1, iy + 1)) * 0.5);
        }
}

// compute_Res! VE (Stokes2D_ve.jl:69-73)
void ora2ve_compute_Res(oarr Rx_, oarr Ry_, oarr Pt_, oarr txx_, oarr tyy_, oarr txy_, double dx, double dy) {
    F2 Rx(Rx_), Ry(Ry_), Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Ry.n2; ++iy)
        for (int64_t ix = 1; ix <= Rx.n1; ++ix) {
            if (ix <= Rx.n1 && iy <= Rx.n2)
                Rx(ix, iy) = (txx(ix + 1, iy + 1) - txx(ix, iy + 1)) / dx + (txy(ix, iy + 1) - txy(ix, iy)) / dy -
                             (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1)) / dx;
            if (ix <= Ry.n1 && iy <= Ry.n2)
                Ry(ix, iy) = (tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) / dy + (txy(ix + 1, iy) - txy(ix, iy)) / dx -
                             (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy)) / dy;
        }
}

// ---------------------------------------------------------------- 2D VE explicit-index (Stokes2D_ve_perf.jl)

// compute_Pt_τ! (Stokes2D_ve_perf.jl:43-53)
void ora2p_compute_Pt_tau(oarr Pt_, oarr txx_, oarr tyy_, oarr txy_, oarr txxo_, oarr tyyo_, oarr txyo_, oarr Gdt_,
                          oarr Vx_, oarr Vy_, oarr Mus_, double r, double G, double dt, double _dx, double _dy) {
    F2 Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_), txxo(txxo_), tyyo(tyyo_), txyo(txyo_), Gdt(Gdt_), Vx(Vx_), Vy(Vy_),
        Mus(Mus_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Pt.n2; ++iy)
        for (int64_t ix = 1; ix <= Pt.n1; ++ix) {
            Pt(ix, iy) = Pt(ix, iy) - r * Gdt(ix, iy) * (_dx * (Vx(ix + 1, iy) - Vx(ix, iy)) + _dy * (Vy(ix, iy + 1) - Vy(ix, iy)));
            const double Gr = Gdt(ix, iy) / (G * dt);
            txx(ix, iy) = (txx(ix, iy) + txxo(ix, iy) * Gr + 2.0 * Gdt(ix, iy) * (_dx * (Vx(ix + 1, iy) - Vx(ix, iy)))) /
                          (1.0 + Gdt(ix, iy) / Mus(ix, iy) + Gr);
            tyy(ix, iy) = (tyy(ix, iy) + tyyo(ix, iy) * Gr + 2.0 * Gdt(ix, iy) * (_dy * (Vy(ix, iy + 1) - Vy(ix, iy)))) /
                          (1.0 + Gdt(ix, iy) / Mus(ix, iy) + Gr);
            if (ix <= txy.n1 && iy <= txy.n2) {
                const double avG = 0.25 * (Gdt(ix, iy) + Gdt(ix + 1, iy) + Gdt(ix, iy + 1) + Gdt(ix + 1, iy + 1));
                const double avM = 0.25 * (Mus(ix, iy) + Mus(ix + 1, iy) + Mus(ix, iy + 1) + Mus(ix + 1, iy + 1));
                const double avGr = avG / (G * dt);
                txy(ix, iy) = (txy(ix, iy) + txyo(ix, iy) * avGr +
                               2.0 * avG * 0.5 *
                                   (_dy * (Vx(ix + 1, iy + 1) - Vx(ix + 1, iy)) + _dx * (Vy(ix + 1, iy + 1) - Vy(ix, iy + 1)))) /
                              (1.0 + avG / avM + avGr);
            }
        }
}

// compute_V! (Stokes2D_ve_perf.jl:55-59), the fused compute_dV!/compute_V! roles.
void ora2p_compute_V(oarr Vx_, oarr Vy_, oarr Pt_, oarr txx_, oarr tyy_, oarr txy_, oarr dtRho_, double _dx,
                     double _dy, int64_t sVx1, int64_t sVx2, int64_t sVy1, int64_t sVy2) {
    F2 Vx(Vx_), Vy(Vy_), Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_), dtR(dtRho_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= std::max(sVx2, sVy2); ++iy)
        for (int64_t ix = 1; ix <= std::max(sVx1, sVy1); ++ix) {
            if (ix <= sVx1 && iy <= sVx2)
                Vx(ix + 1, iy + 1) = Vx(ix + 1, iy + 1) +
                                     (_dx * (txx(ix + 1, iy + 1) - txx(ix, iy + 1)) + _dy * (txy(ix, iy + 1) - txy(ix, iy)) -
                                      _dx * (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1))) *
                                         (0.5 * (dtR(ix, iy + 1) + dtR(ix + 1, iy + 1)));
            if (ix <= sVy1 && iy <= sVy2)
                Vy(ix + 1, iy + 1) = Vy(ix + 1, iy + 1) +
                                     (_dy * (tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) + _dx * (txy(ix + 1, iy) - txy(ix, iy)) -
                                      _dy * (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy))) *
                                         (0.5 * (dtR(ix + 1, iy) + dtR(ix + 1, iy + 1)));
        }
}

// compute_Res! (Stokes2D_ve_perf.jl:61-66): ∇V recomputed from the current V.
void ora2p_compute_Res(oarr divV_, oarr Rx_, oarr Ry_, oarr Pt_, oarr Vx_, oarr Vy_, oarr txx_, oarr tyy_, oarr txy_,
                       double _dx, double _dy) {
    F2 divV(divV_), Rx(Rx_), Ry(Ry_), Pt(Pt_), Vx(Vx_), Vy(Vy_), txx(txx_), tyy(tyy_), txy(txy_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= divV.n2; ++iy)
        for (int64_t ix = 1; ix <= divV.n1; ++ix) {
            divV(ix, iy) = _dx * (Vx(ix + 1, iy) - Vx(ix, iy)) + _dy * (Vy(ix, iy + 1) - Vy(ix, iy));
            if (ix <= Rx.n1 && iy <= Rx.n2)
                Rx(ix, iy) = _dx * (txx(ix + 1, iy + 1) - txx(ix, iy + 1)) + _dy * (txy(ix, iy + 1) - txy(ix, iy)) -
                             _dx * (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1));
            if (ix <= Ry.n1 && iy <= Ry.n2)
                Ry(ix, iy) = _dy * (tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) + _dx * (txy(ix + 1, iy) - txy(ix, iy)) -
                             _dy * (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy));
        }
}

// ---------------------------------------------------------------- 2D viscous sweep form (Stokes2D_param.jl)

// create_inclusions! (Stokes2D_param.jl:83-99): per cell, inside any circle (Xi, Yi, r2)?
void ora2_create_inclusions(oarr Mus_, oarr rhog_, const double* Xi, const double* Yi, int64_t ni, double r2,
                            double mus0, double musi, double rhog0, double rhogi, double dx, double dy, double lx,
                            double ly) {
    F2 Mus(Mus_), rhog(rhog_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Mus.n2; ++iy)
        for (int64_t ix = 1; ix <= Mus.n1; ++ix) {
            const double x = (ix - 1) * dx + 0.5 * dx - 0.5 * lx;
            const double y = (iy - 1) * dy + 0.5 * dy - 0.5 * ly;
            bool inside = false;
            for (int64_t q = 0; q < ni; ++q) {
                const double ddx = x - Xi[q], ddy = y - Yi[q];
                if (ddx * ddx + ddy * ddy < r2) { inside = true; break; }
            }
            Mus(ix, iy) = inside ? musi : mus0;
            rhog(ix, iy) = inside ? rhogi : rhog0;
        }
}

// create_inclusions! (Stokes2D_param.jl:83-99) over a list of inclusions, each with its own
// squared radius r2[q] and viscosity musi[q], in 2D (Zi unused, n3 = 1) or 3D (the same
// test with the z term added last): Mus = musi of the first inclusion the cell centre is
// inside (the reference's loop breaks at the first hit), else mus0. Centres are in the
// reference's centred frame: x = (ix-1)*dx + 0.5*dx - 0.5*lx.
void ora_create_inclusions_list(oarr Mus_, const double* Xi, const double* Yi, const double* Zi, const double* r2,
                                const double* musi, int64_t ni, double mus0, double dx, double dy, double dz,
                                double lx, double ly, double lz, int d3) {
    F3 Mus(Mus_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= Mus.n3; ++iz)
        for (int64_t iy = 1; iy <= Mus.n2; ++iy)
            for (int64_t ix = 1; ix <= Mus.n1; ++ix) {
                const double x = (ix - 1) * dx + 0.5 * dx - 0.5 * lx;
                const double y = (iy - 1) * dy + 0.5 * dy - 0.5 * ly;
                const double z = (iz - 1) * dz + 0.5 * dz - 0.5 * lz;
                double mu = mus0;
                for (int64_t q = 0; q < ni; ++q) {
                    const double ax = x - Xi[q], ay = y - Yi[q];
                    double rad2 = ax * ax + ay * ay;
                    if (d3) {
                        const double az = z - Zi[q];
                        rad2 = rad2 + az * az;
                    }
                    if (rad2 < r2[q]) {
                        mu = musi[q];
                        break;
                    }
                }
                Mus(ix, iy, iz) = mu;
            }
}

// compute_τ! (Stokes2D_param.jl:48-55): τ = 2μ_veτ(ε̇ + τ/Gdτ/2), μ_veτ = 1/(1/Gdτ + 1/Mus)
void ora2s_compute_tau(oarr txx_, oarr tyy_, oarr txy_, oarr Vx_, oarr Vy_, oarr Mus_, oarr Gdt_, double dx,
                       double dy) {
    F2 txx(txx_), tyy(tyy_), txy(txy_), Vx(Vx_), Vy(Vy_), Mus(Mus_), Gdt(Gdt_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= txx.n2; ++iy)
        for (int64_t ix = 1; ix <= txx.n1; ++ix) {
            const double mu = 1.0 / (1.0 / Gdt(ix, iy) + 1.0 / Mus(ix, iy));
            txx(ix, iy) = 2.0 * mu * ((Vx(ix + 1, iy) - Vx(ix, iy)) / dx + txx(ix, iy) / Gdt(ix, iy) / 2.0);
            tyy(ix, iy) = 2.0 * mu * ((Vy(ix, iy + 1) - Vy(ix, iy)) / dy + tyy(ix, iy) / Gdt(ix, iy) / 2.0);
            if (ix <= txy.n1 && iy <= txy.n2) {
                const double avG = (Gdt(ix, iy) + Gdt(ix + 1, iy) + Gdt(ix, iy + 1) + Gdt(ix + 1, iy + 1)) * 0.25;
                const double avM = (Mus(ix, iy) + Mus(ix + 1, iy) + Mus(ix, iy + 1) + Mus(ix + 1, iy + 1)) * 0.25;
                const double mua = 1.0 / (1.0 / avG + 1.0 / avM);
                txy(ix, iy) = 2.0 * mua *
                              (0.5 * ((Vx(ix + 1, iy + 1) - Vx(ix + 1, iy)) / dy + (Vy(ix + 1, iy + 1) - Vy(ix, iy + 1)) / dx) +
                               txy(ix, iy) / avG / 2.0);
            }
        }
}

// compute_dV! (Stokes2D_param.jl:57-63): as Stokes2D.jl with the buoyancy term -@av_yi(ρg) in Ry.
void ora2s_compute_dV(oarr Rx_, oarr Ry_, oarr dVx_, oarr dVy_, oarr Pt_, oarr txx_, oarr tyy_, oarr txy_,
                      oarr dtRho_, oarr rhog_, double dx, double dy) {
    F2 Rx(Rx_), Ry(Ry_), dVx(dVx_), dVy(dVy_), Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_), dtR(dtRho_), rg(rhog_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Ry.n2; ++iy)
        for (int64_t ix = 1; ix <= Rx.n1; ++ix) {
            if (ix <= Rx.n1 && iy <= Rx.n2) {
                Rx(ix, iy) = (txx(ix + 1, iy + 1) - txx(ix, iy + 1)) / dx + (txy(ix, iy + 1) - txy(ix, iy)) / dy -
                             (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1)) / dx;
                dVx(ix, iy) = (dtR(ix, iy + 1) + dtR(ix + 1, iy + 1)) * 0.5 * Rx(ix, iy);
            }
            if (ix <= Ry.n1 && iy <= Ry.n2) {
                Ry(ix, iy) = (tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) / dy + (txy(ix + 1, iy) - txy(ix, iy)) / dx -
                             (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy)) / dy - (rg(ix + 1, iy) + rg(ix + 1, iy + 1)) * 0.5;
                dVy(ix, iy) = (dtR(ix + 1, iy) + dtR(ix + 1, iy + 1)) * 0.5 * Ry(ix, iy);
            }
        }
}

// ---------------------------------------------------------------- 2D damped scheme ("accel. 1")
// scripts/previous_damp/Stokes2D0.jl (viscous) and Stokes2D_ve0.jl (Maxwell visco-elastic):
// numerical compressibility β_n, a damped velocity rate dV/dτ and per-face pseudo-time steps.

// compute_timesteps! (Stokes2D_ve0.jl:27-32, Stokes2D0.jl:26-31)
void ora2d_timesteps(oarr dtVx_, oarr dtVy_, oarr dtPt_, oarr Must_, double Vsc, double Ptsc, double min_dxy2,
                     double beta_n, double max_nxy) {
    F2 dtVx(dtVx_), dtVy(dtVy_), dtPt(dtPt_), M(Must_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= M.n2; ++iy)
        for (int64_t ix = 1; ix <= M.n1; ++ix) {
            if (ix <= dtVx.n1 && iy <= dtVx.n2)
                dtVx(ix, iy) = 1.0 / 4.1 / Vsc * min_dxy2 / ((M(ix, iy + 1) + M(ix + 1, iy + 1)) * 0.5) / (1.0 + beta_n);
            if (ix <= dtVy.n1 && iy <= dtVy.n2)
                dtVy(ix, iy) = 1.0 / 4.1 / Vsc * min_dxy2 / ((M(ix + 1, iy) + M(ix + 1, iy + 1)) * 0.5) / (1.0 + beta_n);
            dtPt(ix, iy) = 4.1 * (1.0 + beta_n) / Ptsc / max_nxy * M(ix, iy);
        }
}

// compute_P! (Stokes2D_ve0.jl:41-45, Stokes2D0.jl:33-37): ∇V, Pt -= dτPt*∇V
void ora2d_compute_P(oarr divV_, oarr Pt_, oarr Vx_, oarr Vy_, oarr dtPt_, double dx, double dy) {
    F2 divV(divV_), Pt(Pt_), Vx(Vx_), Vy(Vy_), dtPt(dtPt_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Pt.n2; ++iy)
        for (int64_t ix = 1; ix <= Pt.n1; ++ix) {
            divV(ix, iy) = (Vx(ix + 1, iy) - Vx(ix, iy)) / dx + (Vy(ix, iy + 1) - Vy(ix, iy)) / dy;
            Pt(ix, iy) = Pt(ix, iy) - dtPt(ix, iy) * divV(ix, iy);
        }
}

// compute_τ! viscous (Stokes2D0.jl:39-44) and Maxwell (Stokes2D_ve0.jl:47-54, Xsi = Mus/(G*dt)):
//   τ = τ_o*Xsi/(Xsi+1) + 2Mus/(Xsi+1)*(ε̇ - ∇V/3 + β_n ∇V)  [elastic]   τ = 2Mus*(ε̇ - ∇V/3 + β_n ∇V)
void ora2d_compute_tau(oarr txx_, oarr tyy_, oarr txy_, oarr txxo_, oarr tyyo_, oarr txyo_, oarr Vx_, oarr Vy_,
                       oarr Mus_, oarr divV_, double G, double dt, double beta_n, double dx, double dy, int elastic) {
    F2 txx(txx_), tyy(tyy_), txy(txy_), Vx(Vx_), Vy(Vy_), M(Mus_), dv(divV_);
    const bool el = elastic != 0;
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= txx.n2; ++iy)
        for (int64_t ix = 1; ix <= txx.n1; ++ix) {
            const double exx = (Vx(ix + 1, iy) - Vx(ix, iy)) / dx - 1.0 / 3.0 * dv(ix, iy) + beta_n * dv(ix, iy);
            const double eyy = (Vy(ix, iy + 1) - Vy(ix, iy)) / dy - 1.0 / 3.0 * dv(ix, iy) + beta_n * dv(ix, iy);
            if (el) {
                const F2 txxo(txxo_), tyyo(tyyo_);
                const double X = M(ix, iy) / (G * dt);
                txx(ix, iy) = txxo(ix, iy) * X / (X + 1.0) + 2.0 * M(ix, iy) / (X + 1.0) * exx;
                tyy(ix, iy) = tyyo(ix, iy) * X / (X + 1.0) + 2.0 * M(ix, iy) / (X + 1.0) * eyy;
            } else {
                txx(ix, iy) = 2.0 * M(ix, iy) * exx;
                tyy(ix, iy) = 2.0 * M(ix, iy) * eyy;
            }
            if (ix <= txy.n1 && iy <= txy.n2) {
                const double am = (M(ix, iy) + M(ix + 1, iy) + M(ix, iy + 1) + M(ix + 1, iy + 1)) * 0.25;
                const double exy = 0.5 * ((Vx(ix + 1, iy + 1) - Vx(ix + 1, iy)) / dy + (Vy(ix + 1, iy + 1) - Vy(ix, iy + 1)) / dx);
                if (el) {
                    const F2 txyo(txyo_);
                    const double X = am / (G * dt);
                    txy(ix, iy) = txyo(ix, iy) * X / (X + 1.0) + 2.0 * am / (X + 1.0) * exy;
                } else {
                    txy(ix, iy) = 2.0 * am * exy;
                }
            }
        }
}

// compute_dV! (Stokes2D_ve0.jl:56-62, Stokes2D0.jl:46-52): R as in Stokes2D.jl, dV/dτ = damp*dV/dτ + R
void ora2d_compute_dV(oarr Rx_, oarr Ry_, oarr dVx_, oarr dVy_, oarr Pt_, oarr txx_, oarr tyy_, oarr txy_, double dampX,
                      double dampY, double dx, double dy) {
    F2 Rx(Rx_), Ry(Ry_), dVx(dVx_), dVy(dVy_), Pt(Pt_), txx(txx_), tyy(tyy_), txy(txy_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Ry.n2; ++iy)
        for (int64_t ix = 1; ix <= Rx.n1; ++ix) {
            if (ix <= Rx.n1 && iy <= Rx.n2) {
                Rx(ix, iy) = (txx(ix + 1, iy + 1) - txx(ix, iy + 1)) / dx + (txy(ix, iy + 1) - txy(ix, iy)) / dy -
                             (Pt(ix + 1, iy + 1) - Pt(ix, iy + 1)) / dx;
                dVx(ix, iy) = dampX * dVx(ix, iy) + Rx(ix, iy);
            }
            if (ix <= Ry.n1 && iy <= Ry.n2) {
                Ry(ix, iy) = (tyy(ix + 1, iy + 1) - tyy(ix + 1, iy)) / dy + (txy(ix + 1, iy) - txy(ix, iy)) / dx -
                             (Pt(ix + 1, iy + 1) - Pt(ix + 1, iy)) / dy;
                dVy(ix, iy) = dampY * dVy(ix, iy) + Ry(ix, iy);
            }
        }
}

// compute_V! (Stokes2D_ve0.jl:64-68, Stokes2D0.jl:54-58): @inn(V) += dτV*dV/dτ
void ora2d_compute_V(oarr Vx_, oarr Vy_, oarr dVx_, oarr dVy_, oarr dtVx_, oarr dtVy_) {
    F2 Vx(Vx_), Vy(Vy_), dVx(dVx_), dVy(dVy_), dtVx(dtVx_), dtVy(dtVy_);
#pragma omp parallel for schedule(static)
    for (int64_t iy = 1; iy <= Vy.n2 - 2; ++iy)
        for (int64_t ix = 1; ix <= Vx.n1 - 2; ++ix) {
            if (ix <= dVx.n1 && iy <= dVx.n2) Vx(ix + 1, iy + 1) = Vx(ix + 1, iy + 1) + dtVx(ix, iy) * dVx(ix, iy);
            if (ix <= dVy.n1 && iy <= dVy.n2) Vy(ix + 1, iy + 1) = Vy(ix + 1, iy + 1) + dtVy(ix, iy) * dVy(ix, iy);
        }
}

// ---------------------------------------------------------------- 3D set-up kernels

// smooth! (Stokes3D_ve_perf.jl:24-27): @inn(A2) = @inn(A) + 1.0/6.1/fact*(@d2_xi(A) + @d2_yi(A) + @d2_zi(A))
void ora3_smooth(oarr A2_, oarr A_, double fact) {
    F3 A2(A2_), A(A_);
    const double c = 1.0 / 6.1 / fact;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= A2.n3 - 2; ++iz)
        for (int64_t iy = 1; iy <= A2.n2 - 2; ++iy)
            for (int64_t ix = 1; ix <= A2.n1 - 2; ++ix) {
                const int64_t i = ix + 1, j = iy + 1, k = iz + 1;
                const double d2x = (A(i + 1, j, k) - A(i, j, k)) - (A(i, j, k) - A(i - 1, j, k));
                const double d2y = (A(i, j + 1, k) - A(i, j, k)) - (A(i, j, k) - A(i, j - 1, k));
                const double d2z = (A(i, j, k + 1) - A(i, j, k)) - (A(i, j, k) - A(i, j, k - 1));
                A2(i, j, k) = A(i, j, k) + c * (d2x + d2y + d2z);
            }
}

// compute_maxloc! (Stokes3D_ve_perf.jl:29-32): max over the point and its six axis neighbours.
void ora3_maxloc(oarr B_, oarr A_) {
    F3 B(B_), A(A_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= B.n3 - 2; ++iz)
        for (int64_t iy = 1; iy <= B.n2 - 2; ++iy)
            for (int64_t ix = 1; ix <= B.n1 - 2; ++ix) {
                const int64_t i = ix + 1, j = iy + 1, k = iz + 1;
                B(i, j, k) = std::max(
                    std::max(std::max(std::max(std::max(std::max(A(i - 1, j, k), A(i + 1, j, k)), A(i, j, k)),
                                               A(i, j - 1, k)),
                                      A(i, j + 1, k)),
                             A(i, j, k - 1)),
                    A(i, j, k + 1));
            }
}

// bc_x! / bc_y! / bc_z! (Stokes3D_ve_perf.jl:98-114)
void ora3_bc_x(oarr A_) {
    F3 A(A_);
    for (int64_t iz = 1; iz <= A.n3; ++iz)
        for (int64_t iy = 1; iy <= A.n2; ++iy) {
            A(1, iy, iz) = A(2, iy, iz);
            A(A.n1, iy, iz) = A(A.n1 - 1, iy, iz);
        }
}
void ora3_bc_y(oarr A_) {
    F3 A(A_);
    for (int64_t iz = 1; iz <= A.n3; ++iz)
        for (int64_t ix = 1; ix <= A.n1; ++ix) {
            A(ix, 1, iz) = A(ix, 2, iz);
            A(ix, A.n2, iz) = A(ix, A.n2 - 1, iz);
        }
}
void ora3_bc_z(oarr A_) {
    F3 A(A_);
    for (int64_t iy = 1; iy <= A.n2; ++iy)
        for (int64_t ix = 1; ix <= A.n1; ++ix) {
            A(ix, iy, 1) = A(ix, iy, 2);
            A(ix, iy, A.n3) = A(ix, iy, A.n3 - 1);
        }
}

// ---------------------------------------------------------------- 3D VE, macro form (Stokes3D_ve_multixpu.jl)

// compute_P! (Stokes3D_ve_multixpu.jl:57-61)
void ora3m_compute_P(oarr divV_, oarr Pt_, oarr Vx_, oarr Vy_, oarr Vz_, oarr Gdt_, double r, double dx, double dy,
                     double dz) {
    F3 divV(divV_), Pt(Pt_), Vx(Vx_), Vy(Vy_), Vz(Vz_), Gdt(Gdt_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= Pt.n3; ++iz)
        for (int64_t iy = 1; iy <= Pt.n2; ++iy)
            for (int64_t ix = 1; ix <= Pt.n1; ++ix) {
                divV(ix, iy, iz) = (Vx(ix + 1, iy, iz) - Vx(ix, iy, iz)) / dx + (Vy(ix, iy + 1, iz) - Vy(ix, iy, iz)) / dy +
                                   (Vz(ix, iy, iz + 1) - Vz(ix, iy, iz)) / dz;
                Pt(ix, iy, iz) = Pt(ix, iy, iz) - r * Gdt(ix, iy, iz) * divV(ix, iy, iz);
            }
}

// compute_τ! (Stokes3D_ve_multixpu.jl:63-77). With elastic=0 the τ_o and Gr terms are
// dropped (the 3D viscous operator, which the reference has only in 2D: Stokes2D.jl:39-44).
static inline double tau_normal_div(double t, double to, double g, double m, double gdt, double d, double h,
                                    bool elastic) {
    // (τ + τ_o*Gr + 2.0*Gdτ*(d/h)) / (1.0 + Gdτ/Mus + Gr)
    if (elastic) {
        const double Gr = g / gdt;
        return (t + to * Gr + 2.0 * g * (d / h)) / (1.0 + g / m + Gr);
    }
    return (t + 2.0 * g * (d / h)) / (1.0 + g / m);
}
static inline double tau_shear_div(double t, double to, double avg, double avm, double gdt, double d1, double h1,
                                   double d2, double h2, bool elastic) {
    // (τ + τ_o*av_Gr + 2.0*av(Gdτ)*(0.5*(d1/h1 + d2/h2))) / (1.0 + av(Gdτ)/av(Mus) + av_Gr)
    if (elastic) {
        const double Gr = avg / gdt;
        return (t + to * Gr + 2.0 * avg * (0.5 * (d1 / h1 + d2 / h2))) / (1.0 + avg / avm + Gr);
    }
    return (t + 2.0 * avg * (0.5 * (d1 / h1 + d2 / h2))) / (1.0 + avg / avm);
}

void ora3m_compute_tau(oarr txx_, oarr tyy_, oarr tzz_, oarr txy_, oarr txz_, oarr tyz_, oarr txxo_, oarr tyyo_,
                       oarr tzzo_, oarr txyo_, oarr txzo_, oarr tyzo_, oarr Vx_, oarr Vy_, oarr Vz_, oarr Mus_,
                       oarr Gdt_, double G, double dt, double dx, double dy, double dz, int elastic) {
    F3 txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_), Vx(Vx_), Vy(Vy_), Vz(Vz_), M(Mus_), Gd(Gdt_);
    const bool el = elastic != 0;
    const double gdt = G * dt;
    auto TO = [&](const oarr& a, int64_t i, int64_t j, int64_t k) -> double {
        return el ? F3(a)(i, j, k) : 0.0;
    };
    const int64_t nx = Gd.n1, ny = Gd.n2, nz = Gd.n3;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= nz; ++iz)
        for (int64_t iy = 1; iy <= ny; ++iy)
            for (int64_t ix = 1; ix <= nx; ++ix) {
                const int64_t ixi = ix + 1, iyi = iy + 1, izi = iz + 1;
                if (ix <= txx.n1 && iy <= txx.n2 && iz <= txx.n3)
                    txx(ix, iy, iz) = tau_normal_div(txx(ix, iy, iz), TO(txxo_, ix, iy, iz), Gd(ix, iyi, izi),
                                                     M(ix, iyi, izi), gdt, Vx(ix + 1, iyi, izi) - Vx(ix, iyi, izi), dx, el);
                if (ix <= tyy.n1 && iy <= tyy.n2 && iz <= tyy.n3)
                    tyy(ix, iy, iz) = tau_normal_div(tyy(ix, iy, iz), TO(tyyo_, ix, iy, iz), Gd(ixi, iy, izi),
                                                     M(ixi, iy, izi), gdt, Vy(ixi, iy + 1, izi) - Vy(ixi, iy, izi), dy, el);
                if (ix <= tzz.n1 && iy <= tzz.n2 && iz <= tzz.n3)
                    tzz(ix, iy, iz) = tau_normal_div(tzz(ix, iy, iz), TO(tzzo_, ix, iy, iz), Gd(ixi, iyi, iz),
                                                     M(ixi, iyi, iz), gdt, Vz(ixi, iyi, iz + 1) - Vz(ixi, iyi, iz), dz, el);
                if (ix <= txy.n1 && iy <= txy.n2 && iz <= txy.n3) {
                    const double ag = (Gd(ix, iy, izi) + Gd(ix + 1, iy, izi) + Gd(ix, iy + 1, izi) + Gd(ix + 1, iy + 1, izi)) * 0.25;
                    const double am = (M(ix, iy, izi) + M(ix + 1, iy, izi) + M(ix, iy + 1, izi) + M(ix + 1, iy + 1, izi)) * 0.25;
                    txy(ix, iy, iz) = tau_shear_div(txy(ix, iy, iz), TO(txyo_, ix, iy, iz), ag, am, gdt,
                                                    Vx(ixi, iy + 1, izi) - Vx(ixi, iy, izi), dy,
                                                    Vy(ix + 1, iyi, izi) - Vy(ix, iyi, izi), dx, el);
                }
                if (ix <= txz.n1 && iy <= txz.n2 && iz <= txz.n3) {
                    const double ag = (Gd(ix, iyi, iz) + Gd(ix + 1, iyi, iz) + Gd(ix, iyi, iz + 1) + Gd(ix + 1, iyi, iz + 1)) * 0.25;
                    const double am = (M(ix, iyi, iz) + M(ix + 1, iyi, iz) + M(ix, iyi, iz + 1) + M(ix + 1, iyi, iz + 1)) * 0.25;
                    txz(ix, iy, iz) = tau_shear_div(txz(ix, iy, iz), TO(txzo_, ix, iy, iz), ag, am, gdt,
                                                    Vx(ixi, iyi, iz + 1) - Vx(ixi, iyi, iz), dz,
                                                    Vz(ix + 1, iyi, izi) - Vz(ix, iyi, izi), dx, el);
                }
                if (ix <= tyz.n1 && iy <= tyz.n2 && iz <= tyz.n3) {
                    const double ag = (Gd(ixi, iy, iz) + Gd(ixi, iy + 1, iz) + Gd(ixi, iy, iz + 1) + Gd(ixi, iy + 1, iz + 1)) * 0.25;
                    const double am = (M(ixi, iy, iz) + M(ixi, iy + 1, iz) + M(ixi, iy, iz + 1) + M(ixi, iy + 1, iz + 1)) * 0.25;
                    tyz(ix, iy, iz) = tau_shear_div(tyz(ix, iy, iz), TO(tyzo_, ix, iy, iz), ag, am, gdt,
                                                    Vy(ixi, iyi, iz + 1) - Vy(ixi, iyi, iz), dz,
                                                    Vz(ixi, iy + 1, izi) - Vz(ixi, iy, izi), dy, el);
                }
            }
}

// compute_dV! (Stokes3D_ve_multixpu.jl:79-84) when store_dV, else compute_Res!
// (Stokes3D_ve_multixpu.jl:93-98): the same momentum residual, without / with the
// @av_xi(dτ_Rho) factor.
void ora3m_compute_dV(oarr dVx_, oarr dVy_, oarr dVz_, oarr Pt_, oarr txx_, oarr tyy_, oarr tzz_, oarr txy_,
                      oarr txz_, oarr tyz_, oarr dtRho_, double dx, double dy, double dz, int residual_only) {
    F3 dVx(dVx_), dVy(dVy_), dVz(dVz_), Pt(Pt_), txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_);
    const bool res = residual_only != 0;
    const int64_t nx = Pt.n1, ny = Pt.n2, nz = Pt.n3;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= nz; ++iz)
        for (int64_t iy = 1; iy <= ny; ++iy)
            for (int64_t ix = 1; ix <= nx; ++ix) {
                const int64_t ixi = ix + 1, iyi = iy + 1, izi = iz + 1;
                if (ix <= dVx.n1 && iy <= dVx.n2 && iz <= dVx.n3) {
                    const double R = (txx(ix + 1, iy, iz) - txx(ix, iy, iz)) / dx + (txy(ix, iy + 1, iz) - txy(ix, iy, iz)) / dy +
                                     (txz(ix, iy, iz + 1) - txz(ix, iy, iz)) / dz - (Pt(ix + 1, iyi, izi) - Pt(ix, iyi, izi)) / dx;
                    if (res) dVx(ix, iy, iz) = R;
                    else {
                        F3 d(dtRho_);
                        dVx(ix, iy, iz) = R * ((d(ix, iyi, izi) + d(ix + 1, iyi, izi)) * 0.5);
                    }
                }
                if (ix <= dVy.n1 && iy <= dVy.n2 && iz <= dVy.n3) {
                    const double R = (tyy(ix, iy + 1, iz) - tyy(ix, iy, iz)) / dy + (txy(ix + 1, iy, iz) - txy(ix, iy, iz)) / dx +
                                     (tyz(ix, iy, iz + 1) - tyz(ix, iy, iz)) / dz - (Pt(ixi, iy + 1, izi) - Pt(ixi, iy, izi)) / dy;
                    if (res) dVy(ix, iy, iz) = R;
                    else {
                        F3 d(dtRho_);
                        dVy(ix, iy, iz) = R * ((d(ixi, iy, izi) + d(ixi, iy + 1, izi)) * 0.5);
                    }
                }
                if (ix <= dVz.n1 && iy <= dVz.n2 && iz <= dVz.n3) {
                    const double R = (tzz(ix, iy, iz + 1) - tzz(ix, iy, iz)) / dz + (txz(ix + 1, iy, iz) - txz(ix, iy, iz)) / dx +
                                     (tyz(ix, iy + 1, iz) - tyz(ix, iy, iz)) / dy - (Pt(ixi, iyi, iz + 1) - Pt(ixi, iyi, iz)) / dz;
                    if (res) dVz(ix, iy, iz) = R;
                    else {
                        F3 d(dtRho_);
                        dVz(ix, iy, iz) = R * ((d(ixi, iyi, iz) + d(ixi, iyi, iz + 1)) * 0.5);
                    }
                }
            }
}

// compute_V! (Stokes3D_ve_multixpu.jl:86-91): @inn(V) = @inn(V) + @all(dV)
void ora3_compute_V(oarr Vx_, oarr Vy_, oarr Vz_, oarr dVx_, oarr dVy_, oarr dVz_) {
    F3 Vx(Vx_), Vy(Vy_), Vz(Vz_), dVx(dVx_), dVy(dVy_), dVz(dVz_);
    const int64_t n3 = std::max(dVx.n3, std::max(dVy.n3, dVz.n3));
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= n3; ++iz)
        for (int64_t iy = 1; iy <= std::max(dVx.n2, std::max(dVy.n2, dVz.n2)); ++iy)
            for (int64_t ix = 1; ix <= std::max(dVx.n1, std::max(dVy.n1, dVz.n1)); ++ix) {
                if (ix <= dVx.n1 && iy <= dVx.n2 && iz <= dVx.n3) Vx(ix + 1, iy + 1, iz + 1) = Vx(ix + 1, iy + 1, iz + 1) + dVx(ix, iy, iz);
                if (ix <= dVy.n1 && iy <= dVy.n2 && iz <= dVy.n3) Vy(ix + 1, iy + 1, iz + 1) = Vy(ix + 1, iy + 1, iz + 1) + dVy(ix, iy, iz);
                if (ix <= dVz.n1 && iy <= dVz.n2 && iz <= dVz.n3) Vz(ix + 1, iy + 1, iz + 1) = Vz(ix + 1, iy + 1, iz + 1) + dVz(ix, iy, iz);
            }
}

// ---------------------------------------------------------------- 3D damped scheme (viscous)
// scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl on one rank: the "accel. 1" scheme
// of the 2D damped scripts in 3D.

// compute_timesteps! (Stokes3D0_multixpu.jl:37-43); note the 3D order 1/6.1/(1+β_n)/Vsc*…
void ora3d_timesteps(oarr dtVx_, oarr dtVy_, oarr dtVz_, oarr dtPt_, oarr Must_, double Vsc, double Ptsc,
                     double min_dxyz2, double beta_n, double max_nxyz) {
    F3 dtVx(dtVx_), dtVy(dtVy_), dtVz(dtVz_), dtPt(dtPt_), M(Must_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= M.n3; ++iz)
        for (int64_t iy = 1; iy <= M.n2; ++iy)
            for (int64_t ix = 1; ix <= M.n1; ++ix) {
                const double c = 1.0 / 6.1 / (1.0 + beta_n) / Vsc * min_dxyz2;
                if (ix <= dtVx.n1 && iy <= dtVx.n2 && iz <= dtVx.n3)
                    dtVx(ix, iy, iz) = c / ((M(ix, iy + 1, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.5);
                if (ix <= dtVy.n1 && iy <= dtVy.n2 && iz <= dtVy.n3)
                    dtVy(ix, iy, iz) = c / ((M(ix + 1, iy, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.5);
                if (ix <= dtVz.n1 && iy <= dtVz.n2 && iz <= dtVz.n3)
                    dtVz(ix, iy, iz) = c / ((M(ix + 1, iy + 1, iz) + M(ix + 1, iy + 1, iz + 1)) * 0.5);
                dtPt(ix, iy, iz) = 6.1 * (1.0 + beta_n) / Ptsc / max_nxyz * M(ix, iy, iz);
            }
}

// compute_P! (Stokes3D0_multixpu.jl:45-49): ∇V, Pt = Pt - dτPt*∇V
void ora3d_compute_P(oarr divV_, oarr Pt_, oarr Vx_, oarr Vy_, oarr Vz_, oarr dtPt_, double dx, double dy, double dz) {
    F3 divV(divV_), Pt(Pt_), Vx(Vx_), Vy(Vy_), Vz(Vz_), dtPt(dtPt_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= Pt.n3; ++iz)
        for (int64_t iy = 1; iy <= Pt.n2; ++iy)
            for (int64_t ix = 1; ix <= Pt.n1; ++ix) {
                divV(ix, iy, iz) = (Vx(ix + 1, iy, iz) - Vx(ix, iy, iz)) / dx + (Vy(ix, iy + 1, iz) - Vy(ix, iy, iz)) / dy +
                                   (Vz(ix, iy, iz + 1) - Vz(ix, iy, iz)) / dz;
                Pt(ix, iy, iz) = Pt(ix, iy, iz) - dtPt(ix, iy, iz) * divV(ix, iy, iz);
            }
}

// compute_τ! (Stokes3D0_multixpu.jl:51-59):
//   τxx = 2@inn_yz(Mus)*(@d_xi(Vx)/dx - 1/3*@inn_yz(∇V) + β_n*@inn_yz(∇V)),
//   τxy = 2@av_xyi(Mus)*(0.5*(@d_yi(Vx)/dy + @d_xi(Vy)/dx)), ...
void ora3d_compute_tau(oarr divV_, oarr txx_, oarr tyy_, oarr tzz_, oarr txy_, oarr txz_, oarr tyz_, oarr Vx_,
                       oarr Vy_, oarr Vz_, oarr Mus_, double beta_n, double dx, double dy, double dz) {
    F3 dv(divV_), txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_), Vx(Vx_), Vy(Vy_), Vz(Vz_), M(Mus_);
    const int64_t nx = M.n1, ny = M.n2, nz = M.n3;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= nz; ++iz)
        for (int64_t iy = 1; iy <= ny; ++iy)
            for (int64_t ix = 1; ix <= nx; ++ix) {
                const int64_t ixi = ix + 1, iyi = iy + 1, izi = iz + 1;
                if (ix <= txx.n1 && iy <= txx.n2 && iz <= txx.n3) {
                    const double d = dv(ix, iyi, izi);
                    txx(ix, iy, iz) = 2.0 * M(ix, iyi, izi) *
                                      ((Vx(ix + 1, iyi, izi) - Vx(ix, iyi, izi)) / dx - 1.0 / 3.0 * d + beta_n * d);
                }
                if (ix <= tyy.n1 && iy <= tyy.n2 && iz <= tyy.n3) {
                    const double d = dv(ixi, iy, izi);
                    tyy(ix, iy, iz) = 2.0 * M(ixi, iy, izi) *
                                      ((Vy(ixi, iy + 1, izi) - Vy(ixi, iy, izi)) / dy - 1.0 / 3.0 * d + beta_n * d);
                }
                if (ix <= tzz.n1 && iy <= tzz.n2 && iz <= tzz.n3) {
                    const double d = dv(ixi, iyi, iz);
                    tzz(ix, iy, iz) = 2.0 * M(ixi, iyi, iz) *
                                      ((Vz(ixi, iyi, iz + 1) - Vz(ixi, iyi, iz)) / dz - 1.0 / 3.0 * d + beta_n * d);
                }
                if (ix <= txy.n1 && iy <= txy.n2 && iz <= txy.n3) {
                    const double am = (M(ix, iy, izi) + M(ix + 1, iy, izi) + M(ix, iy + 1, izi) + M(ix + 1, iy + 1, izi)) * 0.25;
                    txy(ix, iy, iz) = 2.0 * am * (0.5 * ((Vx(ixi, iy + 1, izi) - Vx(ixi, iy, izi)) / dy +
                                                         (Vy(ix + 1, iyi, izi) - Vy(ix, iyi, izi)) / dx));
                }
                if (ix <= txz.n1 && iy <= txz.n2 && iz <= txz.n3) {
                    const double am = (M(ix, iyi, iz) + M(ix + 1, iyi, iz) + M(ix, iyi, iz + 1) + M(ix + 1, iyi, iz + 1)) * 0.25;
                    txz(ix, iy, iz) = 2.0 * am * (0.5 * ((Vx(ixi, iyi, iz + 1) - Vx(ixi, iyi, iz)) / dz +
                                                         (Vz(ix + 1, iyi, izi) - Vz(ix, iyi, izi)) / dx));
                }
                if (ix <= tyz.n1 && iy <= tyz.n2 && iz <= tyz.n3) {
                    const double am = (M(ixi, iy, iz) + M(ixi, iy + 1, iz) + M(ixi, iy, iz + 1) + M(ixi, iy + 1, iz + 1)) * 0.25;
                    tyz(ix, iy, iz) = 2.0 * am * (0.5 * ((Vy(ixi, iyi, iz + 1) - Vy(ixi, iyi, iz)) / dz +
                                                         (Vz(ixi, iy + 1, izi) - Vz(ixi, iy, izi)) / dy));
                }
            }
}

// compute_dV! (Stokes3D0_multixpu.jl:61-69): R as compute_dV! of Stokes3D_ve_multixpu.jl,
// dV/dτ = damp*dV/dτ + R
void ora3d_compute_dV(oarr Rx_, oarr Ry_, oarr Rz_, oarr dVx_, oarr dVy_, oarr dVz_, oarr Pt_, oarr txx_, oarr tyy_,
                      oarr tzz_, oarr txy_, oarr txz_, oarr tyz_, double dampX, double dampY, double dampZ, double dx,
                      double dy, double dz) {
    ora3m_compute_dV(Rx_, Ry_, Rz_, Pt_, txx_, tyy_, tzz_, txy_, txz_, tyz_, oarr{nullptr, 0, 0, 0}, dx, dy, dz, 1);
    F3 Rx(Rx_), Ry(Ry_), Rz(Rz_), dVx(dVx_), dVy(dVy_), dVz(dVz_);
    const int64_t n = Rx.n1 * Rx.n2 * Rx.n3, m = Ry.n1 * Ry.n2 * Ry.n3, l = Rz.n1 * Rz.n2 * Rz.n3;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; ++q) dVx.p[q] = dampX * dVx.p[q] + Rx.p[q];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < m; ++q) dVy.p[q] = dampY * dVy.p[q] + Ry.p[q];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < l; ++q) dVz.p[q] = dampZ * dVz.p[q] + Rz.p[q];
}

// compute_V! (Stokes3D0_multixpu.jl:71-76): @inn(V) = @inn(V) + dτV*dV/dτ
void ora3d_compute_V(oarr Vx_, oarr Vy_, oarr Vz_, oarr dVx_, oarr dVy_, oarr dVz_, oarr dtVx_, oarr dtVy_,
                     oarr dtVz_) {
    F3 Vx(Vx_), Vy(Vy_), Vz(Vz_), dVx(dVx_), dVy(dVy_), dVz(dVz_), tx(dtVx_), ty(dtVy_), tz(dtVz_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= std::max(dVx.n3, dVz.n3); ++iz)
        for (int64_t iy = 1; iy <= std::max(dVx.n2, dVy.n2); ++iy)
            for (int64_t ix = 1; ix <= std::max(dVx.n1, dVy.n1); ++ix) {
                if (ix <= dVx.n1 && iy <= dVx.n2 && iz <= dVx.n3)
                    Vx(ix + 1, iy + 1, iz + 1) = Vx(ix + 1, iy + 1, iz + 1) + tx(ix, iy, iz) * dVx(ix, iy, iz);
                if (ix <= dVy.n1 && iy <= dVy.n2 && iz <= dVy.n3)
                    Vy(ix + 1, iy + 1, iz + 1) = Vy(ix + 1, iy + 1, iz + 1) + ty(ix, iy, iz) * dVy(ix, iy, iz);
                if (ix <= dVz.n1 && iy <= dVz.n2 && iz <= dVz.n3)
                    Vz(ix + 1, iy + 1, iz + 1) = Vz(ix + 1, iy + 1, iz + 1) + tz(ix, iy, iz) * dVz(ix, iy, iz);
            }
}

// ---------------------------------------------------------------- 3D VE explicit-index (Stokes3D_ve_perf.jl)

static inline double tau_normal_mul(double t, double to, double g, double m, double gdt, double _h, double d,
                                    bool elastic) {
    // (τ + τ_o*Gr + 2.0*Gdτ*(_h*d)) / (1.0 + Gdτ/Mus + Gr)   (Stokes3D_ve_perf.jl:71-73)
    if (elastic) {
        const double Gr = g / gdt;
        return (t + to * Gr + 2.0 * g * (_h * d)) / (1.0 + g / m + Gr);
    }
    return (t + 2.0 * g * (_h * d)) / (1.0 + g / m);
}
static inline double tau_shear_mul(double t, double to, double avg, double avm, double gdt, double _h1, double d1,
                                   double _h2, double d2, bool elastic) {
    // (τ + τ_o*av_Gr + 2.0*av_Gdτ*(0.5*(_h1*d1 + _h2*d2))) / (1.0 + av_Gdτ/av_Mus + av_Gr)  (:74-76)
    if (elastic) {
        const double Gr = avg / gdt;
        return (t + to * Gr + 2.0 * avg * (0.5 * (_h1 * d1 + _h2 * d2))) / (1.0 + avg / avm + Gr);
    }
    return (t + 2.0 * avg * (0.5 * (_h1 * d1 + _h2 * d2))) / (1.0 + avg / avm);
}

// compute_Pt_τ! (Stokes3D_ve_perf.jl:69-78). elastic=0 gives the 3D viscous operator.
void ora3p_compute_Pt_tau(oarr Pt_, oarr txx_, oarr tyy_, oarr tzz_, oarr txy_, oarr txz_, oarr tyz_, oarr txxo_,
                          oarr tyyo_, oarr tzzo_, oarr txyo_, oarr txzo_, oarr tyzo_, oarr Vx_, oarr Vy_, oarr Vz_,
                          oarr Mus_, oarr Gdt_, double r, double G, double dt, double _dx, double _dy, double _dz,
                          int elastic) {
    F3 Pt(Pt_), txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_), Vx(Vx_), Vy(Vy_), Vz(Vz_), M(Mus_),
        Gd(Gdt_);
    const bool el = elastic != 0;
    const double gdt = G * dt;
    auto TO = [&](const oarr& a, int64_t i, int64_t j, int64_t k) -> double { return el ? F3(a)(i, j, k) : 0.0; };
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= Pt.n3; ++iz)
        for (int64_t iy = 1; iy <= Pt.n2; ++iy)
            for (int64_t ix = 1; ix <= Pt.n1; ++ix) {
                Pt(ix, iy, iz) = Pt(ix, iy, iz) - r * Gd(ix, iy, iz) *
                                                      (_dx * (Vx(ix + 1, iy, iz) - Vx(ix, iy, iz)) +
                                                       _dy * (Vy(ix, iy + 1, iz) - Vy(ix, iy, iz)) +
                                                       _dz * (Vz(ix, iy, iz + 1) - Vz(ix, iy, iz)));
                if (ix <= txx.n1 && iy <= txx.n2 && iz <= txx.n3)
                    txx(ix, iy, iz) = tau_normal_mul(txx(ix, iy, iz), TO(txxo_, ix, iy, iz), Gd(ix, iy + 1, iz + 1),
                                                     M(ix, iy + 1, iz + 1), gdt, _dx,
                                                     Vx(ix + 1, iy + 1, iz + 1) - Vx(ix, iy + 1, iz + 1), el);
                if (ix <= tyy.n1 && iy <= tyy.n2 && iz <= tyy.n3)
                    tyy(ix, iy, iz) = tau_normal_mul(tyy(ix, iy, iz), TO(tyyo_, ix, iy, iz), Gd(ix + 1, iy, iz + 1),
                                                     M(ix + 1, iy, iz + 1), gdt, _dy,
                                                     Vy(ix + 1, iy + 1, iz + 1) - Vy(ix + 1, iy, iz + 1), el);
                if (ix <= tzz.n1 && iy <= tzz.n2 && iz <= tzz.n3)
                    tzz(ix, iy, iz) = tau_normal_mul(tzz(ix, iy, iz), TO(tzzo_, ix, iy, iz), Gd(ix + 1, iy + 1, iz),
                                                     M(ix + 1, iy + 1, iz), gdt, _dz,
                                                     Vz(ix + 1, iy + 1, iz + 1) - Vz(ix + 1, iy + 1, iz), el);
                if (ix <= txy.n1 && iy <= txy.n2 && iz <= txy.n3) {
                    const double ag = (Gd(ix, iy, iz + 1) + Gd(ix + 1, iy, iz + 1) + Gd(ix, iy + 1, iz + 1) + Gd(ix + 1, iy + 1, iz + 1)) * 0.25;
                    const double am = (M(ix, iy, iz + 1) + M(ix + 1, iy, iz + 1) + M(ix, iy + 1, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.25;
                    txy(ix, iy, iz) = tau_shear_mul(txy(ix, iy, iz), TO(txyo_, ix, iy, iz), ag, am, gdt, _dy,
                                                    Vx(ix + 1, iy + 1, iz + 1) - Vx(ix + 1, iy, iz + 1), _dx,
                                                    Vy(ix + 1, iy + 1, iz + 1) - Vy(ix, iy + 1, iz + 1), el);
                }
                if (ix <= txz.n1 && iy <= txz.n2 && iz <= txz.n3) {
                    const double ag = (Gd(ix, iy + 1, iz) + Gd(ix + 1, iy + 1, iz) + Gd(ix, iy + 1, iz + 1) + Gd(ix + 1, iy + 1, iz + 1)) * 0.25;
                    const double am = (M(ix, iy + 1, iz) + M(ix + 1, iy + 1, iz) + M(ix, iy + 1, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.25;
                    txz(ix, iy, iz) = tau_shear_mul(txz(ix, iy, iz), TO(txzo_, ix, iy, iz), ag, am, gdt, _dz,
                                                    Vx(ix + 1, iy + 1, iz + 1) - Vx(ix + 1, iy + 1, iz), _dx,
                                                    Vz(ix + 1, iy + 1, iz + 1) - Vz(ix, iy + 1, iz + 1), el);
                }
                if (ix <= tyz.n1 && iy <= tyz.n2 && iz <= tyz.n3) {
                    const double ag = (Gd(ix + 1, iy, iz) + Gd(ix + 1, iy + 1, iz) + Gd(ix + 1, iy, iz + 1) + Gd(ix + 1, iy + 1, iz + 1)) * 0.25;
                    const double am = (M(ix + 1, iy, iz) + M(ix + 1, iy + 1, iz) + M(ix + 1, iy, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.25;
                    tyz(ix, iy, iz) = tau_shear_mul(tyz(ix, iy, iz), TO(tyzo_, ix, iy, iz), ag, am, gdt, _dz,
                                                    Vy(ix + 1, iy + 1, iz + 1) - Vy(ix + 1, iy + 1, iz), _dy,
                                                    Vz(ix + 1, iy + 1, iz + 1) - Vz(ix + 1, iy, iz + 1), el);
                }
            }
}

// compute_V! (Stokes3D_ve_perf.jl:80-88)
void ora3p_compute_V(oarr Vx_, oarr Vy_, oarr Vz_, oarr Pt_, oarr txx_, oarr tyy_, oarr tzz_, oarr txy_, oarr txz_,
                     oarr tyz_, oarr dtRho_, double _dx, double _dy, double _dz) {
    F3 Vx(Vx_), Vy(Vy_), Vz(Vz_), Pt(Pt_), txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_), d(dtRho_);
    const int64_t nx = Pt.n1, ny = Pt.n2, nz = Pt.n3;
    const int64_t nx_1 = nx - 1, nx_2 = nx - 2, ny_1 = ny - 1, ny_2 = ny - 2, nz_1 = nz - 1, nz_2 = nz - 2;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= nz_1; ++iz)
        for (int64_t iy = 1; iy <= ny_1; ++iy)
            for (int64_t ix = 1; ix <= nx_1; ++ix) {
                if (ix <= nx_1 && iy <= ny_2 && iz <= nz_2)
                    Vx(ix + 1, iy + 1, iz + 1) =
                        Vx(ix + 1, iy + 1, iz + 1) +
                        (_dx * (txx(ix + 1, iy, iz) - txx(ix, iy, iz)) + _dy * (txy(ix, iy + 1, iz) - txy(ix, iy, iz)) +
                         _dz * (txz(ix, iy, iz + 1) - txz(ix, iy, iz)) - _dx * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix, iy + 1, iz + 1))) *
                            ((d(ix, iy + 1, iz + 1) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                if (ix <= nx_2 && iy <= ny_1 && iz <= nz_2)
                    Vy(ix + 1, iy + 1, iz + 1) =
                        Vy(ix + 1, iy + 1, iz + 1) +
                        (_dy * (tyy(ix, iy + 1, iz) - tyy(ix, iy, iz)) + _dx * (txy(ix + 1, iy, iz) - txy(ix, iy, iz)) +
                         _dz * (tyz(ix, iy, iz + 1) - tyz(ix, iy, iz)) - _dy * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix + 1, iy, iz + 1))) *
                            ((d(ix + 1, iy, iz + 1) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                if (ix <= nx_2 && iy <= ny_2 && iz <= nz_1)
                    Vz(ix + 1, iy + 1, iz + 1) =
                        Vz(ix + 1, iy + 1, iz + 1) +
                        (_dz * (tzz(ix, iy, iz + 1) - tzz(ix, iy, iz)) + _dx * (txz(ix + 1, iy, iz) - txz(ix, iy, iz)) +
                         _dy * (tyz(ix, iy + 1, iz) - tyz(ix, iy, iz)) - _dz * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix + 1, iy + 1, iz))) *
                            ((d(ix + 1, iy + 1, iz) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
            }
}

// compute_V! with momentum sources (adjoint solves; no reference counterpart): as
// ora3p_compute_V with V += (R + F)*@av(dτ_Rho), F on the interior faces (extents of Rx, Ry, Rz).
void ora3p_compute_V_src(oarr Vx_, oarr Vy_, oarr Vz_, oarr Pt_, oarr txx_, oarr tyy_, oarr tzz_, oarr txy_,
                         oarr txz_, oarr tyz_, oarr dtRho_, oarr Fx_, oarr Fy_, oarr Fz_, double _dx, double _dy,
                         double _dz) {
    F3 Vx(Vx_), Vy(Vy_), Vz(Vz_), Pt(Pt_), txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_), d(dtRho_),
        Fx(Fx_), Fy(Fy_), Fz(Fz_);
    const int64_t nx = Pt.n1, ny = Pt.n2, nz = Pt.n3;
    const int64_t nx_1 = nx - 1, nx_2 = nx - 2, ny_1 = ny - 1, ny_2 = ny - 2, nz_1 = nz - 1, nz_2 = nz - 2;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= nz_1; ++iz)
        for (int64_t iy = 1; iy <= ny_1; ++iy)
            for (int64_t ix = 1; ix <= nx_1; ++ix) {
                if (ix <= nx_1 && iy <= ny_2 && iz <= nz_2) {
                    const double R = _dx * (txx(ix + 1, iy, iz) - txx(ix, iy, iz)) + _dy * (txy(ix, iy + 1, iz) - txy(ix, iy, iz)) +
                                     _dz * (txz(ix, iy, iz + 1) - txz(ix, iy, iz)) - _dx * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix, iy + 1, iz + 1));
                    Vx(ix + 1, iy + 1, iz + 1) = Vx(ix + 1, iy + 1, iz + 1) +
                                                 (R + Fx(ix, iy, iz)) * ((d(ix, iy + 1, iz + 1) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                }
                if (ix <= nx_2 && iy <= ny_1 && iz <= nz_2) {
                    const double R = _dy * (tyy(ix, iy + 1, iz) - tyy(ix, iy, iz)) + _dx * (txy(ix + 1, iy, iz) - txy(ix, iy, iz)) +
                                     _dz * (tyz(ix, iy, iz + 1) - tyz(ix, iy, iz)) - _dy * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix + 1, iy, iz + 1));
                    Vy(ix + 1, iy + 1, iz + 1) = Vy(ix + 1, iy + 1, iz + 1) +
                                                 (R + Fy(ix, iy, iz)) * ((d(ix + 1, iy, iz + 1) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                }
                if (ix <= nx_2 && iy <= ny_2 && iz <= nz_1) {
                    const double R = _dz * (tzz(ix, iy, iz + 1) - tzz(ix, iy, iz)) + _dx * (txz(ix + 1, iy, iz) - txz(ix, iy, iz)) +
                                     _dy * (tyz(ix, iy + 1, iz) - tyz(ix, iy, iz)) - _dz * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix + 1, iy + 1, iz));
                    Vz(ix + 1, iy + 1, iz + 1) = Vz(ix + 1, iy + 1, iz + 1) +
                                                 (R + Fz(ix, iy, iz)) * ((d(ix + 1, iy + 1, iz) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                }
            }
}

// τ = 2·Mus·ε̇(V), the fixed point of the viscous compute_Pt_τ! update (explicit-index _dx form;
// shear rates 0.5*(_dy*∂Vx + _dx*∂Vy) with the 4-cell average of Mus as in :57-62).
void ora3v_tau_exact(oarr txx_, oarr tyy_, oarr tzz_, oarr txy_, oarr txz_, oarr tyz_, oarr Vx_, oarr Vy_, oarr Vz_,
                     oarr Mus_, double _dx, double _dy, double _dz) {
    F3 txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_), Vx(Vx_), Vy(Vy_), Vz(Vz_), M(Mus_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= M.n3; ++iz)
        for (int64_t iy = 1; iy <= M.n2; ++iy)
            for (int64_t ix = 1; ix <= M.n1; ++ix) {
                if (ix <= txx.n1 && iy <= txx.n2 && iz <= txx.n3)
                    txx(ix, iy, iz) = 2.0 * M(ix, iy + 1, iz + 1) * (_dx * (Vx(ix + 1, iy + 1, iz + 1) - Vx(ix, iy + 1, iz + 1)));
                if (ix <= tyy.n1 && iy <= tyy.n2 && iz <= tyy.n3)
                    tyy(ix, iy, iz) = 2.0 * M(ix + 1, iy, iz + 1) * (_dy * (Vy(ix + 1, iy + 1, iz + 1) - Vy(ix + 1, iy, iz + 1)));
                if (ix <= tzz.n1 && iy <= tzz.n2 && iz <= tzz.n3)
                    tzz(ix, iy, iz) = 2.0 * M(ix + 1, iy + 1, iz) * (_dz * (Vz(ix + 1, iy + 1, iz + 1) - Vz(ix + 1, iy + 1, iz)));
                if (ix <= txy.n1 && iy <= txy.n2 && iz <= txy.n3) {
                    const double am = (M(ix, iy, iz + 1) + M(ix + 1, iy, iz + 1) + M(ix, iy + 1, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.25;
                    txy(ix, iy, iz) = 2.0 * am * (0.5 * (_dy * (Vx(ix + 1, iy + 1, iz + 1) - Vx(ix + 1, iy, iz + 1)) +
                                                         _dx * (Vy(ix + 1, iy + 1, iz + 1) - Vy(ix, iy + 1, iz + 1))));
                }
                if (ix <= txz.n1 && iy <= txz.n2 && iz <= txz.n3) {
                    const double am = (M(ix, iy + 1, iz) + M(ix + 1, iy + 1, iz) + M(ix, iy + 1, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.25;
                    txz(ix, iy, iz) = 2.0 * am * (0.5 * (_dz * (Vx(ix + 1, iy + 1, iz + 1) - Vx(ix + 1, iy + 1, iz)) +
                                                         _dx * (Vz(ix + 1, iy + 1, iz + 1) - Vz(ix, iy + 1, iz + 1))));
                }
                if (ix <= tyz.n1 && iy <= tyz.n2 && iz <= tyz.n3) {
                    const double am = (M(ix + 1, iy, iz) + M(ix + 1, iy + 1, iz) + M(ix + 1, iy, iz + 1) + M(ix + 1, iy + 1, iz + 1)) * 0.25;
                    tyz(ix, iy, iz) = 2.0 * am * (0.5 * (_dz * (Vy(ix + 1, iy + 1, iz + 1) - Vy(ix + 1, iy + 1, iz)) +
                                                         _dy * (Vz(ix + 1, iy + 1, iz + 1) - Vz(ix + 1, iy, iz + 1))));
                }
            }
}

// Residual of the transposed (adjoint) system at the interior faces of a 3D_V problem (no
// reference counterpart). With B the free-slip extension (ghost faces copy their clamped
// interior face), the adjoint of the momentum rows sums, at each interior face, its own
// residual and those of the ghost faces copying it; a ghost's residual is the interior
// stencil with zero wherever it reaches a stress point that does not exist. Order: own,
// ghosts below/above along the first tangential axis, along the second, then corners.
// Written with 0-based unified coordinates: a field's element (a,b,c) sits at reference
// index (a-s0+1, b-s1+1, c-s2+1) for the field's start (s0,s1,s2) (zero outside its extents).
void ora3v_res_adj(oarr Rx_, oarr Ry_, oarr Rz_, oarr Pt_, oarr txx_, oarr tyy_, oarr tzz_, oarr txy_, oarr txz_,
                   oarr tyz_, double _dx, double _dy, double _dz) {
    F3 Rx(Rx_), Ry(Ry_), Rz(Rz_), P(Pt_), txx(txx_), tyy(tyy_), tzz(tzz_), txy(txy_), txz(txz_), tyz(tyz_);
    const int64_t nx = P.n1, ny = P.n2, nz = P.n3;
    auto T = [](const F3& A, int s0, int s1, int s2, int64_t a, int64_t b, int64_t c) -> double {
        const int64_t u = a - s0 + 1, v = b - s1 + 1, w = c - s2 + 1;
        if (u < 1 || u > A.n1 || v < 1 || v > A.n2 || w < 1 || w > A.n3) return 0.0;
        return A(u, v, w);
    };
    auto rx = [&](int64_t i, int64_t j, int64_t k) {
        return ((_dx * (T(txx, 0, 1, 1, i, j, k) - T(txx, 0, 1, 1, i - 1, j, k)) +
                 _dy * (T(txy, 1, 1, 1, i, j + 1, k) - T(txy, 1, 1, 1, i, j, k))) +
                _dz * (T(txz, 1, 1, 1, i, j, k + 1) - T(txz, 1, 1, 1, i, j, k))) -
               _dx * (T(P, 0, 0, 0, i, j, k) - T(P, 0, 0, 0, i - 1, j, k));
    };
    auto ry = [&](int64_t i, int64_t j, int64_t k) {
        return ((_dy * (T(tyy, 1, 0, 1, i, j, k) - T(tyy, 1, 0, 1, i, j - 1, k)) +
                 _dx * (T(txy, 1, 1, 1, i + 1, j, k) - T(txy, 1, 1, 1, i, j, k))) +
                _dz * (T(tyz, 1, 1, 1, i, j, k + 1) - T(tyz, 1, 1, 1, i, j, k))) -
               _dy * (T(P, 0, 0, 0, i, j, k) - T(P, 0, 0, 0, i, j - 1, k));
    };
    auto rz = [&](int64_t i, int64_t j, int64_t k) {
        return ((_dz * (T(tzz, 1, 1, 0, i, j, k) - T(tzz, 1, 1, 0, i, j, k - 1)) +
                 _dx * (T(txz, 1, 1, 1, i + 1, j, k) - T(txz, 1, 1, 1, i, j, k))) +
                _dy * (T(tyz, 1, 1, 1, i, j + 1, k) - T(tyz, 1, 1, 1, i, j, k))) -
               _dz * (T(P, 0, 0, 0, i, j, k) - T(P, 0, 0, 0, i, j, k - 1));
    };
    // fold over (a, b): the two tangential coordinates with interior range [1, ahi] x [1, bhi]
    auto fold = [](auto&& at, int64_t a, int64_t b, int64_t ahi, int64_t bhi) {
        const int64_t ga0 = (a == 1) ? 0 : -1, ga1 = (a == ahi) ? ahi + 1 : -1;
        const int64_t gb0 = (b == 1) ? 0 : -1, gb1 = (b == bhi) ? bhi + 1 : -1;
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
    };
#pragma omp parallel for schedule(static)
    for (int64_t k = 1; k <= nz - 1; ++k)
        for (int64_t j = 1; j <= ny - 1; ++j)
            for (int64_t i = 1; i <= nx - 1; ++i) {
                if (j <= ny - 2 && k <= nz - 2)
                    Rx(i, j, k) = fold([&](int64_t a, int64_t b) { return rx(i, a, b); }, j, k, ny - 2, nz - 2);
                if (i <= nx - 2 && k <= nz - 2)
                    Ry(i, j, k) = fold([&](int64_t a, int64_t b) { return ry(a, j, b); }, i, k, nx - 2, nz - 2);
                if (i <= nx - 2 && j <= ny - 2)
                    Rz(i, j, k) = fold([&](int64_t a, int64_t b) { return rz(a, b, k); }, i, j, nx - 2, ny - 2);
            }
}

// V += (R + F)*@av(dτ_Rho) on the interior faces from given residuals (the adjoint-mode V
// update; no free-slip copies). R and F have the extents of Rx, Ry, Rz.
void ora3v_update_V(oarr Vx_, oarr Vy_, oarr Vz_, oarr Rx_, oarr Ry_, oarr Rz_, oarr Fx_, oarr Fy_, oarr Fz_,
                    oarr dtRho_) {
    F3 Vx(Vx_), Vy(Vy_), Vz(Vz_), Rx(Rx_), Ry(Ry_), Rz(Rz_), Fx(Fx_), Fy(Fy_), Fz(Fz_), d(dtRho_);
    const int64_t nx = d.n1, ny = d.n2, nz = d.n3;
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= nz - 1; ++iz)
        for (int64_t iy = 1; iy <= ny - 1; ++iy)
            for (int64_t ix = 1; ix <= nx - 1; ++ix) {
                if (iy <= ny - 2 && iz <= nz - 2)
                    Vx(ix + 1, iy + 1, iz + 1) = Vx(ix + 1, iy + 1, iz + 1) +
                                                 (Rx(ix, iy, iz) + Fx(ix, iy, iz)) * ((d(ix, iy + 1, iz + 1) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                if (ix <= nx - 2 && iz <= nz - 2)
                    Vy(ix + 1, iy + 1, iz + 1) = Vy(ix + 1, iy + 1, iz + 1) +
                                                 (Ry(ix, iy, iz) + Fy(ix, iy, iz)) * ((d(ix + 1, iy, iz + 1) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
                if (ix <= nx - 2 && iy <= ny - 2)
                    Vz(ix + 1, iy + 1, iz + 1) = Vz(ix + 1, iy + 1, iz + 1) +
                                                 (Rz(ix, iy, iz) + Fz(ix, iy, iz)) * ((d(ix + 1, iy + 1, iz) + d(ix + 1, iy + 1, iz + 1)) * 0.5);
            }
}

// ∂J/∂log μ per cell for the 3D viscous operator (no reference counterpart), from the forward
// velocity V and the adjoint velocity L (the transposed system's solution, zero ghosts):
//   g_c = -Mus_c (2 Σ_n ε̇_n(V) ε̇_n(L) + Σ_{edges around c} ε̇_s(V) ε̇_s(L)),
// normal rates on the cells where compute_τ! updates them, shear rates on the interior edges
// (each averaging 4 cells). Written with 0-based cell coordinates (i,j,k); a face or edge
// takes the coordinates of the cell above it.
void ora3v_grad_logmu(oarr grad_, oarr Vx_, oarr Vy_, oarr Vz_, oarr Lx_, oarr Ly_, oarr Lz_, oarr Mus_, double _dx,
                      double _dy, double _dz) {
    F3 G(grad_), Vx(Vx_), Vy(Vy_), Vz(Vz_), Lx(Lx_), Ly(Ly_), Lz(Lz_), M(Mus_);
    const int64_t nx = M.n1, ny = M.n2, nz = M.n3;
    auto at = [](const F3& A, int64_t i, int64_t j, int64_t k) { return A(i + 1, j + 1, k + 1); };
    auto rxy = [&](const F3& X, const F3& Y, int64_t i, int64_t j, int64_t k) {
        return 0.5 * (_dy * (at(X, i, j, k) - at(X, i, j - 1, k)) + _dx * (at(Y, i, j, k) - at(Y, i - 1, j, k)));
    };
    auto rxz = [&](const F3& X, const F3& Z, int64_t i, int64_t j, int64_t k) {
        return 0.5 * (_dz * (at(X, i, j, k) - at(X, i, j, k - 1)) + _dx * (at(Z, i, j, k) - at(Z, i - 1, j, k)));
    };
    auto ryz = [&](const F3& Y, const F3& Z, int64_t i, int64_t j, int64_t k) {
        return 0.5 * (_dz * (at(Y, i, j, k) - at(Y, i, j, k - 1)) + _dy * (at(Z, i, j, k) - at(Z, i, j - 1, k)));
    };
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                double nrm = 0.0, shr = 0.0;
                if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
                    nrm = nrm + (_dx * (at(Vx, i + 1, j, k) - at(Vx, i, j, k))) * (_dx * (at(Lx, i + 1, j, k) - at(Lx, i, j, k)));
                if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
                    nrm = nrm + (_dy * (at(Vy, i, j + 1, k) - at(Vy, i, j, k))) * (_dy * (at(Ly, i, j + 1, k) - at(Ly, i, j, k)));
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
                    nrm = nrm + (_dz * (at(Vz, i, j, k + 1) - at(Vz, i, j, k))) * (_dz * (at(Lz, i, j, k + 1) - at(Lz, i, j, k)));
                if (k >= 1 && k <= nz - 2)
                    for (int dj = 0; dj < 2; ++dj)
                        for (int di = 0; di < 2; ++di) {
                            const int64_t ie = i + di, je = j + dj;
                            if (ie < 1 || ie > nx - 1 || je < 1 || je > ny - 1) continue;
                            shr = shr + rxy(Vx, Vy, ie, je, k) * rxy(Lx, Ly, ie, je, k);
                        }
                if (j >= 1 && j <= ny - 2)
                    for (int dk = 0; dk < 2; ++dk)
                        for (int di = 0; di < 2; ++di) {
                            const int64_t ie = i + di, ke = k + dk;
                            if (ie < 1 || ie > nx - 1 || ke < 1 || ke > nz - 1) continue;
                            shr = shr + rxz(Vx, Vz, ie, j, ke) * rxz(Lx, Lz, ie, j, ke);
                        }
                if (i >= 1 && i <= nx - 2)
                    for (int dk = 0; dk < 2; ++dk)
                        for (int dj = 0; dj < 2; ++dj) {
                            const int64_t je = j + dj, ke = k + dk;
                            if (je < 1 || je > ny - 1 || ke < 1 || ke > nz - 1) continue;
                            shr = shr + ryz(Vy, Vz, i, je, ke) * ryz(Ly, Lz, i, je, ke);
                        }
                G(i + 1, j + 1, k + 1) = -(at(M, i, j, k) * (2.0 * nrm + shr));
            }
}

// One physical step's term of ∂J/∂log μ for the visco-elastic operator (no reference
// counterpart), from the forward step's converged stresses T and the adjoint step's stresses A:
//   g_c (+)= -[Σ_n A_n T_n/(2 Mus_c) + Mus_c Σ_{edges e around c} A_e T_e/(4 μ̄_e²)],
// μ̄_e the 4-cell average of Mus on the edge. Written with 0-based unified coordinates: a
// stress element (a,b,c) sits at reference index (a-s0+1, b-s1+1, c-s2+1) for the field's
// start (s0,s1,s2); zero outside its extents. add != 0 accumulates into g.
void ora3ve_grad_logmu(oarr grad_, oarr Txx_, oarr Tyy_, oarr Tzz_, oarr Txy_, oarr Txz_, oarr Tyz_, oarr Axx_,
                       oarr Ayy_, oarr Azz_, oarr Axy_, oarr Axz_, oarr Ayz_, oarr Mus_, int add) {
    F3 G(grad_), Txx(Txx_), Tyy(Tyy_), Tzz(Tzz_), Txy(Txy_), Txz(Txz_), Tyz(Tyz_), Axx(Axx_), Ayy(Ayy_), Azz(Azz_),
        Axy(Axy_), Axz(Axz_), Ayz(Ayz_), M(Mus_);
    const int64_t nx = M.n1, ny = M.n2, nz = M.n3;
    auto T = [](const F3& A, int s0, int s1, int s2, int64_t a, int64_t b, int64_t c) -> double {
        const int64_t u = a - s0 + 1, v = b - s1 + 1, w = c - s2 + 1;
        if (u < 1 || u > A.n1 || v < 1 || v > A.n2 || w < 1 || w > A.n3) return 0.0;
        return A(u, v, w);
    };
    auto m = [&](int64_t i, int64_t j, int64_t k) { return M(i + 1, j + 1, k + 1); };
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                const double Mc = m(i, j, k);
                double nrm = 0.0, shr = 0.0;
                if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
                    nrm = nrm + T(Axx, 0, 1, 1, i, j, k) * T(Txx, 0, 1, 1, i, j, k);
                if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
                    nrm = nrm + T(Ayy, 1, 0, 1, i, j, k) * T(Tyy, 1, 0, 1, i, j, k);
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
                    nrm = nrm + T(Azz, 1, 1, 0, i, j, k) * T(Tzz, 1, 1, 0, i, j, k);
                if (k >= 1 && k <= nz - 2)
                    for (int dj = 0; dj < 2; ++dj)
                        for (int di = 0; di < 2; ++di) {
                            const int64_t ie = i + di, je = j + dj;
                            if (ie < 1 || ie > nx - 1 || je < 1 || je > ny - 1) continue;
                            const double mb = (((m(ie - 1, je - 1, k) + m(ie, je - 1, k)) + m(ie - 1, je, k)) + m(ie, je, k)) * 0.25;
                            shr = shr + T(Axy, 1, 1, 1, ie, je, k) * T(Txy, 1, 1, 1, ie, je, k) / (mb * mb);
                        }
                if (j >= 1 && j <= ny - 2)
                    for (int dk = 0; dk < 2; ++dk)
                        for (int di = 0; di < 2; ++di) {
                            const int64_t ie = i + di, ke = k + dk;
                            if (ie < 1 || ie > nx - 1 || ke < 1 || ke > nz - 1) continue;
                            const double mb = (((m(ie - 1, j, ke - 1) + m(ie, j, ke - 1)) + m(ie - 1, j, ke)) + m(ie, j, ke)) * 0.25;
                            shr = shr + T(Axz, 1, 1, 1, ie, j, ke) * T(Txz, 1, 1, 1, ie, j, ke) / (mb * mb);
                        }
                if (i >= 1 && i <= nx - 2)
                    for (int dk = 0; dk < 2; ++dk)
                        for (int dj = 0; dj < 2; ++dj) {
                            const int64_t je = j + dj, ke = k + dk;
                            if (je < 1 || je > ny - 1 || ke < 1 || ke > nz - 1) continue;
                            const double mb = (((m(i, je - 1, ke - 1) + m(i, je, ke - 1)) + m(i, je - 1, ke)) + m(i, je, ke)) * 0.25;
                            shr = shr + T(Ayz, 1, 1, 1, i, je, ke) * T(Tyz, 1, 1, 1, i, je, ke) / (mb * mb);
                        }
                const double t = -(nrm / (2.0 * Mc) + Mc * (shr * 0.25));
                G(i + 1, j + 1, k + 1) = add ? G(i + 1, j + 1, k + 1) + t : t;
            }
}

// compute_Res! (Stokes3D_ve_perf.jl:90-96): ∇V from the current V plus Rx, Ry, Rz.
void ora3p_compute_Res(oarr divV_, oarr Rx_, oarr Ry_, oarr Rz_, oarr Vx_, oarr Vy_, oarr Vz_, oarr Pt_, oarr txx_,
                       oarr tyy_, oarr tzz_, oarr txy_, oarr txz_, oarr tyz_, double _dx, double _dy, double _dz) {
    F3 divV(divV_), Rx(Rx_), Ry(Ry_), Rz(Rz_), Vx(Vx_), Vy(Vy_), Vz(Vz_), Pt(Pt_), txx(txx_), tyy(tyy_), tzz(tzz_),
        txy(txy_), txz(txz_), tyz(tyz_);
#pragma omp parallel for schedule(static)
    for (int64_t iz = 1; iz <= divV.n3; ++iz)
        for (int64_t iy = 1; iy <= divV.n2; ++iy)
            for (int64_t ix = 1; ix <= divV.n1; ++ix) {
                divV(ix, iy, iz) = _dx * (Vx(ix + 1, iy, iz) - Vx(ix, iy, iz)) + _dy * (Vy(ix, iy + 1, iz) - Vy(ix, iy, iz)) +
                                   _dz * (Vz(ix, iy, iz + 1) - Vz(ix, iy, iz));
                if (ix <= Rx.n1 && iy <= Rx.n2 && iz <= Rx.n3)
                    Rx(ix, iy, iz) = _dx * (txx(ix + 1, iy, iz) - txx(ix, iy, iz)) + _dy * (txy(ix, iy + 1, iz) - txy(ix, iy, iz)) +
                                     _dz * (txz(ix, iy, iz + 1) - txz(ix, iy, iz)) - _dx * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix, iy + 1, iz + 1));
                if (ix <= Ry.n1 && iy <= Ry.n2 && iz <= Ry.n3)
                    Ry(ix, iy, iz) = _dy * (tyy(ix, iy + 1, iz) - tyy(ix, iy, iz)) + _dx * (txy(ix + 1, iy, iz) - txy(ix, iy, iz)) +
                                     _dz * (tyz(ix, iy, iz + 1) - tyz(ix, iy, iz)) - _dy * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix + 1, iy, iz + 1));
                if (ix <= Rz.n1 && iy <= Rz.n2 && iz <= Rz.n3)
                    Rz(ix, iy, iz) = _dz * (tzz(ix, iy, iz + 1) - tzz(ix, iy, iz)) + _dx * (txz(ix + 1, iy, iz) - txz(ix, iy, iz)) +
                                     _dy * (tyz(ix, iy + 1, iz) - tyz(ix, iy, iz)) - _dz * (Pt(ix + 1, iy + 1, iz + 1) - Pt(ix + 1, iy + 1, iz));
            }
}

// ---------------------------------------------------------------- reductions for the convergence check

// Sum of squares (norm(A)^2), min and max over a whole array (Stokes2D.jl:137-141).
void ora_stats(oarr A, double* sumsq, double* mn, double* mx) {
    const int64_t n = A.n1 * A.n2 * A.n3;
    double s = 0.0, lo = INFINITY, hi = -INFINITY;
#pragma omp parallel for reduction(+ : s) reduction(min : lo) reduction(max : hi) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double v = A.p[i];
        s += v * v;
        lo = std::min(lo, v);
        hi = std::max(hi, v);
    }
    *sumsq = s; *mn = lo; *mx = hi;
}

int ora_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
