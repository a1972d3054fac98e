// pts_expr64.cuh -- the FP64 stress-update expressions of compute_τ! / compute_Pt_τ!,
// shared by every FP64 translation unit (all compiled with --fmad=false).
//
// Each expression is written in the reference's left-to-right order, so a kernel that
// evaluates it on the same operands reproduces the reference's Float64 arithmetic bit for
// bit, whichever way the kernel fetches those operands.
#pragma once

namespace pts {
namespace expr {

// Gr = Gdτ/(G*dt). When G*dt is exactly 1.0 the quotient is Gdτ itself (IEEE division by
// one is exact), so the division is skipped; the result is the same bits either way.
__device__ __forceinline__ double gr_of(double g, double gdt) {
    if (gdt == 1.0) return g;
    return g / gdt;
}

// Normal stress update. Perf form (Stokes3D_ve_perf.jl:71-73):
//   (τ + τ_o*Gr + 2.0*Gdτ*(_dx*d)) / (1.0 + Gdτ/Mus + Gr),  Gr = Gdτ/(G*dt)
// Role form (Stokes3D_ve_multixpu.jl:70-72): the same with (d/dx).
// Viscous: the τ_o and Gr terms are absent.
template <bool EL, bool PERF>
__device__ __forceinline__ double tau_n(double t, double to, double g, double m, double gdt, double h, double ih,
                                        double d) {
    const double e = PERF ? (ih * d) : (d / h);
    if (EL) {
        const double Gr = gr_of(g, gdt);
        return ((t + to * Gr) + (2.0 * g) * e) / ((1.0 + g / m) + Gr);
    }
    return (t + (2.0 * g) * e) / (1.0 + g / m);
}

// Shear stress update (Stokes3D_ve_perf.jl:74-76, Stokes3D_ve_multixpu.jl:73-75):
//   (τ + τ_o*av_Gr + 2.0*av_Gdτ*(0.5*(_h1*d1 + _h2*d2))) / (1.0 + av_Gdτ/av_Mus + av_Gr)
template <bool EL, bool PERF>
__device__ __forceinline__ double tau_s(double t, double to, double ag, double am, double gdt, double h1, double ih1,
                                        double d1, double h2, double ih2, double d2) {
    const double s = PERF ? (ih1 * d1 + ih2 * d2) : (d1 / h1 + d2 / h2);
    if (EL) {
        const double Gr = gr_of(ag, gdt);
        return ((t + to * Gr) + (2.0 * ag) * (0.5 * s)) / ((1.0 + ag / am) + Gr);
    }
    return (t + (2.0 * ag) * (0.5 * s)) / (1.0 + ag / am);
}

// Normal stress update with the denominator computed once per cell: τxx, τyy, τzz share
// Gdτ and Mus at the cell centre, so (1.0 + Gdτ/Mus + Gr) and Gr are the same three times
// (same operations, same bits as tau_n).
template <bool EL, bool PERF>
__device__ __forceinline__ double tau_n_den(double t, double to, double g, double Gr, double den, double h, double ih,
                                            double d) {
    const double e = PERF ? (ih * d) : (d / h);
    if (EL) return ((t + to * Gr) + (2.0 * g) * e) / den;
    return (t + (2.0 * g) * e) / den;
}

// One spatial derivative: _h*d in the perf form, d/h in the role form.
template <bool PERF>
__device__ __forceinline__ double dsc(double d, double h, double ih) {
    return PERF ? (ih * d) : (d / h);
}

}  // namespace expr
}  // namespace pts
