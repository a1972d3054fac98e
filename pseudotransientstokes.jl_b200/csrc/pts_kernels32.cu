// pts_kernels32.cu -- FP32 inner sweeps of the mixed-precision PT solve (3D, _dx form).
//
// The state of the sweeps is a correction δ to the FP64 iterate X (Pt, τ, V). The FP64
// residuals of X enter as sources, computed once per outer step (pts_kernels64.cu):
//   aP = ∇·V_X,  aτ = τ_o*Gr + 2Gdτ*ε̇(V_X) - τ_X*(D - 1),  D = 1 + Gdτ/Mus + Gr
// and the sweep is the reference's PT iteration (compute_Pt_τ!, compute_V! + bc,
// Stokes3D_ve_perf.jl:69-88,202-207) written for X + δ with X held fixed:
//   δPt' = δPt - r*Gdτ*(aP + ∇·δV)
//   δτ'  = (δτ + aτ + 2Gdτ*ε̇(δV)) / D
//   δV'  = δV + (R(δτ', δPt') + R(τ_X, Pt_X)) * av(dτ_Rho)
// The stress corrections are carried as u = δτ - w with w = aτ/(D - 1), which turns the
// stress update into u' = (u + 2Gdτ*ε̇(δV)) / D with no source, and the momentum update
// into δV' = δV + (R(u', δPt') + aV) * av(dτ_Rho) with aV = R(τ_X, Pt_X) + R_τ(w) (the
// stress part of R); w, aV and the start u = -w come from the outer step, which folds
// δτ = u + w into X. In exact arithmetic X + δ follows the FP64 iteration step for step;
// in FP32 the rounding is relative to the size of δ and w, which the outer step folds
// into X (in FP64) every nout sweeps. The sweeps read no stress source, and the stress
// and velocity fields move half the bytes of the FP64 kernels. Compiled with FMA
// contraction (no bit-exact target here).
#include <cuda_runtime.h>

#include "pts_internal.h"

namespace pts {
namespace {

struct Num32 {
    float _dx, _dy, _dz, r, gdt;
    int gdt_one;
};

__device__ __forceinline__ float gr32(float g, const Num32& n) { return n.gdt_one ? g : __fdividef(g, n.gdt); }

// δ-form compute_Pt_τ! (stresses as u = δτ - w), one thread per cell (arrays it only reads go through the read-only
// data path).
template <bool EL>
__global__ void __launch_bounds__(256) k3_corrA(Geom g, Mixed32 m, Num32 n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    const float dvx = __ldg(&m.dVx[c + sx]) - __ldg(&m.dVx[c]);
    const float dvy = __ldg(&m.dVy[c + sy]) - __ldg(&m.dVy[c]);
    const float dvz = __ldg(&m.dVz[c + sz]) - __ldg(&m.dVz[c]);
    const float2 gmc = __ldg(&m.GM[c]);
    const float Gc = gmc.x, Mc = gmc.y;
    // 4-point averages of Gdτ and Mus on an edge from the interleaved pairs at c-o1-o2, c-o2, c-o1, c
    auto avg = [&](idx_t o1, idx_t o2, float* ag, float* am) {
        const float2 a = __ldg(&m.GM[c - o1 - o2]), b = __ldg(&m.GM[c - o2]), d = __ldg(&m.GM[c - o1]);
        *ag = (((a.x + b.x) + d.x) + Gc) * 0.25f;
        *am = (((a.y + b.y) + d.y) + Mc) * 0.25f;
    };
    m.dPt[c] = m.dPt[c] - n.r * Gc * (__ldg(&m.aP[c]) + ((n._dx * dvx + n._dy * dvy) + n._dz * dvz));
    const float Dn = (1.0f + __fdividef(Gc, Mc)) + (EL ? gr32(Gc, n) : 0.0f);
    const float G2 = 2.0f * Gc;
    const float rDn = __fdividef(1.0f, Dn);
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
        m.dtxx[c] = (m.dtxx[c] + G2 * (n._dx * dvx)) * rDn;
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
        m.dtyy[c] = (m.dtyy[c] + G2 * (n._dy * dvy)) * rDn;
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
        m.dtzz[c] = (m.dtzz[c] + G2 * (n._dz * dvz)) * rDn;
    if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2) {
        float ag, am;
        avg(sx, sy, &ag, &am);
        const float s = 0.5f * (n._dy * (__ldg(&m.dVx[c]) - __ldg(&m.dVx[c - sy])) + n._dx * (__ldg(&m.dVy[c]) - __ldg(&m.dVy[c - sx])));
        m.dtxy[c] = __fdividef(m.dtxy[c] + (2.0f * ag) * s, (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
    }
    if (i >= 1 && j >= 1 && j <= ny - 2 && k >= 1) {
        float ag, am;
        avg(sx, sz, &ag, &am);
        const float s = 0.5f * (n._dz * (__ldg(&m.dVx[c]) - __ldg(&m.dVx[c - sz])) + n._dx * (__ldg(&m.dVz[c]) - __ldg(&m.dVz[c - sx])));
        m.dtxz[c] = __fdividef(m.dtxz[c] + (2.0f * ag) * s, (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && k >= 1) {
        float ag, am;
        avg(sy, sz, &ag, &am);
        const float s = 0.5f * (n._dz * (__ldg(&m.dVy[c]) - __ldg(&m.dVy[c - sz])) + n._dy * (__ldg(&m.dVz[c]) - __ldg(&m.dVz[c - sy])));
        m.dtyz[c] = __fdividef(m.dtyz[c] + (2.0f * ag) * s, (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
    }
}

__device__ __forceinline__ void bc_copies32(float* A, idx_t c, float v, int a, int alo, int ahi, idx_t sa, int b,
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

// δ-form compute_V! with the free-slip copies, one thread per face point.
__global__ void __launch_bounds__(256) k3_corrB(Geom g, Mixed32 m, Num32 n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i > nx || j > ny) return;
    const idx_t c = gidx32(g, i, j, k);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
        float v = m.dVx[c];
        if (i >= 1 && i <= nx - 1) {
            const float R = (((n._dx * (__ldg(&m.dtxx[c]) - __ldg(&m.dtxx[c - sx])) + n._dy * (__ldg(&m.dtxy[c + sy]) - __ldg(&m.dtxy[c]))) +
                              n._dz * (__ldg(&m.dtxz[c + sz]) - __ldg(&m.dtxz[c]))) -
                             n._dx * (__ldg(&m.dPt[c]) - __ldg(&m.dPt[c - sx]))) +
                            __ldg(&m.aVx[c]);
            v = v + R * ((__ldg(&m.dtRho[c - sx]) + __ldg(&m.dtRho[c])) * 0.5f);
            m.dVx[c] = v;
        }
        bc_copies32(m.dVx, c, v, j, 1, ny - 2, sy, k, 1, nz - 2, sz);
    }
    if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) {
        float v = m.dVy[c];
        if (j >= 1 && j <= ny - 1) {
            const float R = (((n._dy * (__ldg(&m.dtyy[c]) - __ldg(&m.dtyy[c - sy])) + n._dx * (__ldg(&m.dtxy[c + sx]) - __ldg(&m.dtxy[c]))) +
                              n._dz * (__ldg(&m.dtyz[c + sz]) - __ldg(&m.dtyz[c]))) -
                             n._dy * (__ldg(&m.dPt[c]) - __ldg(&m.dPt[c - sy]))) +
                            __ldg(&m.aVy[c]);
            v = v + R * ((__ldg(&m.dtRho[c - sy]) + __ldg(&m.dtRho[c])) * 0.5f);
            m.dVy[c] = v;
        }
        bc_copies32(m.dVy, c, v, i, 1, nx - 2, sx, k, 1, nz - 2, sz);
    }
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
        float v = m.dVz[c];
        if (k >= 1 && k <= nz - 1) {
            const float R = (((n._dz * (__ldg(&m.dtzz[c]) - __ldg(&m.dtzz[c - sz])) + n._dx * (__ldg(&m.dtxz[c + sx]) - __ldg(&m.dtxz[c]))) +
                              n._dy * (__ldg(&m.dtyz[c + sy]) - __ldg(&m.dtyz[c]))) -
                             n._dz * (__ldg(&m.dPt[c]) - __ldg(&m.dPt[c - sz]))) +
                            __ldg(&m.aVz[c]);
            v = v + R * ((__ldg(&m.dtRho[c - sz]) + __ldg(&m.dtRho[c])) * 0.5f);
            m.dVz[c] = v;
        }
        bc_copies32(m.dVz, c, v, i, 1, nx - 2, sx, j, 1, ny - 2, sy);
    }
}

Num32 num32(const Num& n) {
    return Num32{(float)n._dx, (float)n._dy, (float)n._dz, (float)n.r, (float)n.gdt, n.gdt == 1.0 ? 1 : 0};
}

}  // namespace

cudaError_t launch_corr_A32(int v, const Geom& g, const Mixed32& m, const Num& n, cudaStream_t s) {
    const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz), blk(32, 8, 1);
    if (v == VE3D_PERF) k3_corrA<true><<<grid, blk, 0, s>>>(g, m, num32(n));
    else if (v == V3D) k3_corrA<false><<<grid, blk, 0, s>>>(g, m, num32(n));
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_corr_B32(int v, const Geom& g, const Mixed32& m, const Num& n, cudaStream_t s) {
    if (v != VE3D_PERF && v != V3D) return cudaErrorInvalidValue;
    const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nz + 1), blk(32, 8, 1);
    k3_corrB<<<grid, blk, 0, s>>>(g, m, num32(n));
    return cudaGetLastError();
}

}  // namespace pts
