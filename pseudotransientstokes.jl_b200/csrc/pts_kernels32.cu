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

#include <cstring>

#include "pts_internal.h"
#include "pts_tma.cuh"
#include "pts_zvbc.cuh"

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

// ---- the δ-form compute_Pt_τ! as a z-marching kernel with TMA-staged planes ----
//
// The same arithmetic as k3_corrA, with the operands staged like the FP64 z-marching
// compute_Pt_τ! (pts_zstage.cu): a CTA owns a 32 x TY tile, TY consumer warps march through
// a chunk of z-planes and one producer warp issues one 3D tensor copy per array and plane
// into a ring of R shared-memory slots. Slot of plane s:
//   halo group (rows j0-1 .. j0+TY):  δVx(s), δVy(s), δVz(s+1)  boxes of 40 floats from i0-4;
//                                     (Gdτ, Mus)(s) pairs       box of 36 pairs from i0-2
//   point group (TX x TY):            δPt, aP, u_xx .. u_yz at s
// (x offsets are multiples of 16 bytes, the TMA rule). The values of plane k-1 (the -z
// neighbours) are carried in registers. Waits are bounded (pts_tma.cuh).
namespace zs32 {
using namespace tma;
constexpr int TX = 32;
constexpr int HWF = TX + 8;  // float halo box width: i0-4 .. i0+TX+3
constexpr int HWP = TX + 4;  // pair halo box width:  i0-2 .. i0+TX+1
constexpr int NP = 8;

struct alignas(64) Maps {
    CUtensorMap h[4];   // δVx δVy δVz GM
    CUtensorMap p[NP];  // δPt aP u_xx u_yy u_zz u_xy u_xz u_yz
};

template <int TY>
struct Cfg {
    static constexpr int HH = TY + 2;
    static constexpr int FBOX = HWF * HH * 4;
    static constexpr int FSTRIDE = (FBOX + 127) / 128 * 128;
    static constexpr int GBOX = HWP * HH * 8;
    static constexpr int GSTRIDE = (GBOX + 127) / 128 * 128;
    static constexpr int PBOX = TX * TY * 4;
    static constexpr int SLOT = 3 * FSTRIDE + GSTRIDE + NP * PBOX;
};

template <bool EL, int TY, int R>
__global__ void __launch_bounds__(32 * (TY + 1)) k3_corrA_zs(const __grid_constant__ Maps maps, Geom g, Mixed32 m,
                                                              Num32 n, int kz, int* err) {
    using C = Cfg<TY>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* full = (uint64_t*)(smem + (size_t)R * C::SLOT);
    uint64_t* empty = full + R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int kb = blockIdx.z * kz;
    const int ke = min(kb + kz, g.nz);
    const int nst = ke - kb + 1;
    if (threadIdx.x == 0) {
        for (int q = 0; q < R; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], TY);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == TY) {
        if (lane != 0) return;
        for (int q = 0; q < 4; ++q) prefetch_map(&maps.h[q]);
        for (int q = 0; q < NP; ++q) prefetch_map(&maps.p[q]);
        bool ok = true;
        int issued = 0;
        for (int t = 0; t < nst; ++t) {
            const int slot = t % R, use = t / R;
            if (use > 0 && !mbar_wait(&empty[slot], (use - 1) & 1)) {
                ok = false;
                break;
            }
            const int s = kb - 1 + t;
            unsigned char* base = smem + (size_t)slot * C::SLOT;
            mbar_expect_tx(&full[slot], 3 * C::FBOX + C::GBOX + (t > 0 ? NP * C::PBOX : 0));
            tma_load3(base, &maps.h[0], i0 - 4, j0 - 1, s, &full[slot]);
            tma_load3(base + C::FSTRIDE, &maps.h[1], i0 - 4, j0 - 1, s, &full[slot]);
            tma_load3(base + 2 * C::FSTRIDE, &maps.h[2], i0 - 4, j0 - 1, s + 1, &full[slot]);
            tma_load3(base + 3 * C::FSTRIDE, &maps.h[3], i0 - 2, j0 - 1, s, &full[slot]);
            if (t > 0) {
                unsigned char* pb = base + 3 * C::FSTRIDE + C::GSTRIDE;
#pragma unroll
                for (int q = 0; q < NP; ++q) tma_load3(pb + q * C::PBOX, &maps.p[q], i0, j0, s, &full[slot]);
            }
            issued = t + 1;
        }
        if (!ok) atomicExch(err, 1);
        for (int t = (issued > R ? issued - R : 0); t < issued; ++t)
            if (!mbar_wait(&full[t % R], (t / R) & 1)) {
                atomicExch(err, 1);
                break;
            }
        return;
    }
    const int i = i0 + lane, j = j0 + warp;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in = i < nx && j < ny;
    const bool jI = j >= 1 && j <= ny - 2, iI = i >= 1 && i <= nx - 2;
    const bool cx = in && jI, cy = in && iI, czz = in && iI && jI;
    const bool cxy = in && i >= 1 && j >= 1, cxz = in && i >= 1 && jI, cyz = in && iI && j >= 1;
    const int hf = (warp + 1) * HWF + (lane + 4);  // this cell in a float halo box
    const int hp = (warp + 1) * HWP + (lane + 2);  // this cell in the pair halo box
    const int pc = warp * TX + lane;
    constexpr int PS = TX * TY;
    float vx_m, vy_m, vz_c, vz_x, vz_y;
    float2 g_m, gx_m, gy_m;
    idx_t c = gidx32(g, i, j, kb);
    const idx_t sz = (idx_t)g.pxy;
    for (int t = 0; t < nst; ++t) {
        const int slot = t % R;
        if (!mbar_wait(&full[slot], (t / R) & 1)) {
            atomicExch(err, 1);
            return;
        }
        const unsigned char* base = smem + (size_t)slot * C::SLOT;
        const float* hVx = (const float*)base;
        const float* hVy = (const float*)(base + C::FSTRIDE);
        const float* hVz = (const float*)(base + 2 * C::FSTRIDE);  // δVz of plane s+1
        const float2* hGM = (const float2*)(base + 3 * C::FSTRIDE);
        const float vx = hVx[hf], vy = hVy[hf];
        const float2 gm = hGM[hp], gmx = hGM[hp - 1], gmy = hGM[hp - HWP];
        const float vzn = hVz[hf], vznx = hVz[hf - 1], vzny = hVz[hf - HWF];
        if (t > 0 && in) {
            const int k = kb + t - 1;
            const float* P = (const float*)(base + 3 * C::FSTRIDE + C::GSTRIDE);
            const float Gc = gm.x, Mc = gm.y;
            const float dvx = hVx[hf + 1] - vx;
            const float dvy = hVy[hf + HWF] - vy;
            const float dvz = vzn - vz_c;
            m.dPt[c] = P[pc] - n.r * Gc * (P[PS + pc] + ((n._dx * dvx + n._dy * dvy) + n._dz * dvz));
            const bool kI = k >= 1 && k <= nz - 2, k1 = k >= 1;
            const float Dn = (1.0f + __fdividef(Gc, Mc)) + (EL ? gr32(Gc, n) : 0.0f);
            const float G2 = 2.0f * Gc;
            const float rDn = __fdividef(1.0f, Dn);
            if (cx && kI) m.dtxx[c] = (P[2 * PS + pc] + G2 * (n._dx * dvx)) * rDn;
            if (cy && kI) m.dtyy[c] = (P[3 * PS + pc] + G2 * (n._dy * dvy)) * rDn;
            if (czz) m.dtzz[c] = (P[4 * PS + pc] + G2 * (n._dz * dvz)) * rDn;
            if (cxy && kI) {
                const float2 a = hGM[hp - HWP - 1];
                const float ag = (((a.x + gmy.x) + gmx.x) + Gc) * 0.25f;
                const float am = (((a.y + gmy.y) + gmx.y) + Mc) * 0.25f;
                const float sh = 0.5f * (n._dy * (vx - hVx[hf - HWF]) + n._dx * (vy - hVy[hf - 1]));
                m.dtxy[c] = __fdividef(P[5 * PS + pc] + (2.0f * ag) * sh,
                                       (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
            }
            if (cxz && k1) {
                const float ag = (((gx_m.x + g_m.x) + gmx.x) + Gc) * 0.25f;
                const float am = (((gx_m.y + g_m.y) + gmx.y) + Mc) * 0.25f;
                const float sh = 0.5f * (n._dz * (vx - vx_m) + n._dx * (vz_c - vz_x));
                m.dtxz[c] = __fdividef(P[6 * PS + pc] + (2.0f * ag) * sh,
                                       (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
            }
            if (cyz && k1) {
                const float ag = (((gy_m.x + g_m.x) + gmy.x) + Gc) * 0.25f;
                const float am = (((gy_m.y + g_m.y) + gmy.y) + Mc) * 0.25f;
                const float sh = 0.5f * (n._dz * (vy - vy_m) + n._dy * (vz_c - vz_y));
                m.dtyz[c] = __fdividef(P[7 * PS + pc] + (2.0f * ag) * sh,
                                       (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
            }
            c += sz;
        }
        vx_m = vx, vy_m = vy, g_m = gm, gx_m = gmx, gy_m = gmy;
        vz_c = vzn, vz_x = vznx, vz_y = vzny;
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
    }
}

// Tile configurations (TY, R). Shared memory per block: 8x2 32 KB, 8x3 48 KB (4 blocks/SM),
// 4x3 26 KB, 16x2 60 KB. The first is the fastest measured at 511^3 on a B200.
constexpr int kTiles[][2] = {{8, 2}, {8, 3}, {4, 3}, {16, 2}};
constexpr int kNumTiles = (int)(sizeof(kTiles) / sizeof(kTiles[0]));

template <bool EL, int TY, int R>
cudaError_t launch(const Geom& g, const Mixed32& m, const Num32& n, int kz, int* err, cudaStream_t s) {
    using C = Cfg<TY>;
    Maps maps;
    memset(&maps, 0, sizeof(maps));
    const void* hsrc[3] = {m.dVx, m.dVy, m.dVz};
    for (int q = 0; q < 3; ++q)
        if (!encode_field(&maps.h[q], hsrc[q], g, 4, HWF, C::HH)) return cudaErrorInvalidValue;
    if (!encode_field(&maps.h[3], m.GM, g, 8, HWP, C::HH)) return cudaErrorInvalidValue;
    const void* psrc[NP] = {m.dPt, m.aP, m.dtxx, m.dtyy, m.dtzz, m.dtxy, m.dtxz, m.dtyz};
    for (int q = 0; q < NP; ++q)
        if (!encode_field(&maps.p[q], psrc[q], g, 4, TX, TY)) return cudaErrorInvalidValue;
    const size_t smem = 128 + (size_t)R * C::SLOT + 2 * R * sizeof(uint64_t);
    static bool attr[64] = {};  // per device: the opt-in to more than 48 KB of shared memory
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e =
            cudaFuncSetAttribute(k3_corrA_zs<EL, TY, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    const dim3 grid((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, (g.nz + kz - 1) / kz);
    k3_corrA_zs<EL, TY, R><<<grid, 32 * (TY + 1), smem, s>>>(maps, g, m, n, kz, err);
    return cudaGetLastError();
}

template <bool EL>
cudaError_t launch_form(int tile, const Geom& g, const Mixed32& m, const Num32& n, int kz, int* err, cudaStream_t s) {
    switch (tile) {
        case 0: return launch<EL, kTiles[0][0], kTiles[0][1]>(g, m, n, kz, err, s);
        case 1: return launch<EL, kTiles[1][0], kTiles[1][1]>(g, m, n, kz, err, s);
        case 2: return launch<EL, kTiles[2][0], kTiles[2][1]>(g, m, n, kz, err, s);
        case 3: return launch<EL, kTiles[3][0], kTiles[3][1]>(g, m, n, kz, err, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace zs32

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

cudaError_t launch_corr_A32_zs(int v, int tile, const Geom& g, const Mixed32& m, const Num& n, int kz, int* err,
                               cudaStream_t s) {
    if (kz <= 0) kz = 32;
    if (v == VE3D_PERF) return zs32::launch_form<true>(tile, g, m, num32(n), kz, err, s);
    if (v == V3D) return zs32::launch_form<false>(tile, g, m, num32(n), kz, err, s);
    return cudaErrorInvalidValue;
}

int zstage32_num_configs() { return zs32::kNumTiles; }

bool zstage32_tile_info(int tile, int* ty, int* ring) {
    if (tile < 0 || tile >= zs32::kNumTiles) return false;
    if (ty) *ty = zs32::kTiles[tile][0];
    if (ring) *ring = zs32::kTiles[tile][1];
    return true;
}

// The δ-form compute_V! + bc as the z-staged template of pts_zvbc.cuh (FP32, sources aV).
namespace zvbc32 {
using namespace zvbc;
struct VTile {
    int ty, r, pw, minb;
};
constexpr VTile kVTiles[] = {{8, 2, 1, 4}, {8, 2, 0, 5}, {4, 2, 1, 8}, {8, 3, 1, 3}};
constexpr int kNumVTiles = (int)(sizeof(kVTiles) / sizeof(kVTiles[0]));

template <int Q>
cudaError_t launch32(const Geom& g, const Mixed32& m, const Num& n, int kz, int* err, cudaStream_t s) {
    constexpr VTile c = kVTiles[Q];
    MapsV maps;
    memset(&maps, 0, sizeof(maps));
    const void* hsrc[NHV] = {m.dtxx, m.dtyy, m.dtxy, m.dPt, m.dtRho, m.dtxz, m.dtyz};
    const void* psrc[9] = {m.dVx, m.dVy, m.dVz, m.dtzz, m.dPt, m.dtRho, m.aVx, m.aVy, m.aVz};
    if (!make_maps<float, c.ty, true>(&maps, g, hsrc, psrc)) return cudaErrorInvalidValue;
    ArgsV<float> a{m.dVx, m.dVy, m.dVz, {m.aVx, m.aVy, m.aVz}};
    NumV<float> nv{(float)n.dx, (float)n.dy, (float)n.dz, (float)n._dx, (float)n._dy, (float)n._dz, 0.5f};
    return launch_v<float, true, true, c.ty, c.r, c.pw != 0, c.minb>(g, maps, a, nv, kz, err, s);
}
}  // namespace zvbc32

cudaError_t launch_corr_B32_zs(int v, int tile, const Geom& g, const Mixed32& m, const Num& n, int kz, int* err,
                               cudaStream_t s) {
    if (v != VE3D_PERF && v != V3D) return cudaErrorInvalidValue;
    switch (tile) {
        case 0: return zvbc32::launch32<0>(g, m, n, kz, err, s);
        case 1: return zvbc32::launch32<1>(g, m, n, kz, err, s);
        case 2: return zvbc32::launch32<2>(g, m, n, kz, err, s);
        case 3: return zvbc32::launch32<3>(g, m, n, kz, err, s);
        default: return cudaErrorInvalidValue;
    }
}

int zvbc32_num_configs() { return zvbc32::kNumVTiles; }

cudaError_t launch_corr_B32(int v, const Geom& g, const Mixed32& m, const Num& n, cudaStream_t s) {
    if (v != VE3D_PERF && v != V3D) return cudaErrorInvalidValue;
    const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nz + 1), blk(32, 8, 1);
    k3_corrB<<<grid, blk, 0, s>>>(g, m, num32(n));
    return cudaGetLastError();
}

}  // namespace pts
