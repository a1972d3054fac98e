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
    float _dx, _dy, _dz, r;
    float igdt;  // 1/(G*dt): Gr = Gdτ/(G*dt) as one multiply (exact when G*dt = 1, as in the scripts)
};

__device__ __forceinline__ float gr32(float g, const Num32& n) { return g * n.igdt; }

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
    return Num32{(float)n._dx, (float)n._dy, (float)n._dz, (float)n.r, (float)(1.0 / n.gdt)};
}

// ---- compute_V! + bc of one sweep and compute_Pt_τ! of the next in one z-marching pass ----
//
// The two δ-form kernels above exchange u and δPt through memory every sweep: the stress
// kernel writes them and the velocity kernel reads them back (and δV the other way). This
// kernel does the velocity update of sweep q and the stress/pressure update of sweep q+1
// in one pass, so per pair it reads δV, u, δPt, the sources and the coefficients once and
// writes δV, u, δPt once (27 arrays of 4 B instead of 37). The updates are the same
// expressions as k3_corrB / the FP32 zvbc instantiation and k3_corrA_zs, in the same order.
//
// Inputs come from one set of buffers (`m`) and the results go to the other (`o`): a CTA
// computes velocities on a halo of its tile that neighbouring CTAs own, so the update
// cannot be in place. A CTA owns a 32 x TY column of cells and marches through a chunk of
// z-planes; stage t of the ring holds plane p = kb-1+t of every input as halo boxes
// (columns i0-4 .. i0+35, rows j0-2 .. j0+TY+1): δVx δVy δVz u_xx u_yy u_zz u_xy u_xz
// u_yz δPt dτ_Rho aVx aVy aVz, plus the (Gdτ, Mus) pairs (columns i0-2 .. i0+31, rows
// j0-1 .. j0+TY-1) and aP (the tile). At step t (newest plane s = kb-1+t):
//   1. velocities of plane s-1 (δVx, δVy) and of z-face s (δVz) on the extended region
//      E = columns i0-1 .. i0+32, rows j0-1 .. j0+TY, into shared memory (three rotating
//      planes); the free-slip copies are values of the interior point they copy (the
//      tangential index clamped into the interior), the boundary faces keep their value;
//      the owned part is written to `o`;
//   2. after a barrier of the consumer warps, u and δPt of cell plane s-1 from those
//      velocities, into `o`.
// The z-ghost planes of δVx and δVy are the copies of planes 1 and nz-2: plane nz-2's
// values are still in shared memory when plane nz-1 is reached; plane 1 comes one step
// after plane 0, so δPt of plane 0 (the only update of plane 0 that reads δVx, δVy there)
// is finished one step late, and τxz/τyz of z-face 1 see a zero z-difference, as the copy
// makes them. Waits are bounded; a warp whose wait gives up keeps taking the barriers with
// the others and skips its work.
//
// Measured on a B200 at 511^3 (3D VE): 4.58 ms per sweep against 3.68 ms for the two
// kernels, although it moves 27% fewer bytes. Each block holds two full planes of 14 halo
// boxes (about 60 KB at TY = 8) while it computes, so two blocks fit on an SM with only one
// stage of each in flight: too few bytes in flight to cover HBM latency. It is therefore
// opt-in (pts_desc.mixed_sweep = 1 + tile).
namespace zf32 {
using namespace tma;
constexpr int TX = 32;
constexpr int XP = 4;            // halo boxes start 4 floats (16 bytes) left of the tile
constexpr int HW = TX + 2 * XP;  // 40 columns
constexpr int NB = 14;           // halo-box arrays
enum { B_VX, B_VY, B_VZ, B_XX, B_YY, B_ZZ, B_XY, B_XZ, B_YZ, B_PT, B_RHO, B_AX, B_AY, B_AZ };
constexpr int GW = TX + 2;  // (Gdτ, Mus) pair box: columns i0-2 .. i0+31
constexpr int EW = TX + 2;  // extended region: columns i0-1 .. i0+TX

struct alignas(64) Maps {
    CUtensorMap h[NB];
    CUtensorMap gm;
    CUtensorMap ap;
};

// The other buffer set of the ten iterated corrections.
struct Out {
    float *dPt, *dVx, *dVy, *dVz;
    float* u[6];  // xx yy zz xy xz yz
};

template <int TY>
struct Cfg {
    static constexpr int HH = TY + 4;
    static constexpr int HBOX = HW * HH * 4;
    static constexpr int HS = (HBOX + 127) / 128 * 128 / 4;  // floats between halo boxes
    static constexpr int GH = TY + 1;
    static constexpr int GBOX = GW * GH * 8;
    static constexpr int GSTRIDE = (GBOX + 127) / 128 * 128;
    static constexpr int PBOX = TX * TY * 4;
    static constexpr int PSTRIDE = (PBOX + 127) / 128 * 128;
    static constexpr int SLOT = NB * HS * 4 + GSTRIDE + PSTRIDE;
    static constexpr int EH = TY + 2;
    static constexpr int EN = EW * EH;
    static constexpr int VBUF = 3 * 3 * EN * 4;  // δVx, δVy, δVz of three rotating planes
    static constexpr uint32_t TXB = NB * HBOX + GBOX + PBOX;
};

template <int TY, int R>
__device__ __forceinline__ void issue_f(const Maps& maps, unsigned char* smem, uint64_t* full, int t, int i0, int j0,
                                        int kb) {
    using C = Cfg<TY>;
    const int slot = t % R, p = kb - 1 + t;
    unsigned char* base = smem + (size_t)slot * C::SLOT;
    mbar_expect_tx(&full[slot], C::TXB);
#pragma unroll
    for (int q = 0; q < NB; ++q) tma_load3(base + q * C::HS * 4, &maps.h[q], i0 - XP, j0 - 2, p, &full[slot]);
    tma_load3(base + NB * C::HS * 4, &maps.gm, i0 - 2, j0 - 1, p, &full[slot]);
    tma_load3(base + NB * C::HS * 4 + C::GSTRIDE, &maps.ap, i0, j0, p, &full[slot]);
}

__device__ __forceinline__ void consumer_sync(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

template <bool EL, int TY, int R, int MINB>
__global__ void __launch_bounds__(32 * (TY + 1), MINB)
    k3_corrBA_zs(const __grid_constant__ Maps maps, Geom g, Out o, Num32 n, int kz, int* err) {
    using C = Cfg<TY>;
    constexpr int HS = C::HS, EN = C::EN, NT = 32 * TY;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    float* sv = (float*)(smem + (size_t)R * C::SLOT);
    uint64_t* full = (uint64_t*)(smem + (size_t)R * C::SLOT + C::VBUF);
    uint64_t* empty = full + R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int kb = blockIdx.z * kz;
    const int ke = min(kb + kz, g.nz);
    const int nst = ke - kb + 2;  // planes kb-1 .. ke
    if (threadIdx.x == 0) {
        for (int q = 0; q < R; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], TY);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == TY) {  // producer warp: lane 0 keeps the ring R-1 stages ahead
        if (lane != 0) return;
        for (int q = 0; q < NB; ++q) prefetch_map(&maps.h[q]);
        prefetch_map(&maps.gm);
        prefetch_map(&maps.ap);
        int issued = 0;
        for (int t = 0; t < nst; ++t) {
            if (t >= R && !mbar_wait(&empty[t % R], (t / R - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            issue_f<TY, R>(maps, smem, full, t, i0, j0, kb);
            issued = t + 1;
        }
        // wait (bounded) for the copies nobody will consume, so none is in flight at exit
        for (int t = (issued > R ? issued - R : 0); t < issued; ++t)
            if (!mbar_wait(&full[t % R], (t / R) & 1)) {
                atomicExch(err, 1);
                break;
            }
        return;
    }
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const idx_t sz = (idx_t)g.pxy;
    // own cell of the stress/pressure update
    const int i = i0 + lane, j = j0 + warp;
    const bool in = i < nx && j < ny;
    const bool jI = j >= 1 && j <= ny - 2, iI = i >= 1 && i <= nx - 2;
    const bool cx = in && jI, cy = in && iI, czz = in && iI && jI;
    const bool cxy = in && i >= 1 && j >= 1, cxz = in && i >= 1 && jI, cyz = in && iI && j >= 1;
    const int e0 = (warp + 1) * EW + (lane + 1);     // own cell in the extended region
    const int h0 = (warp + 2) * HW + (lane + XP);    // own cell in a halo box
    const int g0 = (warp + 1) * GW + (lane + 2);     // own cell in the pair box
    const int p0 = warp * TX + lane;                 // own cell in the aP box
    float vx_m = 0.0f, vy_m = 0.0f;                  // δVx, δVy of plane k-1 at the own cell
    float2 g_m = make_float2(0.0f, 0.0f), gx_m = g_m, gy_m = g_m;  // pairs of plane k-1: c, c-x, c-y
    float pt0 = 0.0f, gc0 = 0.0f, ap0 = 0.0f, dvz0 = 0.0f;        // δPt of plane 0, finished at plane 1
    bool ok = true;
    for (int t = 0; t < nst; ++t) {
        const int slot = t % R;
        if (ok && !mbar_wait(&full[slot], (t / R) & 1)) {
            atomicExch(err, 1);
            ok = false;
        }
        if (t == 0) continue;  // plane kb-1 only arrives
        const int s = kb - 1 + t, kv = s - 1;
        const float* Hc = (const float*)(smem + (size_t)slot * C::SLOT);                // plane s
        const float* Hp = (const float*)(smem + (size_t)((t + R - 1) % R) * C::SLOT);   // plane s-1
        float* vxn = sv + (t % 3) * 3 * EN;  // δVx, δVy of plane s-1 and δVz of face s
        float* vyn = vxn + EN;
        float* vzn = vyn + EN;
        const float* vxo = sv + ((t + 2) % 3) * 3 * EN;  // the step before: plane s-2, face s-1
        const float* vzo = vxo + 2 * EN;
        const bool own_v = kv >= kb && kv < ke, own_f = s >= kb && s < ke;
        const bool zlo = kv == 0, zhi = kv == nz - 1;
        // ---- 1. velocities on the extended region
        if (ok) {
            for (int e = threadIdx.x; e < EN; e += NT) {
                const int ex = e % EW, ey = e / EW;
                const int x = i0 - 1 + ex, y = j0 - 1 + ey;
                const bool owned = ex >= 1 && ex <= TX && ey >= 1 && ey <= TY;
                float vx = 0.0f, vy = 0.0f, vz = 0.0f;
                // δVx of plane kv: x-faces 0 and nx keep their value; rows 0 and ny-1 and the
                // z-planes 0 and nz-1 are copies
                if (kv >= 0 && kv < nz && x >= 0 && x <= nx && y >= 0 && y <= ny - 1) {
                    if (zhi) {
                        vx = vxo[e];
                    } else if (!zlo) {
                        const int h = (min(max(y, 1), ny - 2) - j0 + 2) * HW + (x - i0 + XP);
                        float v = Hp[B_VX * HS + h];
                        if (x >= 1 && x <= nx - 1) {
                            float Rx = ((n._dx * (Hp[B_XX * HS + h] - Hp[B_XX * HS + h - 1]) +
                                         n._dy * (Hp[B_XY * HS + h + HW] - Hp[B_XY * HS + h])) +
                                        n._dz * (Hc[B_XZ * HS + h] - Hp[B_XZ * HS + h])) -
                                       n._dx * (Hp[B_PT * HS + h] - Hp[B_PT * HS + h - 1]);
                            Rx = Rx + Hp[B_AX * HS + h];
                            v = v + Rx * ((Hp[B_RHO * HS + h - 1] + Hp[B_RHO * HS + h]) * 0.5f);
                        }
                        vx = v;
                    }
                    if (owned && own_v && !zlo) {
                        o.dVx[gidx32(g, x, y, kv)] = vx;
                        if (kv == 1) o.dVx[gidx32(g, x, y, 0)] = vx;  // the copy into z-plane 0
                    }
                }
                // δVy of plane kv: y-faces 0 and ny keep their value; columns 0 and nx-1 and
                // the z-planes 0 and nz-1 are copies
                if (kv >= 0 && kv < nz && x >= 0 && x <= nx - 1 && y >= 0 && y <= ny) {
                    if (zhi) {
                        vy = vxo[EN + e];
                    } else if (!zlo) {
                        const int h = (y - j0 + 2) * HW + (min(max(x, 1), nx - 2) - i0 + XP);
                        float v = Hp[B_VY * HS + h];
                        if (y >= 1 && y <= ny - 1) {
                            float Ry = ((n._dy * (Hp[B_YY * HS + h] - Hp[B_YY * HS + h - HW]) +
                                         n._dx * (Hp[B_XY * HS + h + 1] - Hp[B_XY * HS + h])) +
                                        n._dz * (Hc[B_YZ * HS + h] - Hp[B_YZ * HS + h])) -
                                       n._dy * (Hp[B_PT * HS + h] - Hp[B_PT * HS + h - HW]);
                            Ry = Ry + Hp[B_AY * HS + h];
                            v = v + Ry * ((Hp[B_RHO * HS + h - HW] + Hp[B_RHO * HS + h]) * 0.5f);
                        }
                        vy = v;
                    }
                    if (owned && own_v && !zlo) {
                        o.dVy[gidx32(g, x, y, kv)] = vy;
                        if (kv == 1) o.dVy[gidx32(g, x, y, 0)] = vy;
                    }
                }
                // δVz of z-face s: faces 0 and nz keep their value; columns 0, nx-1 and rows
                // 0, ny-1 are copies
                if (s >= 0 && s <= nz && x >= 0 && x <= nx - 1 && y >= 0 && y <= ny - 1) {
                    const int h = (min(max(y, 1), ny - 2) - j0 + 2) * HW + (min(max(x, 1), nx - 2) - i0 + XP);
                    float v = Hc[B_VZ * HS + h];
                    if (s >= 1 && s <= nz - 1) {
                        float Rz = ((n._dz * (Hc[B_ZZ * HS + h] - Hp[B_ZZ * HS + h]) +
                                     n._dx * (Hc[B_XZ * HS + h + 1] - Hc[B_XZ * HS + h])) +
                                    n._dy * (Hc[B_YZ * HS + h + HW] - Hc[B_YZ * HS + h])) -
                                   n._dz * (Hc[B_PT * HS + h] - Hp[B_PT * HS + h]);
                        Rz = Rz + Hc[B_AZ * HS + h];
                        v = v + Rz * ((Hp[B_RHO * HS + h] + Hc[B_RHO * HS + h]) * 0.5f);
                    }
                    vz = v;
                    if (owned && own_f) o.dVz[gidx32(g, x, y, s)] = vz;
                }
                vxn[e] = vx;
                vyn[e] = vy;
                vzn[e] = vz;
            }
        }
        consumer_sync(NT);
        // ---- 2. u and δPt of cell plane k = s-1
        const int k = kv;
        if (ok && k >= kb && k < ke && in) {
            const float2* GM = (const float2*)(Hp + NB * HS);
            const float* AP = (const float*)((const unsigned char*)(Hp + NB * HS) + C::GSTRIDE);
            const idx_t c = gidx32(g, i, j, k);
            const float2 gm = GM[g0], gmx = GM[g0 - 1], gmy = GM[g0 - GW];
            const float Gc = gm.x, Mc = gm.y;
            const float vx = vxn[e0], vy = vyn[e0];
            const float dvx = vxn[e0 + 1] - vx;
            const float dvy = vyn[e0 + EW] - vy;
            const float dvz = vzn[e0] - vzo[e0];
            if (k == 0) {  // δVx, δVy of plane 0 are the copies of plane 1: finished next step
                pt0 = Hp[B_PT * HS + h0];
                gc0 = Gc;
                ap0 = AP[p0];
                dvz0 = dvz;
            } else {
                o.dPt[c] = Hp[B_PT * HS + h0] - n.r * Gc * (AP[p0] + ((n._dx * dvx + n._dy * dvy) + n._dz * dvz));
                if (k == 1 && kb == 0)
                    o.dPt[c - sz] = pt0 - n.r * gc0 * (ap0 + ((n._dx * dvx + n._dy * dvy) + n._dz * dvz0));
            }
            const bool kI = k >= 1 && k <= nz - 2, k1 = k >= 1;
            if (k == 1 && kb == 0) vx_m = vx, vy_m = vy;  // the z-plane 0 copies
            const float Dn = (1.0f + __fdividef(Gc, Mc)) + (EL ? gr32(Gc, n) : 0.0f);
            const float G2 = 2.0f * Gc;
            const float rDn = __fdividef(1.0f, Dn);
            if (cx && kI) o.u[0][c] = (Hp[B_XX * HS + h0] + G2 * (n._dx * dvx)) * rDn;
            if (cy && kI) o.u[1][c] = (Hp[B_YY * HS + h0] + G2 * (n._dy * dvy)) * rDn;
            if (czz) o.u[2][c] = (Hp[B_ZZ * HS + h0] + G2 * (n._dz * dvz)) * rDn;
            if (cxy && kI) {
                const float2 a = GM[g0 - GW - 1];
                const float ag = (((a.x + gmy.x) + gmx.x) + Gc) * 0.25f;
                const float am = (((a.y + gmy.y) + gmx.y) + Mc) * 0.25f;
                const float sh = 0.5f * (n._dy * (vx - vxn[e0 - EW]) + n._dx * (vy - vyn[e0 - 1]));
                o.u[3][c] = __fdividef(Hp[B_XY * HS + h0] + (2.0f * ag) * sh,
                                       (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
            }
            if (cxz && k1) {
                const float ag = (((gx_m.x + g_m.x) + gmx.x) + Gc) * 0.25f;
                const float am = (((gx_m.y + g_m.y) + gmx.y) + Mc) * 0.25f;
                const float sh = 0.5f * (n._dz * (vx - vx_m) + n._dx * (vzo[e0] - vzo[e0 - 1]));
                o.u[4][c] = __fdividef(Hp[B_XZ * HS + h0] + (2.0f * ag) * sh,
                                       (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
            }
            if (cyz && k1) {
                const float ag = (((gy_m.x + g_m.x) + gmy.x) + Gc) * 0.25f;
                const float am = (((gy_m.y + g_m.y) + gmy.y) + Mc) * 0.25f;
                const float sh = 0.5f * (n._dz * (vy - vy_m) + n._dy * (vzo[e0] - vzo[e0 - EW]));
                o.u[5][c] = __fdividef(Hp[B_YZ * HS + h0] + (2.0f * ag) * sh,
                                       (1.0f + __fdividef(ag, am)) + (EL ? gr32(ag, n) : 0.0f));
            }
        }
        // this plane becomes the -z neighbour of the next
        if (ok) {
            const float2* GM = (const float2*)(Hp + NB * HS);
            vx_m = vxn[e0];
            vy_m = vyn[e0];
            g_m = GM[g0];
            gx_m = GM[g0 - 1];
            gy_m = GM[g0 - GW];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[(t + R - 1) % R]);  // stage t-1 is no longer read
    }
}

// Tile configurations (TY, R, blocks per SM). Shared memory per block: 8x3 104 KB,
// 4x3 67 KB, 4x4 87 KB.
struct FTile {
    int ty, r, minb;
};
constexpr FTile kFTiles[] = {{8, 3, 2}, {4, 3, 3}, {4, 4, 2}};
constexpr int kNumFTiles = (int)(sizeof(kFTiles) / sizeof(kFTiles[0]));

template <bool EL, int Q>
cudaError_t launch_f(const Geom& g, const Mixed32& m, const Out& o, const Num32& n, int kz, int* err, cudaStream_t s) {
    constexpr FTile f = kFTiles[Q];
    using C = Cfg<f.ty>;
    Maps maps;
    memset(&maps, 0, sizeof(maps));
    const void* hsrc[NB] = {m.dVx, m.dVy, m.dVz, m.dtxx, m.dtyy, m.dtzz, m.dtxy,
                            m.dtxz, m.dtyz, m.dPt, m.dtRho, m.aVx, m.aVy, m.aVz};
    for (int q = 0; q < NB; ++q)
        if (!encode_field(&maps.h[q], hsrc[q], g, 4, HW, C::HH)) return cudaErrorInvalidValue;
    if (!encode_field(&maps.gm, m.GM, g, 8, GW, C::GH)) return cudaErrorInvalidValue;
    if (!encode_field(&maps.ap, m.aP, g, 4, TX, f.ty)) return cudaErrorInvalidValue;
    const size_t smem = 128 + (size_t)f.r * C::SLOT + C::VBUF + 2 * f.r * sizeof(uint64_t);
    static bool attr[64] = {};  // per device: the opt-in to more than 48 KB of shared memory
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k3_corrBA_zs<EL, f.ty, f.r, f.minb>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    if (kz <= 0) kz = 64;
    if (kz < 2) kz = 2;  // plane 0's δPt is finished at plane 1 by the same block
    const dim3 grid((g.nx + TX - 1) / TX, (g.ny + f.ty - 1) / f.ty, (g.nz + kz - 1) / kz);
    k3_corrBA_zs<EL, f.ty, f.r, f.minb><<<grid, 32 * (f.ty + 1), smem, s>>>(maps, g, o, n, kz, err);
    return cudaGetLastError();
}

template <bool EL>
cudaError_t launch_f_form(int tile, const Geom& g, const Mixed32& m, const Out& o, const Num32& n, int kz, int* err,
                          cudaStream_t s) {
    switch (tile) {
        case 0: return launch_f<EL, 0>(g, m, o, n, kz, err, s);
        case 1: return launch_f<EL, 1>(g, m, o, n, kz, err, s);
        case 2: return launch_f<EL, 2>(g, m, o, n, kz, err, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace zf32

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

cudaError_t launch_corr_BA32_zs(int v, int tile, const Geom& g, const Mixed32& m, const Mixed32& out, const Num& n,
                                int kz, int* err, cudaStream_t s) {
    zf32::Out o{out.dPt, out.dVx, out.dVy, out.dVz, {out.dtxx, out.dtyy, out.dtzz, out.dtxy, out.dtxz, out.dtyz}};
    for (float* p : {o.dPt, o.dVx, o.dVy, o.dVz, o.u[0], o.u[1], o.u[2], o.u[3], o.u[4], o.u[5]})
        if (!p) return cudaErrorInvalidValue;
    if (v == VE3D_PERF) return zf32::launch_f_form<true>(tile, g, m, o, num32(n), kz, err, s);
    if (v == V3D) return zf32::launch_f_form<false>(tile, g, m, o, num32(n), kz, err, s);
    return cudaErrorInvalidValue;
}

int zfused32_num_configs() { return zf32::kNumFTiles; }

cudaError_t launch_corr_B32(int v, const Geom& g, const Mixed32& m, const Num& n, cudaStream_t s) {
    if (v != VE3D_PERF && v != V3D) return cudaErrorInvalidValue;
    const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nz + 1), blk(32, 8, 1);
    k3_corrB<<<grid, blk, 0, s>>>(g, m, num32(n));
    return cudaGetLastError();
}

}  // namespace pts
