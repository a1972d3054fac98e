// pts_zstage.cu -- compute_Pt_τ! (3D) as a z-marching kernel whose input planes are
// staged in shared memory by the tensor-memory accelerator (TMA).
//
// Reference: compute_Pt_τ! (scripts/stokes_3D/Stokes3D_ve_perf.jl:51-78) and the role
// pair compute_P! + compute_τ! (Stokes3D_ve_multixpu.jl:57-77). The arithmetic is the
// one-thread-per-point kernel's (pts_expr64.cuh, --fmad=false), operand for operand, so
// the result is the same bits; only the way the operands reach the threads differs.
//
// Why: the one-thread-per-point kernel issues ~870 instructions per cell, half of them
// address, bounds and constant-bank work around its ~50 scalar loads, and its memory
// parallelism is capped by its registers. Here
//  * a CTA owns a 32 x TY tile of cells (one warp per y-row, one cell per lane) and marches
//    through a chunk of z-planes;
//  * one producer warp issues, per plane, one 3D tensor copy per input array into a ring of
//    R shared-memory slots (completion on an mbarrier per slot), so the bytes in flight do
//    not depend on registers;
//  * consumers read their operands from shared memory at compile-time offsets and carry
//    the values of the previous plane (the -z neighbours) in registers, so each input value
//    crosses HBM once and each cell reads 30 shared-memory words;
//  * results go straight to global memory (every cell writes only its own Pt and τ, which
//    no other CTA reads in this launch, so the update is in place).
//
// Slot layout of plane s (one tensor copy per array, zero fill outside the array):
//   halo group, box (TX+4) x (TY+2) at (i0-2, j0-1):  Vx(s), Vy(s), Gdτ(s), Mus(s), Vz(s+1)
//   point group, box TX x TY at (i0, j0):             Pt, τxx..τyz [, τxx_o..τyz_o] at s
// The halo box starts two columns left of the tile so that its x offset stays a multiple
// of 16 bytes (the TMA rule); the columns i0-1 .. i0+TX and rows j0-1 .. j0+TY are used.
// The chunk's first stage is plane kb-1, halo group only: it primes the carried registers.
//
// Waits are bounded (2 s of %globaltimer): a wait that gives up sets the context's error
// flag, the producer still waits (bounded) for every copy it issued, and the kernel ends.
// Every copy lands in the issuing CTA's shared memory alone; every tensor map covers this
// GPU's own fields.
#include <cstring>

#include "pts_expr64.cuh"
#include "pts_internal.h"
#include "pts_tma.cuh"
#include "pts_zvbc.cuh"

namespace pts {
namespace zs {

using namespace expr;
using namespace tma;

constexpr int TX = 32;           // tile width: one lane per cell
constexpr int NH = 5;            // halo-group arrays
constexpr int NPMAX = 13;        // point-group arrays (visco-elastic)

struct alignas(64) Maps {
    CUtensorMap h[NH];     // Vx Vy Gdτ Mus Vz
    CUtensorMap p[NPMAX];  // Pt τxx τyy τzz τxy τxz τyz [τ_o x6]
};

template <int TY, bool EL>
struct Cfg {
    static constexpr int HW = TX + 4;  // halo box width (elements)
    static constexpr int HH = TY + 2;  // halo box rows
    static constexpr int HBOX = HW * HH * 8;
    static constexpr int HSTRIDE = (HBOX + 127) / 128 * 128;
    static constexpr int NP = EL ? 13 : 7;
    static constexpr int PBOX = TX * TY * 8;
    static constexpr int SLOT = NH * HSTRIDE + NP * PBOX;
};

// The copies of stage t (plane kb-1+t) into its ring slot, completion on full[slot]; one
// thread issues them. Stage 0 brings the halo group only (it primes the carried registers).
template <bool EL, int TY, int R>
__device__ __forceinline__ void issue_stage(const Maps& maps, unsigned char* smem, uint64_t* full, int t, int i0,
                                            int j0, int kb) {
    using C = Cfg<TY, EL>;
    const int slot = t % R, s = kb - 1 + t;
    unsigned char* base = smem + (size_t)slot * C::SLOT;
    mbar_expect_tx(&full[slot], NH * C::HBOX + (t > 0 ? C::NP * C::PBOX : 0));
    tma_load3(base + 0 * C::HSTRIDE, &maps.h[0], i0 - 2, j0 - 1, s, &full[slot]);
    tma_load3(base + 1 * C::HSTRIDE, &maps.h[1], i0 - 2, j0 - 1, s, &full[slot]);
    tma_load3(base + 2 * C::HSTRIDE, &maps.h[2], i0 - 2, j0 - 1, s, &full[slot]);
    tma_load3(base + 3 * C::HSTRIDE, &maps.h[3], i0 - 2, j0 - 1, s, &full[slot]);
    tma_load3(base + 4 * C::HSTRIDE, &maps.h[4], i0 - 2, j0 - 1, s + 1, &full[slot]);
    if (t > 0) {
        unsigned char* pb = base + NH * C::HSTRIDE;
#pragma unroll
        for (int q = 0; q < C::NP; ++q) tma_load3(pb + q * C::PBOX, &maps.p[q], i0, j0, s, &full[slot]);
    }
}

// Bounded wait for every copy of stages [from, issued) to land (the CTA may not end while
// a copy into its shared memory is in flight).
template <int R>
__device__ __forceinline__ void drain(uint64_t* full, int from, int issued, int* err) {
    for (int t = (from > issued - R ? from : issued - R); t < issued; ++t)
        if (t >= 0 && !mbar_wait(&full[t % R], (t / R) & 1)) {
            atomicExch(err, 1);
            return;
        }
}

// compute_Pt_τ! over a 32 x TY tile and planes [kb, ke): TY consumer warps, and either one
// extra producer warp (PW) or thread 0 issuing the copies between its own steps (a warp's
// registers saved). R = slots in the shared-memory ring; MINB = blocks per SM the register
// allocation must allow.
template <bool EL, bool PERF, int TY, int R, bool PW, int MINB>
__global__ void __launch_bounds__(32 * (TY + (PW ? 1 : 0)), MINB)
    k3_Pt_tau_zs(const __grid_constant__ Maps maps, Geom g, Fields64 f, Num n, int kz, int store_divV, int* err) {
    using C = Cfg<TY, EL>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* full = (uint64_t*)(smem + (size_t)R * C::SLOT);
    uint64_t* empty = full + R;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int kb = blockIdx.z * kz;
    const int ke = min(kb + kz, g.nz);
    const int nst = ke - kb + 1;  // stages: plane kb-1 (halo only), then kb .. ke-1

    if (threadIdx.x == 0) {
        for (int s = 0; s < R; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], TY);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (PW && warp == TY) {
        // ---------------- producer warp: one lane issues every copy, R stages ahead
        if (lane != 0) return;
        for (int q = 0; q < NH; ++q) prefetch_map(&maps.h[q]);
        for (int q = 0; q < C::NP; ++q) prefetch_map(&maps.p[q]);
        int issued = 0;
        for (int t = 0; t < nst; ++t) {
            const int use = t / R;
            if (use > 0 && !mbar_wait(&empty[t % R], (use - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            issue_stage<EL, TY, R>(maps, smem, full, t, i0, j0, kb);
            issued = t + 1;
        }
        drain<R>(full, 0, issued, err);
        return;
    }
    // without a producer warp, thread 0 keeps R-1 stages in flight: before its step t it
    // refills the slot of stage t-1 once every warp has left that stage
    const bool prod = !PW && threadIdx.x == 0;
    int issued = 0;
    if (prod) {
        for (int q = 0; q < NH; ++q) prefetch_map(&maps.h[q]);
        for (int q = 0; q < C::NP; ++q) prefetch_map(&maps.p[q]);
        for (; issued < R - 1 && issued < nst; ++issued) issue_stage<EL, TY, R>(maps, smem, full, issued, i0, j0, kb);
    }

    // ---------------- consumers: warp = tile row, lane = tile column
    const int i = i0 + lane, j = j0 + warp;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in = i < nx && j < ny;
    // tangential conditions of each stress point that do not depend on k
    const bool jI = j >= 1 && j <= ny - 2, iI = i >= 1 && i <= nx - 2;
    const bool cx = in && jI, cy = in && iI, czz = in && iI && jI;                   // τxx, τyy, τzz
    const bool cxy = in && i >= 1 && j >= 1, cxz = in && i >= 1 && jI, cyz = in && iI && j >= 1;
    const double gdt = n.gdt;

    // halo-box offsets (elements) of this cell and its -x / -y neighbours
    const int hc = (warp + 1) * C::HW + (lane + 2);
    const int hxm = hc - 1, hym = hc - C::HW, hxp = hc + 1, hyp = hc + C::HW, hxym = hc - C::HW - 1;
    const int pc = warp * TX + lane;

    // registers carried from the previous plane (the -z neighbours)
    double vx_m, vy_m, g_m, gx_m, gy_m, m_m, mx_m, my_m;  // plane k-1
    double vz_c, vz_x, vz_y;                               // Vz at plane k: c, c-sx, c-sy

    idx_t c = gidx32(g, i, j, kb);
    const idx_t sz = (idx_t)g.pxy;
    int t = 0;
    for (; t < nst; ++t) {
        const int slot = t % R;
        if (prod && issued < nst) {  // stage t+R-1 into the slot stage t-1 leaves
            if (issued >= R && !mbar_wait(&empty[issued % R], (issued / R - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            issue_stage<EL, TY, R>(maps, smem, full, issued, i0, j0, kb);
            ++issued;
        }
        if (!mbar_wait(&full[slot], (t / R) & 1)) {
            atomicExch(err, 1);
            break;
        }
        const double* H = (const double*)(smem + (size_t)slot * C::SLOT);
        const double* hVx = H;
        const double* hVy = H + C::HSTRIDE / 8;
        const double* hG = H + 2 * (C::HSTRIDE / 8);
        const double* hM = H + 3 * (C::HSTRIDE / 8);
        const double* hVz = H + 4 * (C::HSTRIDE / 8);  // Vz of plane s+1
        const double vx = hVx[hc], vy = hVy[hc], Gc = hG[hc], Mc = hM[hc];
        const double Gx = hG[hxm], Gy = hG[hym], Mx = hM[hxm], My = hM[hym];
        const double vzn = hVz[hc], vznx = hVz[hxm], vzny = hVz[hym];
        if (t > 0 && in) {
            const int k = kb + t - 1;
            const double* P = H + NH * (C::HSTRIDE / 8);
            const double dvx = hVx[hxp] - vx;
            const double dvy = hVy[hyp] - vy;
            const double dvz = vzn - vz_c;
            if (PERF) {
                f.Pt[c] = P[pc] - n.r * Gc * ((n._dx * dvx + n._dy * dvy) + n._dz * dvz);
            } else {
                const double dv = (dvx / n.dx + dvy / n.dy) + dvz / n.dz;
                if (store_divV) f.divV[c] = dv;
                f.Pt[c] = P[pc] - n.r * Gc * dv;
            }
            const bool kI = k >= 1 && k <= nz - 2, k1 = k >= 1;
            const double* Po = P + 7 * (C::PBOX / 8);  // τ_o
            constexpr int PS = C::PBOX / 8;
            if ((cx && kI) || (cy && kI) || czz) {
                const double Gr = EL ? gr_of(Gc, gdt) : 0.0;
                const double den = EL ? ((1.0 + Gc / Mc) + Gr) : (1.0 + Gc / Mc);
                if (cx && kI)
                    f.txx[c] = tau_n_den<EL, PERF>(P[1 * PS + pc], EL ? Po[0 * PS + pc] : 0.0, Gc, Gr, den, n.dx,
                                                   n._dx, dvx);
                if (cy && kI)
                    f.tyy[c] = tau_n_den<EL, PERF>(P[2 * PS + pc], EL ? Po[1 * PS + pc] : 0.0, Gc, Gr, den, n.dy,
                                                   n._dy, dvy);
                if (czz)
                    f.tzz[c] = tau_n_den<EL, PERF>(P[3 * PS + pc], EL ? Po[2 * PS + pc] : 0.0, Gc, Gr, den, n.dz,
                                                   n._dz, dvz);
            }
            // τxy on edge (x-face i, y-face j, cell k): i in [1,nx-1], j in [1,ny-1], k in [1,nz-2]
            if (cxy && kI) {
                const double ag = (((hG[hxym] + Gy) + Gx) + Gc) * 0.25;
                const double am = (((hM[hxym] + My) + Mx) + Mc) * 0.25;
                f.txy[c] = tau_s<EL, PERF>(P[4 * PS + pc], EL ? Po[3 * PS + pc] : 0.0, ag, am, gdt, n.dy, n._dy,
                                           vx - hVx[hym], n.dx, n._dx, vy - hVy[hxm]);
            }
            // τxz on edge (x-face i, cell j, z-face k): i in [1,nx-1], j in [1,ny-2], k in [1,nz-1]
            if (cxz && k1) {
                const double ag = (((gx_m + g_m) + Gx) + Gc) * 0.25;
                const double am = (((mx_m + m_m) + Mx) + Mc) * 0.25;
                f.txz[c] = tau_s<EL, PERF>(P[5 * PS + pc], EL ? Po[4 * PS + pc] : 0.0, ag, am, gdt, n.dz, n._dz,
                                           vx - vx_m, n.dx, n._dx, vz_c - vz_x);
            }
            // τyz on edge (cell i, y-face j, z-face k): i in [1,nx-2], j in [1,ny-1], k in [1,nz-1]
            if (cyz && k1) {
                const double ag = (((gy_m + g_m) + Gy) + Gc) * 0.25;
                const double am = (((my_m + m_m) + My) + Mc) * 0.25;
                f.tyz[c] = tau_s<EL, PERF>(P[6 * PS + pc], EL ? Po[5 * PS + pc] : 0.0, ag, am, gdt, n.dz, n._dz,
                                           vy - vy_m, n.dy, n._dy, vz_c - vz_y);
            }
            c += sz;
        }
        // this plane becomes the -z neighbour of the next
        vx_m = vx, vy_m = vy, g_m = Gc, gx_m = Gx, gy_m = Gy, m_m = Mc, mx_m = Mx, my_m = My;
        vz_c = vzn, vz_x = vznx, vz_y = vzny;
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
    }
    if (prod) drain<R>(full, t, issued, err);  // copies this thread issued and nobody consumed
}

// ---- host side ----

template <bool EL, bool PERF, int TY, int R, bool PW, int MINB>
cudaError_t launch_cfg(const Geom& g, const Fields64& f, const Num& n, int kz, bool store_divV, int* err,
                       cudaStream_t s) {
    using C = Cfg<TY, EL>;
    Maps maps;
    memset(&maps, 0, sizeof(maps));
    const double* hsrc[NH] = {f.Vx, f.Vy, f.Gdt, f.Mus, f.Vz};
    for (int q = 0; q < NH; ++q)
        if (!encode_field(&maps.h[q], hsrc[q], g, 8, C::HW, C::HH)) return cudaErrorInvalidValue;
    const double* psrc[NPMAX] = {f.Pt,    f.txx,   f.tyy,   f.tzz,   f.txy,   f.txz,  f.tyz,
                                 f.txx_o, f.tyy_o, f.tzz_o, f.txy_o, f.txz_o, f.tyz_o};
    for (int q = 0; q < C::NP; ++q)
        if (!encode_field(&maps.p[q], psrc[q], g, 8, TX, TY)) return cudaErrorInvalidValue;
    const size_t smem = 128 + (size_t)R * C::SLOT + 2 * R * sizeof(uint64_t);
    static bool attr[64] = {};  // per device: the opt-in to more than 48 KB of shared memory
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k3_Pt_tau_zs<EL, PERF, TY, R, PW, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    const dim3 grid((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, (g.nz + kz - 1) / kz);
    k3_Pt_tau_zs<EL, PERF, TY, R, PW, MINB>
        <<<grid, 32 * (TY + (PW ? 1 : 0)), smem, s>>>(maps, g, f, n, kz, store_divV ? 1 : 0, err);
    return cudaGetLastError();
}

// Tile configurations: tile height TY, ring slots R, producer warp PW, blocks per SM MINB
// the registers must allow. Shared memory per block for the visco-elastic form: 32x4 with 2
// slots 45 KB (4 blocks/SM by registers), 32x8 83 KB (2), 32x6 63 KB (3). The first is the
// fastest measured at 511^3 on a B200 (5.01 ms; without the producer warp 5.07, 32x8 5.12).
struct TileCfg {
    int ty, r, pw, minb;
};
constexpr TileCfg kTiles[] = {{4, 2, 1, 4}, {4, 2, 0, 5}, {8, 2, 1, 2}, {6, 2, 1, 3}, {8, 2, 0, 2}};
constexpr int kNumTiles = (int)(sizeof(kTiles) / sizeof(kTiles[0]));

template <bool EL, bool PERF, int Q>
cudaError_t launch_q(const Geom& g, const Fields64& f, const Num& n, int kz, bool sd, int* err, cudaStream_t s) {
    constexpr TileCfg c = kTiles[Q];
    return launch_cfg<EL, PERF, c.ty, c.r, c.pw != 0, c.minb>(g, f, n, kz, sd, err, s);
}

template <bool EL, bool PERF>
cudaError_t launch_form(int cfg, const Geom& g, const Fields64& f, const Num& n, int kz, bool sd, int* err,
                        cudaStream_t s) {
    switch (cfg) {
        case 0: return launch_q<EL, PERF, 0>(g, f, n, kz, sd, err, s);
        case 1: return launch_q<EL, PERF, 1>(g, f, n, kz, sd, err, s);
        case 2: return launch_q<EL, PERF, 2>(g, f, n, kz, sd, err, s);
        case 3: return launch_q<EL, PERF, 3>(g, f, n, kz, sd, err, s);
        case 4: return launch_q<EL, PERF, 4>(g, f, n, kz, sd, err, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zs

int zstage_num_configs() { return zs::kNumTiles; }

bool zstage_tile_info(int tile, int* ty, int* ring) {
    if (tile < 0 || tile >= zs::kNumTiles) return false;
    if (ty) *ty = zs::kTiles[tile].ty;
    if (ring) *ring = zs::kTiles[tile].r;
    return true;
}

// ---- compute_V! + bc, z-staged (pts_zvbc.cuh), FP64 ----
namespace zvbc {
// Tile configurations (TY, R, producer warp PW, MINB): shared memory per block 66 KB for
// 32x8 (3 blocks/SM), 37 KB for 32x4 (6).
struct VTile {
    int ty, r, pw, minb;
};
constexpr VTile kVTiles[] = {{8, 2, 1, 3}, {8, 2, 0, 3}, {4, 2, 1, 5}, {4, 2, 0, 6}};
constexpr int kNumVTiles = (int)(sizeof(kVTiles) / sizeof(kVTiles[0]));

template <bool PERF, int Q>
cudaError_t launch64(const Geom& g, const Fields64& f, const Num& n, int kz, int* err, cudaStream_t s) {
    constexpr VTile c = kVTiles[Q];
    MapsV maps;
    memset(&maps, 0, sizeof(maps));
    const void* hsrc[NHV] = {f.txx, f.tyy, f.txy, f.Pt, f.dtRho, f.txz, f.tyz};
    const void* psrc[9] = {f.Vx, f.Vy, f.Vz, f.tzz, f.Pt, f.dtRho, nullptr, nullptr, nullptr};
    if (!make_maps<double, c.ty, false>(&maps, g, hsrc, psrc)) return cudaErrorInvalidValue;
    ArgsV<double> a{f.Vx, f.Vy, f.Vz, {nullptr, nullptr, nullptr}};
    NumV<double> nv{n.dx, n.dy, n.dz, n._dx, n._dy, n._dz, 0.5};
    return launch_v<double, PERF, false, c.ty, c.r, c.pw != 0, c.minb>(g, maps, a, nv, kz, err, s);
}

template <bool PERF>
cudaError_t launch64_form(int tile, const Geom& g, const Fields64& f, const Num& n, int kz, int* err, cudaStream_t s) {
    switch (tile) {
        case 0: return launch64<PERF, 0>(g, f, n, kz, err, s);
        case 1: return launch64<PERF, 1>(g, f, n, kz, err, s);
        case 2: return launch64<PERF, 2>(g, f, n, kz, err, s);
        case 3: return launch64<PERF, 3>(g, f, n, kz, err, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace zvbc

int zvbc_num_configs() { return zvbc::kNumVTiles; }

cudaError_t launch_V_bc_zs(int variant, int tile, const Geom& g, const Fields64& f, const Num& n, int kz, int* err,
                           cudaStream_t s) {
    switch (variant) {
        case VE3D_PERF:
        case V3D: return zvbc::launch64_form<true>(tile, g, f, n, kz, err, s);
        case VE3D: return zvbc::launch64_form<false>(tile, g, f, n, kz, err, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---- compute_Pt_τ! (2D) as a y-marching kernel with TMA-staged tiles ----
//
// Reference: compute_Pt_τ! of scripts/Stokes2D_ve_perf.jl:34-53 and the role pairs
// compute_P! + compute_τ! of Stokes2D_ve.jl:35-50 and Stokes2D.jl:33-44, evaluated exactly
// as the one-thread-per-cell kernel (pt_tau_2d in pts_kernels64.cu) evaluates them,
// operand for operand, so the result is the same bits. A CTA owns a 32-column strip and a
// chunk of `ky` rows, which it walks in tiles of TY rows: one consumer warp per row, one
// cell per lane. Per tile one producer warp issues one 3D tensor copy per input array into
// a ring of R shared-memory slots:
//   halo group, box (TX+4) x (TY+2) at (i0-2, j0-1): Vx, Vy, Gdτ, Mus
//   point group, box TX x TY at (i0, j0):            Pt, τxx, τyy, τxy [, τxx_o, τyy_o, τxy_o]
// (the halo box starts two columns left of the tile, the 16-byte rule for the x offset).
// Every cell writes only its own Pt and τ: the update is in place. Waits are bounded.
namespace ys2 {
using namespace expr;
using namespace tma;
constexpr int TX = 32;
constexpr int HW = TX + 4;
constexpr int NH = 4;

struct alignas(64) Maps {
    CUtensorMap h[NH];  // Vx Vy Gdτ Mus
    CUtensorMap p[7];   // Pt τxx τyy τxy [τxx_o τyy_o τxy_o]
};

template <int TY, bool EL>
struct Cfg {
    static constexpr int HH = TY + 2;
    static constexpr int HBOX = HW * HH * 8;
    static constexpr int HSTRIDE = (HBOX + 127) / 128 * 128;
    static constexpr int NP = EL ? 7 : 4;
    static constexpr int PBOX = TX * TY * 8;
    static constexpr int SLOT = NH * HSTRIDE + NP * PBOX;
};

template <bool EL, int TY, int R>
__device__ __forceinline__ void issue_y(const Maps& maps, unsigned char* smem, uint64_t* full, int t, int i0, int jb) {
    using C = Cfg<TY, EL>;
    const int slot = t % R, j0 = jb + t * TY;
    unsigned char* base = smem + (size_t)slot * C::SLOT;
    mbar_expect_tx(&full[slot], NH * C::HBOX + C::NP * C::PBOX);
#pragma unroll
    for (int q = 0; q < NH; ++q) tma_load3(base + q * C::HSTRIDE, &maps.h[q], i0 - 2, j0 - 1, 0, &full[slot]);
#pragma unroll
    for (int q = 0; q < C::NP; ++q) tma_load3(base + NH * C::HSTRIDE + q * C::PBOX, &maps.p[q], i0, j0, 0, &full[slot]);
}

template <int VAR, int TY, int R, int MINB>
__global__ void __launch_bounds__(32 * (TY + 1), MINB)
    k2_Pt_tau_ys(const __grid_constant__ Maps maps, Geom g, Fields64 f, Num n, int ky, int store_divV, int* err) {
    constexpr bool EL = VAR != V2D, PERF = VAR == VE2D_PERF;
    using C = Cfg<TY, EL>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* full = (uint64_t*)(smem + (size_t)R * C::SLOT);
    uint64_t* empty = full + R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * TX, jb = blockIdx.y * ky;
    const int je = min(jb + ky, g.ny);
    const int nst = (je - jb + TY - 1) / TY;
    if (threadIdx.x == 0) {
        for (int q = 0; q < R; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], TY);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == TY) {  // producer warp
        if (lane != 0) return;
        for (int q = 0; q < NH; ++q) prefetch_map(&maps.h[q]);
        for (int q = 0; q < C::NP; ++q) prefetch_map(&maps.p[q]);
        int issued = 0;
        for (int t = 0; t < nst; ++t) {
            if (t >= R && !mbar_wait(&empty[t % R], (t / R - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            issue_y<EL, TY, R>(maps, smem, full, t, i0, jb);
            issued = t + 1;
        }
        for (int t = (issued > R ? issued - R : 0); t < issued; ++t)
            if (!mbar_wait(&full[t % R], (t / R) & 1)) {
                atomicExch(err, 1);
                break;
            }
        return;
    }
    const int nx = g.nx;
    const int i = i0 + lane;
    const int hc = (warp + 1) * HW + (lane + 2);
    const int pc = warp * TX + lane;
    constexpr int PS = TX * TY;
    constexpr int HS = C::HSTRIDE / 8;
    for (int t = 0; t < nst; ++t) {
        const int slot = t % R;
        if (!mbar_wait(&full[slot], (t / R) & 1)) {
            atomicExch(err, 1);
            return;
        }
        const int j = jb + t * TY + warp;
        if (i < nx && j < je) {
            const double* H = (const double*)(smem + (size_t)slot * C::SLOT);
            const double* hVx = H;
            const double* hVy = H + HS;
            const double* hG = H + 2 * HS;
            const double* hM = H + 3 * HS;
            const double* P = H + NH * HS;
            const idx_t c = gidx32(g, i, j, 0);
            const double vx = hVx[hc], vy = hVy[hc];
            const double dvx = hVx[hc + 1] - vx;
            const double dvy = hVy[hc + HW] - vy;
            const double Gc = hG[hc];
            if (VAR == VE2D_PERF) {
                f.Pt[c] = P[pc] - n.r * Gc * (n._dx * dvx + n._dy * dvy);
            } else {
                const double dv = dvx / n.dx + dvy / n.dy;
                if (store_divV) f.divV[c] = dv;
                f.Pt[c] = P[pc] - n.r * Gc * dv;
            }
            const double Mc = hM[hc];
            if (VAR == V2D) {
                const double den = Gc / Mc + 1.0;
                f.txx[c] = (P[PS + pc] + ((2.0 * Gc) * dvx) / n.dx) / den;
                f.tyy[c] = (P[2 * PS + pc] + ((2.0 * Gc) * dvy) / n.dy) / den;
            } else {
                const double Gr = gr_of(Gc, n.gdt);
                const double ex = PERF ? n._dx * dvx : dvx / n.dx;
                const double ey = PERF ? n._dy * dvy : dvy / n.dy;
                const double den = (1.0 + Gc / Mc) + Gr;
                f.txx[c] = ((P[PS + pc] + P[4 * PS + pc] * Gr) + (2.0 * Gc) * ex) / den;
                f.tyy[c] = ((P[2 * PS + pc] + P[5 * PS + pc] * Gr) + (2.0 * Gc) * ey) / den;
            }
            // τxy on the vertex (x-face i, y-face j): i in [1,nx-1], j in [1,ny-1]
            if (i >= 1 && j >= 1) {
                const double ag = (((hG[hc - HW - 1] + hG[hc - HW]) + hG[hc - 1]) + Gc) * 0.25;
                const double am = (((hM[hc - HW - 1] + hM[hc - HW]) + hM[hc - 1]) + Mc) * 0.25;
                const double d1 = vx - hVx[hc - HW];  // @d_yi(Vx)
                const double d2 = vy - hVy[hc - 1];   // @d_xi(Vy)
                if (VAR == V2D) {
                    f.txy[c] = (P[3 * PS + pc] + (2.0 * ag) * (0.5 * (d1 / n.dy + d2 / n.dx))) / (ag / am + 1.0);
                } else if (VAR == VE2D) {
                    const double Gr = gr_of(ag, n.gdt);
                    f.txy[c] = ((P[3 * PS + pc] + P[6 * PS + pc] * Gr) + (2.0 * ag) * (0.5 * (d1 / n.dy + d2 / n.dx))) /
                               ((1.0 + ag / am) + Gr);
                } else {
                    const double Gr = gr_of(ag, n.gdt);
                    f.txy[c] = ((P[3 * PS + pc] + P[6 * PS + pc] * Gr) + ((2.0 * ag) * 0.5) * (n._dy * d1 + n._dx * d2)) /
                               ((1.0 + ag / am) + Gr);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
    }
}

// Tile configurations (TY, R, blocks per SM); shared memory for the visco-elastic form:
// 32x8 with 2 slots 52 KB, 32x4 with 3 slots 42 KB, 32x8 with 3 slots 78 KB, 32x16 2 slots 97 KB.
struct YTile {
    int ty, r, minb;
};
constexpr YTile kYTiles[] = {{8, 2, 3}, {4, 3, 4}, {8, 3, 2}, {16, 2, 1}};
constexpr int kNumYTiles = (int)(sizeof(kYTiles) / sizeof(kYTiles[0]));

template <int VAR, int Q>
cudaError_t launch_y(const Geom& g, const Fields64& f, const Num& n, int ky, bool sd, int* err, cudaStream_t s) {
    constexpr YTile y = kYTiles[Q];
    constexpr bool EL = VAR != V2D;
    using C = Cfg<y.ty, EL>;
    Maps maps;
    memset(&maps, 0, sizeof(maps));
    const double* hsrc[NH] = {f.Vx, f.Vy, f.Gdt, f.Mus};
    for (int q = 0; q < NH; ++q)
        if (!encode_field(&maps.h[q], hsrc[q], g, 8, HW, C::HH)) return cudaErrorInvalidValue;
    const double* psrc[7] = {f.Pt, f.txx, f.tyy, f.txy, f.txx_o, f.tyy_o, f.txy_o};
    for (int q = 0; q < C::NP; ++q)
        if (!encode_field(&maps.p[q], psrc[q], g, 8, TX, y.ty)) return cudaErrorInvalidValue;
    const size_t smem = 128 + (size_t)y.r * C::SLOT + 2 * y.r * sizeof(uint64_t);
    static bool attr[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k2_Pt_tau_ys<VAR, y.ty, y.r, y.minb>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    if (ky <= 0) ky = 128;
    ky = (ky + y.ty - 1) / y.ty * y.ty;  // whole tiles per chunk
    const dim3 grid((g.nx + TX - 1) / TX, (g.ny + ky - 1) / ky, 1);
    k2_Pt_tau_ys<VAR, y.ty, y.r, y.minb><<<grid, 32 * (y.ty + 1), smem, s>>>(maps, g, f, n, ky, sd ? 1 : 0, err);
    return cudaGetLastError();
}

template <int VAR>
cudaError_t launch_y_form(int tile, const Geom& g, const Fields64& f, const Num& n, int ky, bool sd, int* err,
                          cudaStream_t s) {
    switch (tile) {
        case 0: return launch_y<VAR, 0>(g, f, n, ky, sd, err, s);
        case 1: return launch_y<VAR, 1>(g, f, n, ky, sd, err, s);
        case 2: return launch_y<VAR, 2>(g, f, n, ky, sd, err, s);
        case 3: return launch_y<VAR, 3>(g, f, n, ky, sd, err, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace ys2

int ystage_num_configs() { return ys2::kNumYTiles; }

cudaError_t launch_Pt_tau_ys(int variant, int tile, const Geom& g, const Fields64& f, const Num& n, int ky,
                             bool store_divV, int* err, cudaStream_t s) {
    switch (variant) {
        case V2D: return ys2::launch_y_form<V2D>(tile, g, f, n, ky, store_divV, err, s);
        case VE2D: return ys2::launch_y_form<VE2D>(tile, g, f, n, ky, store_divV, err, s);
        case VE2D_PERF: return ys2::launch_y_form<VE2D_PERF>(tile, g, f, n, ky, false, err, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_Pt_tau_zs(int variant, int cfg, const Geom& g, const Fields64& f, const Num& n, int kz,
                             bool store_divV, int* err, cudaStream_t s) {
    if (kz <= 0) kz = 32;
    switch (variant) {
        case VE3D_PERF: return zs::launch_form<true, true>(cfg, g, f, n, kz, false, err, s);
        case V3D: return zs::launch_form<false, true>(cfg, g, f, n, kz, false, err, s);
        case VE3D: return zs::launch_form<true, false>(cfg, g, f, n, kz, store_divV, err, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pts
