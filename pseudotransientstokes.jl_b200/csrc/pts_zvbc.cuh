// pts_zvbc.cuh -- compute_V! + the free-slip bc copies (3D) as a z-marching kernel whose
// input planes the tensor-memory accelerator (TMA) stages in shared memory. A template over
// the precision: the FP64 instantiation (pts_zstage.cu, --fmad=false) is the reference's
// compute_V! operand for operand (Stokes3D_ve_perf.jl:83-88, 202-207; the role form of
// Stokes3D_ve_multixpu.jl:79-91 with PERF = false); the FP32 one (pts_kernels32.cu) is the
// δ-form sweep of the mixed path, whose residual carries the FP64 source aV.
//
// A CTA owns 32 x TY face columns (one warp per y-row, one face per lane, faces i in
// [0, nx], j in [0, ny]) and marches through a chunk of z-planes. Stage s of the ring:
//   halo boxes (rows j0-1 .. j0+TY, columns from i0-16/sizeof(T)):
//       τxx(s) τyy(s) τxy(s) Pt(s) dτ_Rho(s) τxz(s+1) τyz(s+1)
//   point boxes (the 32 x TY faces):
//       Vx(s) Vy(s) Vz(s+1) τzz(s+1) Pt(s+1) dτ_Rho(s+1) [aVx(s) aVy(s) aVz(s+1)]
// At step s a thread updates Vx and Vy of z-plane s and Vz of z-face s+1; what they need of
// plane s that stage s does not hold (τxz, τyz, τzz, Pt, dτ_Rho at its own face) it carries
// in registers from stage s-1, where it came as "s+1". Every face is written only by its
// own thread and the bc copies write faces no thread reads, so the update is in place.
// A producer warp (PW) or thread 0 keeps R-1 stages in flight; waits are bounded (pts_tma.cuh).
#pragma once
#include "pts_internal.h"
#include "pts_tma.cuh"

namespace pts {
namespace zvbc {

using namespace tma;
constexpr int TX = 32;
constexpr int NHV = 7;  // halo-box arrays

template <typename T>
struct NumV {
    T dx, dy, dz, _dx, _dy, _dz, half;
};

// The fields of one precision: halo group, then point group (sources last, may be null).
template <typename T>
struct ArgsV {
    T *Vx, *Vy, *Vz;
    const T* aV[3];  // δ-form momentum sources (FP32 sweep) or null
};

struct alignas(64) MapsV {
    CUtensorMap h[NHV];  // τxx τyy τxy Pt dτ_Rho τxz(+1) τyz(+1)
    CUtensorMap p[9];    // Vx Vy Vz(+1) τzz(+1) Pt(+1) dτ_Rho(+1) [aVx aVy aVz(+1)]
};

template <typename T, int TY, bool SRC>
struct CfgV {
    static constexpr int XP = 16 / (int)sizeof(T);  // halo box starts XP columns left of the tile
    static constexpr int HW = TX + 2 * XP;
    static constexpr int HH = TY + 2;
    static constexpr int HBOX = HW * HH * (int)sizeof(T);
    static constexpr int HSTRIDE = (HBOX + 127) / 128 * 128;
    static constexpr int NP = SRC ? 9 : 6;
    static constexpr int PBOX = TX * TY * (int)sizeof(T);
    static constexpr int SLOT = NHV * HSTRIDE + NP * PBOX;
};

template <typename T, int TY, bool SRC, int R>
__device__ __forceinline__ void issue_v(const MapsV& maps, unsigned char* smem, uint64_t* full, int t, int i0, int j0,
                                        int kb) {
    using C = CfgV<T, TY, SRC>;
    const int slot = t % R, s = kb - 1 + t;
    unsigned char* base = smem + (size_t)slot * C::SLOT;
    mbar_expect_tx(&full[slot], NHV * C::HBOX + C::NP * C::PBOX);
#pragma unroll
    for (int q = 0; q < NHV; ++q)
        tma_load3(base + q * C::HSTRIDE, &maps.h[q], i0 - C::XP, j0 - 1, q < 5 ? s : s + 1, &full[slot]);
    unsigned char* pb = base + NHV * C::HSTRIDE;
    // point group: Vx(s) Vy(s) then the "+1" arrays; the sources aVx(s) aVy(s) aVz(s+1)
    constexpr int zoff[9] = {0, 0, 1, 1, 1, 1, 0, 0, 1};
#pragma unroll
    for (int q = 0; q < C::NP; ++q) tma_load3(pb + q * C::PBOX, &maps.p[q], i0, j0, s + zoff[q], &full[slot]);
}

template <int R>
__device__ __forceinline__ void drain_v(uint64_t* full, int from, int issued, int* err) {
    for (int t = (from > issued - R ? from : issued - R); t < issued; ++t)
        if (t >= 0 && !mbar_wait(&full[t % R], (t / R) & 1)) {
            atomicExch(err, 1);
            return;
        }
}

// One derivative: _h*d (perf form) or d/h (role form).
template <typename T, bool PERF>
__device__ __forceinline__ T dsv(T d, T h, T ih) {
    return PERF ? (ih * d) : (d / h);
}

template <typename T>
__device__ __forceinline__ void copies(T* A, idx_t c, T v, int a, int alo, int ahi, idx_t sa, int b, int blo, int bhi,
                                       idx_t sb) {
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

template <typename T, bool PERF, bool SRC, int TY, int R, bool PW, int MINB>
__global__ void __launch_bounds__(32 * (TY + (PW ? 1 : 0)), MINB)
    k3_V_bc_zs(const __grid_constant__ MapsV maps, Geom g, ArgsV<T> a, NumV<T> n, int kz, int* err) {
    using C = CfgV<T, TY, SRC>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* full = (uint64_t*)(smem + (size_t)R * C::SLOT);
    uint64_t* empty = full + R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int kb = blockIdx.z * kz;
    const int ke = min(kb + kz, g.nz);
    const int nst = ke - kb + 1;  // stages kb-1 .. ke-1
    if (threadIdx.x == 0) {
        for (int q = 0; q < R; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], TY);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (PW && warp == TY) {  // producer warp: one lane issues every copy, R stages ahead
        if (lane != 0) return;
        for (int q = 0; q < NHV; ++q) prefetch_map(&maps.h[q]);
        for (int q = 0; q < C::NP; ++q) prefetch_map(&maps.p[q]);
        int issued = 0;
        for (int t = 0; t < nst; ++t) {
            if (t >= R && !mbar_wait(&empty[t % R], (t / R - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            issue_v<T, TY, SRC, R>(maps, smem, full, t, i0, j0, kb);
            issued = t + 1;
        }
        drain_v<R>(full, 0, issued, err);
        return;
    }
    // without a producer warp, thread 0 issues the copies between its own steps
    const bool prod = !PW && threadIdx.x == 0;
    int issued = 0;
    if (prod) {
        for (int q = 0; q < NHV; ++q) prefetch_map(&maps.h[q]);
        for (int q = 0; q < C::NP; ++q) prefetch_map(&maps.p[q]);
        for (; issued < R - 1 && issued < nst; ++issued) issue_v<T, TY, SRC, R>(maps, smem, full, issued, i0, j0, kb);
    }
    const int i = i0 + lane, j = j0 + warp;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in = i <= nx && j <= ny;
    // the source faces of each component (their tangential indices in the interior)
    const bool fx = in && j >= 1 && j <= ny - 2, ux = fx && i >= 1 && i <= nx - 1;
    const bool fy = in && i >= 1 && i <= nx - 2, uy = fy && j >= 1 && j <= ny - 1;
    const bool fz = in && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
    // faces whose free-slip copies do not depend on the plane: Vx next to a y-boundary, Vy next
    // to an x-boundary, every Vz with a copy (the others copy only on the planes next to a
    // z-boundary)
    const bool ex = j == 1 || j == ny - 2, ey = i == 1 || i == nx - 2, ez = ex || ey;
    const int hc = (warp + 1) * C::HW + (lane + C::XP);
    const int pc = warp * TX + lane;
    constexpr int PS = TX * TY;
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;
    idx_t c = gidx32(g, i, j, kb) - sz;  // this column at plane s = kb-1+t (advanced per step)
    T txz_m = T(0), tyz_m = T(0), tzz_m = T(0), pt_m = T(0), dr_m = T(0);  // plane s at the face, from stage s-1
    int t = 0;
    for (; t < nst; ++t, c += sz) {
        const int slot = t % R, s = kb - 1 + t;
        if (prod && issued < nst) {
            if (issued >= R && !mbar_wait(&empty[issued % R], (issued / R - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            issue_v<T, TY, SRC, R>(maps, smem, full, issued, i0, j0, kb);
            ++issued;
        }
        if (!mbar_wait(&full[slot], (t / R) & 1)) {
            atomicExch(err, 1);
            break;
        }
        const T* H = (const T*)(smem + (size_t)slot * C::SLOT);
        constexpr int HS = C::HSTRIDE / (int)sizeof(T);
        const T* hxx = H;
        const T* hyy = H + HS;
        const T* hxy = H + 2 * HS;
        const T* hP = H + 3 * HS;
        const T* hR = H + 4 * HS;
        const T* hxz = H + 5 * HS;  // τxz of plane s+1
        const T* hyz = H + 6 * HS;  // τyz of plane s+1
        const T* P = H + NHV * HS;
        const T txz_p = hxz[hc], tyz_p = hyz[hc];
        const T tzz_p = P[3 * PS + pc], pt_p = P[4 * PS + pc], dr_p = P[5 * PS + pc];
        if (t > 0 && in) {
            const bool kI = s >= 1 && s <= nz - 2, zedge = s == 1 || s == nz - 2;
            // Vx of plane s (Stokes3D_ve_perf.jl:84, @inn: i in [1,nx-1], j in [1,ny-2], k in [1,nz-2])
            if (fx && kI) {
                T v = P[pc];
                if (ux) {
                    T Rx = ((dsv<T, PERF>(hxx[hc] - hxx[hc - 1], n.dx, n._dx) +
                             dsv<T, PERF>(hxy[hc + C::HW] - hxy[hc], n.dy, n._dy)) +
                            dsv<T, PERF>(txz_p - txz_m, n.dz, n._dz)) -
                           dsv<T, PERF>(hP[hc] - hP[hc - 1], n.dx, n._dx);
                    if (SRC) Rx = Rx + P[6 * PS + pc];
                    v = v + Rx * ((hR[hc - 1] + hR[hc]) * n.half);
                    a.Vx[c] = v;
                }
                if (ex || zedge) copies(a.Vx, c, v, j, 1, ny - 2, sy, s, 1, nz - 2, sz);
            }
            // Vy of plane s (i in [1,nx-2], j in [1,ny-1], k in [1,nz-2])
            if (fy && kI) {
                T v = P[PS + pc];
                if (uy) {
                    T Ry = ((dsv<T, PERF>(hyy[hc] - hyy[hc - C::HW], n.dy, n._dy) +
                             dsv<T, PERF>(hxy[hc + 1] - hxy[hc], n.dx, n._dx)) +
                            dsv<T, PERF>(tyz_p - tyz_m, n.dz, n._dz)) -
                           dsv<T, PERF>(hP[hc] - hP[hc - C::HW], n.dy, n._dy);
                    if (SRC) Ry = Ry + P[7 * PS + pc];
                    v = v + Ry * ((hR[hc - C::HW] + hR[hc]) * n.half);
                    a.Vy[c] = v;
                }
                if (ey || zedge) copies(a.Vy, c, v, i, 1, nx - 2, sx, s, 1, nz - 2, sz);
            }
        }
        // Vz of z-face s+1 (i in [1,nx-2], j in [1,ny-2], k in [1,nz-1]); the first chunk also
        // makes the copies of z-face 0
        if (fz && (t > 0 || kb == 0)) {
            const int kf = s + 1;
            const idx_t cz = c + sz;
            T v = P[2 * PS + pc];
            if (kf >= 1 && kf <= nz - 1) {
                T Rz = ((dsv<T, PERF>(tzz_p - tzz_m, n.dz, n._dz) +
                         dsv<T, PERF>(hxz[hc + 1] - txz_p, n.dx, n._dx)) +
                        dsv<T, PERF>(hyz[hc + C::HW] - tyz_p, n.dy, n._dy)) -
                       dsv<T, PERF>(pt_p - pt_m, n.dz, n._dz);
                if (SRC) Rz = Rz + P[8 * PS + pc];
                v = v + Rz * ((dr_m + dr_p) * n.half);
                a.Vz[cz] = v;
            }
            if (ez) copies(a.Vz, cz, v, i, 1, nx - 2, sx, j, 1, ny - 2, sy);
        }
        txz_m = txz_p, tyz_m = tyz_p, tzz_m = tzz_p, pt_m = pt_p, dr_m = dr_p;
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
    }
    if (prod) drain_v<R>(full, t, issued, err);
}

// Tensor maps of one launch; `hsrc` and `psrc` in the order of MapsV.
template <typename T, int TY, bool SRC>
bool make_maps(MapsV* m, const Geom& g, const void* const hsrc[NHV], const void* const psrc[9]) {
    using C = CfgV<T, TY, SRC>;
    for (int q = 0; q < NHV; ++q)
        if (!encode_field(&m->h[q], hsrc[q], g, (int)sizeof(T), C::HW, C::HH)) return false;
    for (int q = 0; q < C::NP; ++q)
        if (!encode_field(&m->p[q], psrc[q], g, (int)sizeof(T), TX, TY)) return false;
    return true;
}

template <typename T, bool PERF, bool SRC, int TY, int R, bool PW, int MINB>
cudaError_t launch_v(const Geom& g, const MapsV& maps, const ArgsV<T>& a, const NumV<T>& n, int kz, int* err,
                     cudaStream_t s) {
    using C = CfgV<T, TY, SRC>;
    const size_t smem = 128 + (size_t)R * C::SLOT + 2 * R * sizeof(uint64_t);
    static bool attr[64] = {};  // per device: the opt-in to more than 48 KB of shared memory
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k3_V_bc_zs<T, PERF, SRC, TY, R, PW, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    if (kz <= 0) kz = 32;
    const dim3 grid((g.nx + 1 + TX - 1) / TX, (g.ny + 1 + TY - 1) / TY, (g.nz + kz - 1) / kz);
    k3_V_bc_zs<T, PERF, SRC, TY, R, PW, MINB><<<grid, 32 * (TY + (PW ? 1 : 0)), smem, s>>>(maps, g, a, n, kz, err);
    return cudaGetLastError();
}

}  // namespace zvbc
}  // namespace pts
