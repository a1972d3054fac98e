// pts_fused3d.cuh -- single-pass 3D PT iteration kernel (template; instantiated by the
// FP64 and FP32 translation units).
//
// One launch does the velocity update of iteration n and the pressure/stress update of
// iteration n+1 ("B then A"):
//   B: V_n     = V_{n-1} + R(τ_n, Pt_n) * av(dτ_Rho), with the free-slip copies
//      (compute_V! + bc_*!, Stokes3D_ve_perf.jl:83-88,202-207)
//   A: Pt_{n+1}, τ_{n+1} from V_n (compute_Pt_τ!, Stokes3D_ve_perf.jl:69-78)
// so a PT block of m iterations is  A(1) [BA]^(m-1) B(m)  and each field crosses HBM
// once per iteration (29 arrays for the visco-elastic form: the reference's A_eff).
//
// Tiling: a CTA owns a 32 x 8 tile of unified (i,j) points and marches in z over a chunk
// of planes. B at plane s is computed for the owned faces plus a one-face ring (the faces
// A needs from the neighbours: Vx at i+1 and j-1, Vy at j+1 and i-1, Vz at i-1 and j-1);
// the ring is recomputed, not exchanged -- it costs the cheap V update (no divisions),
// never the stress update. V_n of the last three planes lives in shared memory; A at
// plane s-1 runs after B of plane s. The iteration-n inputs and the iteration-(n+1)
// outputs are different buffers (ping-pong), so recomputing a neighbour's ring never
// reads a value that neighbour already overwrote.
//
// Staging: every input plane the CTA needs ([x0-2, x0+34) x [y0-1, y0+8], i.e. tile +
// halo) is copied into shared memory by the bulk-copy engine (cp.async.bulk, one copy per
// row, completion on an mbarrier) one z-step before it is used, into rings of plane slots:
//   G1 τ_n (6), Pt_n, dτ_Rho [+ aV (3)]  4 slots  read by B (halo) and A (own point)
//   G2 V_{n-1} (3)                       2 slots  read by B
//   G3 Gdτ, Mus                          3 slots  read by A (halo -1 in x, y, z)
//   G4 τ_o (6)  [or aτ (6), aP]          2 slots  read by A (own point)
// A slot is refilled only after the CTA-wide barrier that ends the last step reading it.
// Waits on the mbarriers are bounded (2 s of %globaltimer); a timeout sets an error flag
// the host reads, and the kernel runs to completion instead of hanging.
//
// Boundaries: every face computes its own final value as the update at its tangentially
// clamped source face (walls keep their value), which is what the reference's sequence of
// whole-plane bc copies leaves there. Vx/Vy on the first and last interior z-planes
// (whose clamped source is another plane) are computed from global memory.
//
// CORR selects a defect-correction form with stress sources (no instantiation is launched:
// the mixed-precision sweeps are the two FP32 kernels of pts_kernels32.cu, which carry
// the stresses source-free): the state is a correction δ and the FP64 residuals of the
// current iterate enter as sources
//   δPt' = δPt - r*Gdτ*(aP + ∇·δV),   δτ' = (δτ + aτ + 2Gdτ*ε̇(δV)) / D,
//   δV'  = δV + (R(δτ', δPt') + aV) * av(dτ_Rho)
// which is the same PT iteration applied to (FP64 iterate + δ).
#pragma once
#include "pts_internal.h"

namespace pts {

template <typename T>
struct NumT {
    T dx, dy, dz, _dx, _dy, _dz, r, gdt;
    T two, half, one, quarter;
    int gdt_is_one;  // G*dt == 1.0 exactly: x/(G*dt) == x, the division is skipped
};

template <typename T>
struct Fused3Args {
    // iteration-n fields (read, staged)
    const T* g1[11];  // τxx τyy τzz τxy τxz τyz Pt dτ_Rho [aVx aVy aVz]
    const T* g2[3];   // Vx Vy Vz
    const T* g3[2];   // Gdτ Mus
    const T* g4[7];   // τ_o (6) | aτ (6) aP
    // iteration-(n+1) fields (written)
    T *Vx2, *Vy2, *Vz2;
    T *txx2, *tyy2, *tzz2, *txy2, *txz2, *tyz2, *Pt2;
    // ∇V of A's V (role form stores it for the check), may be null
    T* divV;
    int* err;  // set to 1 when a staging wait timed out
};

namespace fused3 {

constexpr int TX = 32, TY = 8;
constexpr int R1 = 4, R2 = 2, R3 = 3, R4 = 2;

template <typename T, bool EL, bool CORR>
struct Cfg {
    static constexpr int XPAD = 16 / (int)sizeof(T);  // 16-byte aligned box start
    static constexpr int BW = TX + 2 * XPAD;          // box width (elements)
    static constexpr int BH = TY + 2;                 // box rows y0-1 .. y0+TY
    static constexpr int BOX = BW * BH;
    static constexpr int NF1 = CORR ? 11 : 8;
    static constexpr int NF2 = 3;
    static constexpr int NF3 = 2;
    static constexpr int NF4 = CORR ? 7 : (EL ? 6 : 0);
    static constexpr int EX = TX + 2, EY = TY + 2;
    static constexpr size_t kBar = 128;
    static constexpr size_t kStage = sizeof(T) * (size_t)BOX * (R1 * NF1 + R2 * NF2 + R3 * NF3 + R4 * NF4);
    static constexpr size_t kSV = sizeof(T) * 9 * EY * EX;
    static constexpr size_t smem_bytes = kBar + kStage + kSV;
};

// ---- bulk-copy / mbarrier primitives (sm_90+; each copy lands in the issuing CTA alone) ----
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"(bytes), "r"(saddr(b))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after 2 s, records the failure and lets the kernel finish.
__device__ __forceinline__ void mbar_wait(uint64_t* b, uint32_t parity, int* err) {
    if (mbar_try(b, parity)) return;
    const uint64_t t0 = gtimer();
    while (!mbar_try(b, parity)) {
        if (gtimer() - t0 > 2000000000ull) {
            atomicExch(err, 1);
            return;
        }
    }
}

// Issue the copies of plane p of one group (nf fields) into its slot (executed by one
// warp). Rows outside the array and columns outside [0, px) are not copied.
template <typename T, int BW, int BH, int BOX>
__device__ __forceinline__ void issue_plane(const T* const* src, int nf, T* dst, uint64_t* bar, const Geom& g, int x0s,
                                            int y0r, int p, int lane) {
    const int xs = x0s < 0 ? 0 : x0s;
    const int xe = (x0s + BW) > g.px ? g.px : (x0s + BW);
    const int ys = y0r < 0 ? 0 : y0r;
    const int ye = (y0r + BH) > g.py ? g.py : (y0r + BH);
    const int nrows = (ye > ys && xe > xs && p >= 0 && p < g.pz) ? (ye - ys) : 0;
    const uint32_t rowbytes = (uint32_t)((xe - xs) * (int)sizeof(T));
    if (lane == 0) {
        fence_proxy_async();
        mbar_expect_tx(bar, (uint32_t)(nf * nrows) * rowbytes);
    }
    __syncwarp();
    for (int q = lane; q < nf * nrows; q += 32) {
        const int f = q / nrows, r = q % nrows;
        const int y = ys + r;
        bulk_g2s(dst + f * BOX + (y - y0r) * BW + (xs - x0s), src[f] + gidx(g, xs, y, p), rowbytes, bar);
    }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <typename T, bool PERF>
__device__ __forceinline__ T sc(T d, T h, T ih) {
    return PERF ? (ih * d) : (d / h);
}

template <typename T>
__device__ __forceinline__ T grel(const NumT<T>& n, T g) {
    return n.gdt_is_one ? g : g / n.gdt;
}

// Stress updates (Stokes3D_ve_perf.jl:71-76), plain or correction form.
template <typename T, bool EL, bool PERF, bool CORR>
__device__ __forceinline__ T tau_n(T t, T src, T gg, T m, const NumT<T>& n, T h, T ih, T d) {
    const T e = PERF ? (ih * d) : (d / h);
    if (CORR) {
        if (EL) return ((t + src) + (n.two * gg) * e) / ((n.one + gg / m) + grel(n, gg));
        return ((t + src) + (n.two * gg) * e) / (n.one + gg / m);
    }
    if (EL) {
        const T Gr = grel(n, gg);
        return ((t + src * Gr) + (n.two * gg) * e) / ((n.one + gg / m) + Gr);
    }
    return (t + (n.two * gg) * e) / (n.one + gg / m);
}
template <typename T, bool EL, bool PERF, bool CORR>
__device__ __forceinline__ T tau_s(T t, T src, T ag, T am, const NumT<T>& n, T h1, T ih1, T d1, T h2, T ih2, T d2) {
    const T s = PERF ? (ih1 * d1 + ih2 * d2) : (d1 / h1 + d2 / h2);
    if (CORR) {
        if (EL) return ((t + src) + (n.two * ag) * (n.half * s)) / ((n.one + ag / am) + grel(n, ag));
        return ((t + src) + (n.two * ag) * (n.half * s)) / (n.one + ag / am);
    }
    if (EL) {
        const T Gr = grel(n, ag);
        return ((t + src * Gr) + (n.two * ag) * (n.half * s)) / ((n.one + ag / am) + Gr);
    }
    return (t + (n.two * ag) * (n.half * s)) / (n.one + ag / am);
}

// ---- B from global memory (z-boundary planes): final V_n of face (i,j,k) ----
template <typename T>
__device__ __forceinline__ T ld(const T* p, int64_t i) {
    return __ldg(p + i);
}
template <typename T, bool PERF, bool CORR, int COMP>
__device__ T face_global(const Fused3Args<T>& a, const NumT<T>& n, const Geom& g, int i, int j, int k) {
    const int64_t sy = g.px, sz = g.pxy;
    const T *txx = a.g1[0], *tyy = a.g1[1], *tzz = a.g1[2], *txy = a.g1[3], *txz = a.g1[4], *tyz = a.g1[5];
    const T *Pt = a.g1[6], *dR = a.g1[7];
    if (COMP == 0) {
        const int64_t c = gidx(g, i, clampi(j, 1, g.ny - 2), clampi(k, 1, g.nz - 2));
        if (!(i >= 1 && i <= g.nx - 1)) return ld(a.g2[0], c);
        T R = ((sc<T, PERF>(ld(txx, c) - ld(txx, c - 1), n.dx, n._dx) + sc<T, PERF>(ld(txy, c + sy) - ld(txy, c), n.dy, n._dy)) +
               sc<T, PERF>(ld(txz, c + sz) - ld(txz, c), n.dz, n._dz)) -
              sc<T, PERF>(ld(Pt, c) - ld(Pt, c - 1), n.dx, n._dx);
        if (CORR) R = R + ld(a.g1[8], c);
        return ld(a.g2[0], c) + R * ((ld(dR, c - 1) + ld(dR, c)) * n.half);
    } else if (COMP == 1) {
        const int64_t c = gidx(g, clampi(i, 1, g.nx - 2), j, clampi(k, 1, g.nz - 2));
        if (!(j >= 1 && j <= g.ny - 1)) return ld(a.g2[1], c);
        T R = ((sc<T, PERF>(ld(tyy, c) - ld(tyy, c - sy), n.dy, n._dy) + sc<T, PERF>(ld(txy, c + 1) - ld(txy, c), n.dx, n._dx)) +
               sc<T, PERF>(ld(tyz, c + sz) - ld(tyz, c), n.dz, n._dz)) -
              sc<T, PERF>(ld(Pt, c) - ld(Pt, c - sy), n.dy, n._dy);
        if (CORR) R = R + ld(a.g1[9], c);
        return ld(a.g2[1], c) + R * ((ld(dR, c - sy) + ld(dR, c)) * n.half);
    } else {
        const int64_t c = gidx(g, clampi(i, 1, g.nx - 2), clampi(j, 1, g.ny - 2), k);
        if (!(k >= 1 && k <= g.nz - 1)) return ld(a.g2[2], c);
        T R = ((sc<T, PERF>(ld(tzz, c) - ld(tzz, c - sz), n.dz, n._dz) + sc<T, PERF>(ld(txz, c + 1) - ld(txz, c), n.dx, n._dx)) +
               sc<T, PERF>(ld(tyz, c + sy) - ld(tyz, c), n.dy, n._dy)) -
              sc<T, PERF>(ld(Pt, c) - ld(Pt, c - sz), n.dz, n._dz);
        if (CORR) R = R + ld(a.g1[10], c);
        return ld(a.g2[2], c) + R * ((ld(dR, c - sz) + ld(dR, c)) * n.half);
    }
}

__device__ __forceinline__ bool valid_face(const Geom& g, int comp, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0) return false;
    if (comp == 0) return i <= g.nx && j < g.ny && k < g.nz;
    if (comp == 1) return i < g.nx && j <= g.ny && k < g.nz;
    return i < g.nx && j < g.ny && k <= g.nz;
}

}  // namespace fused3

// 256 threads (32 x 8), one owned (i,j) column each; `zch` planes per CTA.
template <typename T, bool EL, bool PERF, bool CORR>
__global__ void __launch_bounds__(256, 1) k3_fused_BA(Geom g, Fused3Args<T> a, NumT<T> n, int zch, int store_divV) {
    using namespace fused3;
    using C = Cfg<T, EL, CORR>;
    constexpr int BW = C::BW, BOX = C::BOX, NF1 = C::NF1, NF2 = C::NF2, NF3 = C::NF3, NF4 = C::NF4;
    constexpr int EX = C::EX, EY = C::EY;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // [R1 | R2 | R3 | R4]
    uint64_t *bar1 = bar, *bar2 = bar + R1, *bar3 = bar + R1 + R2, *bar4 = bar + R1 + R2 + R3;
    T* st1 = reinterpret_cast<T*>(smem + C::kBar);  // [R1][NF1][BOX]
    T* st2 = st1 + R1 * NF1 * BOX;                    // [R2][NF2][BOX]
    T* st3 = st2 + R2 * NF2 * BOX;                    // [R3][NF3][BOX]
    T* st4 = st3 + R3 * NF3 * BOX;                    // [R4][NF4][BOX]
    T* sVbase = st4 + R4 * NF4 * BOX;                 // [3 comp][3 planes][EY][EX]
    auto sV = [&](int comp, int slot, int ey, int ex) -> T& { return sVbase[((comp * 3 + slot) * EY + ey) * EX + ex]; };

    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty, lane = tid & 31, warp = tid >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int x0s = x0 - C::XPAD, y0r = y0 - 1;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int k0 = blockIdx.z * zch;
    const int kB_end = min(k0 + zch, nz + 1);
    const int kA_end = min(k0 + zch, nz);
    const int i = x0 + tx, j = y0 + ty;
    const int s_first = max(k0 - 1, 0), s_last = min(k0 + zch, nz);
    // plane ranges of the four groups
    const int p1a = max(s_first - 1, 0), p1b = min(s_last + 1, nz);
    const int p2a = s_first, p2b = s_last;
    const int p3a = max(k0 - 1, 0), p3b = kA_end - 1;
    const int p4a = k0, p4b = kA_end - 1;
    auto slot1 = [&](int p) { return (p - p1a) % R1; };
    auto slot2 = [&](int p) { return (p - p2a) % R2; };
    auto slot3 = [&](int p) { return (p - p3a) % R3; };
    auto slot4 = [&](int p) { return (p - p4a) % R4; };
    auto box1 = [&](int p, int f) -> const T* { return st1 + (slot1(p) * NF1 + f) * BOX; };
    auto box2 = [&](int p, int f) -> const T* { return st2 + (slot2(p) * NF2 + f) * BOX; };
    auto box3 = [&](int p, int f) -> const T* { return st3 + (slot3(p) * NF3 + f) * BOX; };
    auto box4 = [&](int p, int f) -> const T* { return st4 + (slot4(p) * NF4 + f) * BOX; };
    auto issue1 = [&](int p) {
        if (p >= p1a && p <= p1b)
            issue_plane<T, BW, C::BH, BOX>(a.g1, NF1, st1 + slot1(p) * NF1 * BOX, bar1 + slot1(p), g, x0s, y0r, p, lane);
    };
    auto issue2 = [&](int p) {
        if (p >= p2a && p <= p2b)
            issue_plane<T, BW, C::BH, BOX>(a.g2, NF2, st2 + slot2(p) * NF2 * BOX, bar2 + slot2(p), g, x0s, y0r, p, lane);
    };
    auto issue3 = [&](int p) {
        if (p >= p3a && p <= p3b)
            issue_plane<T, BW, C::BH, BOX>(a.g3, NF3, st3 + slot3(p) * NF3 * BOX, bar3 + slot3(p), g, x0s, y0r, p, lane);
    };
    auto issue4 = [&](int p) {
        if (NF4 > 0 && p >= p4a && p <= p4b)
            issue_plane<T, BW, C::BH, BOX>(a.g4, NF4, st4 + slot4(p) * NF4 * BOX, bar4 + slot4(p), g, x0s, y0r, p, lane);
    };
    auto wait1 = [&](int p) { if (p >= p1a && p <= p1b) mbar_wait(bar1 + slot1(p), ((p - p1a) / R1) & 1, a.err); };
    auto wait2 = [&](int p) { if (p >= p2a && p <= p2b) mbar_wait(bar2 + slot2(p), ((p - p2a) / R2) & 1, a.err); };
    auto wait3 = [&](int p) { if (p >= p3a && p <= p3b) mbar_wait(bar3 + slot3(p), ((p - p3a) / R3) & 1, a.err); };
    auto wait4 = [&](int p) {
        if (NF4 > 0 && p >= p4a && p <= p4b) mbar_wait(bar4 + slot4(p), ((p - p4a) / R4) & 1, a.err);
    };
    auto li = [&](int ii, int jj) { return (jj - y0r) * BW + (ii - x0s); };

    if (tid == 0) {
        for (int q = 0; q < R1 + R2 + R3 + R4; ++q) mbar_init(bar + q, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == 0) {
        for (int p = p1a; p <= min(s_first + 1, p1b); ++p) issue1(p);
        issue2(s_first);
    }
    for (int p = p1a; p <= min(s_first, p1b); ++p) wait1(p);

    // ring assignment: 3 components x (TX + TY) faces; thread tid < 3*(TX+TY) takes one
    int rc = -1, rex = 0, rey = 0;
    if (tid < 3 * (TX + TY)) {
        rc = tid / (TX + TY);
        const int q = tid % (TX + TY);
        if (rc == 0) {  // Vx: x-high column, y-low row
            if (q < TY) { rex = TX + 1; rey = 1 + q; } else { rex = 1 + (q - TY); rey = 0; }
        } else if (rc == 1) {  // Vy: x-low column, y-high row
            if (q < TY) { rex = 0; rey = 1 + q; } else { rex = 1 + (q - TY); rey = TY + 1; }
        } else {  // Vz: x-low column, y-low row
            if (q < TY) { rex = 0; rey = 1 + q; } else { rex = 1 + (q - TY); rey = 0; }
        }
    }
    const int ri = x0 - 1 + rex, rj = y0 - 1 + rey;
    // A low ring (x0-1 or y0-1) is read only by the tile's own points i = x0 / j = y0; a
    // tile starting past the last cell (x0 >= nx or y0 >= ny) has none, and there the
    // clamped source of that ring face would lie outside the staged box.
    if ((rex == 0 && x0 >= nx) || (rey == 0 && y0 >= ny)) rc = -1;

    for (int s = s_first; s <= s_last; ++s) {
        if (warp == 0) {
            issue1(s + 2);
            issue2(s + 1);
            issue3(s);
            issue4(s);
        }
        wait1(s + 1);
        wait2(s);
        const int slotV = s % 3;
        // ---------------- B(s): V_n at plane s, owned faces + ring
        {
            const T *b_txx = box1(s, 0), *b_tyy = box1(s, 1), *b_tzz = box1(s, 2), *b_txy = box1(s, 3);
            const T *b_txz = box1(s, 4), *b_tyz = box1(s, 5), *b_Pt = box1(s, 6), *b_dR = box1(s, 7);
            const bool has_p = (s + 1 <= p1b), has_m = (s - 1 >= p1a);
            const T* b_txz_p = has_p ? box1(s + 1, 4) : b_txz;
            const T* b_tyz_p = has_p ? box1(s + 1, 5) : b_tyz;
            const T* b_tzz_m = has_m ? box1(s - 1, 2) : b_tzz;
            const T* b_Pt_m = has_m ? box1(s - 1, 6) : b_Pt;
            const T* b_dR_m = has_m ? box1(s - 1, 7) : b_dR;
            const T *b_Vx = box2(s, 0), *b_Vy = box2(s, 1), *b_Vz = box2(s, 2);
            const bool xy_global = (s == 0 || s >= nz - 1);  // Vx/Vy clamp to another plane
            auto vx_at = [&](int ii, int jj) -> T {
                if (xy_global) return face_global<T, PERF, CORR, 0>(a, n, g, ii, jj, s);
                const int l = li(ii, clampi(jj, 1, ny - 2));
                if (!(ii >= 1 && ii <= nx - 1)) return b_Vx[l];
                T R = ((sc<T, PERF>(b_txx[l] - b_txx[l - 1], n.dx, n._dx) + sc<T, PERF>(b_txy[l + BW] - b_txy[l], n.dy, n._dy)) +
                       sc<T, PERF>(b_txz_p[l] - b_txz[l], n.dz, n._dz)) -
                      sc<T, PERF>(b_Pt[l] - b_Pt[l - 1], n.dx, n._dx);
                if (CORR) R = R + box1(s, 8)[l];
                return b_Vx[l] + R * ((b_dR[l - 1] + b_dR[l]) * n.half);
            };
            auto vy_at = [&](int ii, int jj) -> T {
                if (xy_global) return face_global<T, PERF, CORR, 1>(a, n, g, ii, jj, s);
                const int l = li(clampi(ii, 1, nx - 2), jj);
                if (!(jj >= 1 && jj <= ny - 1)) return b_Vy[l];
                T R = ((sc<T, PERF>(b_tyy[l] - b_tyy[l - BW], n.dy, n._dy) + sc<T, PERF>(b_txy[l + 1] - b_txy[l], n.dx, n._dx)) +
                       sc<T, PERF>(b_tyz_p[l] - b_tyz[l], n.dz, n._dz)) -
                      sc<T, PERF>(b_Pt[l] - b_Pt[l - BW], n.dy, n._dy);
                if (CORR) R = R + box1(s, 9)[l];
                return b_Vy[l] + R * ((b_dR[l - BW] + b_dR[l]) * n.half);
            };
            auto vz_at = [&](int ii, int jj) -> T {
                const int l = li(clampi(ii, 1, nx - 2), clampi(jj, 1, ny - 2));
                if (!(s >= 1 && s <= nz - 1)) return b_Vz[l];
                T R = ((sc<T, PERF>(b_tzz[l] - b_tzz_m[l], n.dz, n._dz) + sc<T, PERF>(b_txz[l + 1] - b_txz[l], n.dx, n._dx)) +
                       sc<T, PERF>(b_tyz[l + BW] - b_tyz[l], n.dy, n._dy)) -
                      sc<T, PERF>(b_Pt[l] - b_Pt_m[l], n.dz, n._dz);
                if (CORR) R = R + box1(s, 10)[l];
                return b_Vz[l] + R * ((b_dR_m[l] + b_dR[l]) * n.half);
            };
            const bool own = (s >= k0 && s < kB_end);
            const int64_t c = gidx(g, i, j, s);
            T v = T(0);
            if (valid_face(g, 0, i, j, s)) {
                v = vx_at(i, j);
                if (own) a.Vx2[c] = v;
            }
            sV(0, slotV, ty + 1, tx + 1) = v;
            v = T(0);
            if (valid_face(g, 1, i, j, s)) {
                v = vy_at(i, j);
                if (own) a.Vy2[c] = v;
            }
            sV(1, slotV, ty + 1, tx + 1) = v;
            v = T(0);
            if (valid_face(g, 2, i, j, s)) {
                v = vz_at(i, j);
                if (own) a.Vz2[c] = v;
            }
            sV(2, slotV, ty + 1, tx + 1) = v;
            if (rc >= 0) {
                T w = T(0);
                if (valid_face(g, rc, ri, rj, s)) w = (rc == 0) ? vx_at(ri, rj) : (rc == 1) ? vy_at(ri, rj) : vz_at(ri, rj);
                sV(rc, slotV, rey, rex) = w;
            }
        }
        const int k = s - 1;
        const bool doA = (k >= k0 && k < kA_end);
        if (doA) {
            if (k == k0) wait3(k - 1);
            wait3(k);
            wait4(k);
        }
        __syncthreads();
        // ---------------- A(k = s-1): Pt, τ at plane k for the owned point
        if (doA && i < nx && j < ny) {
            const int sm = (s + 1) % 3, s0 = (s + 2) % 3, sp = slotV;  // V_n planes k-1, k, k+1
            const int ex = tx + 1, ey = ty + 1;
            const int64_t c = gidx(g, i, j, k);
            const int l = li(i, j);
            const T vx0 = sV(0, s0, ey, ex), vx1 = sV(0, s0, ey, ex + 1);
            const T vy0 = sV(1, s0, ey, ex), vy1 = sV(1, s0, ey + 1, ex);
            const T vz0 = sV(2, s0, ey, ex), vz1 = sV(2, sp, ey, ex);
            const T dvx = vx1 - vx0, dvy = vy1 - vy0, dvz = vz1 - vz0;
            const T* Gk = box3(k, 0);
            const T* Mk = box3(k, 1);
            const T Gc = Gk[l], Mc = Mk[l];
            {
                T dv;
                if (PERF) dv = (n._dx * dvx + n._dy * dvy) + n._dz * dvz;
                else dv = (dvx / n.dx + dvy / n.dy) + dvz / n.dz;
                if (!PERF && store_divV && a.divV) a.divV[c] = dv;
                if (CORR) dv = box4(k, 6)[l] + dv;
                a.Pt2[c] = box1(k, 6)[l] - n.r * Gc * dv;
            }
            constexpr bool SRC = EL || CORR;
            auto src = [&](int f) -> T { return SRC ? box4(k, f)[l] : T(0); };
            if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
                a.txx2[c] = tau_n<T, EL, PERF, CORR>(box1(k, 0)[l], src(0), Gc, Mc, n, n.dx, n._dx, dvx);
            if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
                a.tyy2[c] = tau_n<T, EL, PERF, CORR>(box1(k, 1)[l], src(1), Gc, Mc, n, n.dy, n._dy, dvy);
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
                a.tzz2[c] = tau_n<T, EL, PERF, CORR>(box1(k, 2)[l], src(2), Gc, Mc, n, n.dz, n._dz, dvz);
            if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2) {
                const T ag = (((Gk[l - 1 - BW] + Gk[l - BW]) + Gk[l - 1]) + Gc) * n.quarter;
                const T am = (((Mk[l - 1 - BW] + Mk[l - BW]) + Mk[l - 1]) + Mc) * n.quarter;
                const T d1 = vx0 - sV(0, s0, ey - 1, ex);  // Vx(i,j) - Vx(i,j-1)
                const T d2 = vy0 - sV(1, s0, ey, ex - 1);  // Vy(i,j) - Vy(i-1,j)
                a.txy2[c] = tau_s<T, EL, PERF, CORR>(box1(k, 3)[l], src(3), ag, am, n, n.dy, n._dy, d1, n.dx, n._dx, d2);
            }
            if (k >= 1) {
                const T* Gm = box3(k - 1, 0);
                const T* Mm = box3(k - 1, 1);
                if (i >= 1 && j >= 1 && j <= ny - 2) {
                    const T ag = (((Gm[l - 1] + Gm[l]) + Gk[l - 1]) + Gc) * n.quarter;
                    const T am = (((Mm[l - 1] + Mm[l]) + Mk[l - 1]) + Mc) * n.quarter;
                    const T d1 = vx0 - sV(0, sm, ey, ex);      // Vx(k) - Vx(k-1)
                    const T d2 = vz0 - sV(2, s0, ey, ex - 1);  // Vz(i) - Vz(i-1)
                    a.txz2[c] = tau_s<T, EL, PERF, CORR>(box1(k, 4)[l], src(4), ag, am, n, n.dz, n._dz, d1, n.dx, n._dx, d2);
                }
                if (i >= 1 && i <= nx - 2 && j >= 1) {
                    const T ag = (((Gm[l - BW] + Gm[l]) + Gk[l - BW]) + Gc) * n.quarter;
                    const T am = (((Mm[l - BW] + Mm[l]) + Mk[l - BW]) + Mc) * n.quarter;
                    const T d1 = vy0 - sV(1, sm, ey, ex);      // Vy(k) - Vy(k-1)
                    const T d2 = vz0 - sV(2, s0, ey - 1, ex);  // Vz(j) - Vz(j-1)
                    a.tyz2[c] = tau_s<T, EL, PERF, CORR>(box1(k, 5)[l], src(5), ag, am, n, n.dz, n._dz, d1, n.dy, n._dy, d2);
                }
            }
        }
        __syncthreads();
    }
}

// The same B-then-A single pass without staging: every iteration-n input is read-only in
// the launch (the outputs are the other ping-pong buffers), so B and A load them straight
// from global memory through the read-only data path and let L1/L2 serve the halos. Only
// V_n of the last three planes stays in shared memory (the ring exchange between B and A).
template <typename T, bool EL, bool PERF, bool CORR>
__global__ void __launch_bounds__(256) k3_fused_direct(Geom g, Fused3Args<T> a, NumT<T> n, int zch, int store_divV) {
    using namespace fused3;
    constexpr int EX = TX + 2, EY = TY + 2;
    __shared__ T sVbase[3 * 3 * EY * EX];  // [3 comp][3 planes][EY][EX]
    auto sV = [&](int comp, int slot, int ey, int ex) -> T& { return sVbase[((comp * 3 + slot) * EY + ey) * EX + ex]; };
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int k0 = blockIdx.z * zch;
    const int kB_end = min(k0 + zch, nz + 1);
    const int kA_end = min(k0 + zch, nz);
    const int i = x0 + tx, j = y0 + ty;
    const int s_first = max(k0 - 1, 0), s_last = min(k0 + zch, nz);
    const idx_t sx = 1, sy = g.px, sz = (idx_t)g.pxy;

    // ring assignment as in k3_fused_BA: 3 components x (TX + TY) faces
    int rc = -1, rex = 0, rey = 0;
    if (tid < 3 * (TX + TY)) {
        rc = tid / (TX + TY);
        const int q = tid % (TX + TY);
        if (rc == 0) {
            if (q < TY) { rex = TX + 1; rey = 1 + q; } else { rex = 1 + (q - TY); rey = 0; }
        } else if (rc == 1) {
            if (q < TY) { rex = 0; rey = 1 + q; } else { rex = 1 + (q - TY); rey = TY + 1; }
        } else {
            if (q < TY) { rex = 0; rey = 1 + q; } else { rex = 1 + (q - TY); rey = 0; }
        }
    }
    const int ri = x0 - 1 + rex, rj = y0 - 1 + rey;
    if ((rex == 0 && x0 >= nx) || (rey == 0 && y0 >= ny)) rc = -1;  // read by no point of the tile

    for (int s = s_first; s <= s_last; ++s) {
        const int slotV = s % 3;
        // ---------------- B(s): V_n at plane s, owned faces + ring
        {
            const bool own = (s >= k0 && s < kB_end);
            const int64_t c = gidx(g, i, j, s);
            T v = T(0);
            if (valid_face(g, 0, i, j, s)) {
                v = face_global<T, PERF, CORR, 0>(a, n, g, i, j, s);
                if (own) a.Vx2[c] = v;
            }
            sV(0, slotV, ty + 1, tx + 1) = v;
            v = T(0);
            if (valid_face(g, 1, i, j, s)) {
                v = face_global<T, PERF, CORR, 1>(a, n, g, i, j, s);
                if (own) a.Vy2[c] = v;
            }
            sV(1, slotV, ty + 1, tx + 1) = v;
            v = T(0);
            if (valid_face(g, 2, i, j, s)) {
                v = face_global<T, PERF, CORR, 2>(a, n, g, i, j, s);
                if (own) a.Vz2[c] = v;
            }
            sV(2, slotV, ty + 1, tx + 1) = v;
            if (rc >= 0) {
                T w = T(0);
                if (valid_face(g, rc, ri, rj, s))
                    w = (rc == 0)   ? face_global<T, PERF, CORR, 0>(a, n, g, ri, rj, s)
                        : (rc == 1) ? face_global<T, PERF, CORR, 1>(a, n, g, ri, rj, s)
                                    : face_global<T, PERF, CORR, 2>(a, n, g, ri, rj, s);
                sV(rc, slotV, rey, rex) = w;
            }
        }
        __syncthreads();
        // ---------------- A(k = s-1): Pt, τ at plane k for the owned point
        const int k = s - 1;
        if (k >= k0 && k < kA_end && i < nx && j < ny) {
            const int sm = (s + 1) % 3, s0 = (s + 2) % 3, sp = slotV;  // V_n planes k-1, k, k+1
            const int ex = tx + 1, ey = ty + 1;
            const idx_t c = gidx32(g, i, j, k);
            const T vx0 = sV(0, s0, ey, ex), vx1 = sV(0, s0, ey, ex + 1);
            const T vy0 = sV(1, s0, ey, ex), vy1 = sV(1, s0, ey + 1, ex);
            const T vz0 = sV(2, s0, ey, ex), vz1 = sV(2, sp, ey, ex);
            const T dvx = vx1 - vx0, dvy = vy1 - vy0, dvz = vz1 - vz0;
            const T *Gd = a.g3[0], *Mu = a.g3[1];
            const T Gc = __ldg(Gd + c), Mc = __ldg(Mu + c);
            {
                T dv;
                if (PERF) dv = (n._dx * dvx + n._dy * dvy) + n._dz * dvz;
                else dv = (dvx / n.dx + dvy / n.dy) + dvz / n.dz;
                if (!PERF && store_divV && a.divV) a.divV[c] = dv;
                if (CORR) dv = __ldg(a.g4[6] + c) + dv;
                a.Pt2[c] = __ldg(a.g1[6] + c) - n.r * Gc * dv;
            }
            constexpr bool SRC = EL || CORR;
            auto src = [&](int f) -> T { return SRC ? __ldg(a.g4[f] + c) : T(0); };
            auto tau = [&](int f) -> T { return __ldg(a.g1[f] + c); };
            if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2)
                a.txx2[c] = tau_n<T, EL, PERF, CORR>(tau(0), src(0), Gc, Mc, n, n.dx, n._dx, dvx);
            if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2)
                a.tyy2[c] = tau_n<T, EL, PERF, CORR>(tau(1), src(1), Gc, Mc, n, n.dy, n._dy, dvy);
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)
                a.tzz2[c] = tau_n<T, EL, PERF, CORR>(tau(2), src(2), Gc, Mc, n, n.dz, n._dz, dvz);
            if (i >= 1 && j >= 1 && k >= 1 && k <= nz - 2) {
                const T ag = (((__ldg(Gd + c - sx - sy) + __ldg(Gd + c - sy)) + __ldg(Gd + c - sx)) + Gc) * n.quarter;
                const T am = (((__ldg(Mu + c - sx - sy) + __ldg(Mu + c - sy)) + __ldg(Mu + c - sx)) + Mc) * n.quarter;
                const T d1 = vx0 - sV(0, s0, ey - 1, ex);  // Vx(i,j) - Vx(i,j-1)
                const T d2 = vy0 - sV(1, s0, ey, ex - 1);  // Vy(i,j) - Vy(i-1,j)
                a.txy2[c] = tau_s<T, EL, PERF, CORR>(tau(3), src(3), ag, am, n, n.dy, n._dy, d1, n.dx, n._dx, d2);
            }
            if (k >= 1) {
                if (i >= 1 && j >= 1 && j <= ny - 2) {
                    const T ag = (((__ldg(Gd + c - sx - sz) + __ldg(Gd + c - sz)) + __ldg(Gd + c - sx)) + Gc) * n.quarter;
                    const T am = (((__ldg(Mu + c - sx - sz) + __ldg(Mu + c - sz)) + __ldg(Mu + c - sx)) + Mc) * n.quarter;
                    const T d1 = vx0 - sV(0, sm, ey, ex);      // Vx(k) - Vx(k-1)
                    const T d2 = vz0 - sV(2, s0, ey, ex - 1);  // Vz(i) - Vz(i-1)
                    a.txz2[c] = tau_s<T, EL, PERF, CORR>(tau(4), src(4), ag, am, n, n.dz, n._dz, d1, n.dx, n._dx, d2);
                }
                if (i >= 1 && i <= nx - 2 && j >= 1) {
                    const T ag = (((__ldg(Gd + c - sy - sz) + __ldg(Gd + c - sz)) + __ldg(Gd + c - sy)) + Gc) * n.quarter;
                    const T am = (((__ldg(Mu + c - sy - sz) + __ldg(Mu + c - sz)) + __ldg(Mu + c - sy)) + Mc) * n.quarter;
                    const T d1 = vy0 - sV(1, sm, ey, ex);      // Vy(k) - Vy(k-1)
                    const T d2 = vz0 - sV(2, s0, ey - 1, ex);  // Vz(j) - Vz(j-1)
                    a.tyz2[c] = tau_s<T, EL, PERF, CORR>(tau(5), src(5), ag, am, n, n.dz, n._dz, d1, n.dy, n._dy, d2);
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace pts
