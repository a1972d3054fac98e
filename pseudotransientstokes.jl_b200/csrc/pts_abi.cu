// pts_abi.cu -- the C ABI of libptstokes.so: contexts, fields, set-up, roles and the PT
// loop driver. Host code only (plus launches of the kernels in pts_kernels64.cu).
//
// The PT loop runs on the context's stream. Between two convergence checks the nout
// iterations (two kernels each) and the check are one CUDA graph, so the host wakes
// once per check, reads a small pinned result block and decides whether to go on --
// the `while err > ε && iter <= iterMax` loop of the scripts (Stokes3D_ve_perf.jl:198-223).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pts_internal.h"

using namespace pts;

namespace {
std::string g_create_err;
}

namespace pts {
void set_global_error(const char* msg) { g_create_err = msg; }
}  // namespace pts

struct pts_ctx {
    pts_desc d{};
    int v = 0;
    bool d3 = false, elastic = false, perf = false;
    Geom g{};
    Num n{};
    int device = 0;
    cudaStream_t stream = nullptr;
    Fields64 f{};    // current fields
    Fields64 alt{};  // second buffers of the ten iterated fields (single-pass 3D path)
    bool fused = false;
    bool zs = false;         // compute_Pt_τ! by the z-marching TMA-staged kernel
    bool ys = false;         // 2D: compute_Pt_τ! by the y-marching TMA-staged kernel
    bool mixed = false;      // FP32 inner sweeps + FP64 defect correction
    Mixed32 m{};
    Mixed32 m2{};            // second set of the ten FP32 corrections (one-pass sweeps)
    bool fused32 = false;    // one-pass FP32 sweeps (compute_V! + bc, then compute_Pt_τ!)
    int ftile = 0;           // its tile configuration
    std::vector<float*> owned32;
    int parity = 0;  // number of buffer swaps mod 2
    std::vector<double*> owned;  // every device allocation
    double* partials = nullptr;
    int partials_cap = 0;
    CheckResult* d_result = nullptr;
    CheckResult* h_result = nullptr;  // pinned
    cudaGraphExec_t chunk[2] = {nullptr, nullptr};  // nout iterations + check, per starting parity
    int* d_kerr = nullptr;  // set by a kernel whose bounded wait timed out
    bool timing = false;             // a CUDA event after each kernel of a block (pts_set_kernel_timing)
    std::vector<cudaEvent_t> tev;    // those events, in launch order
    int tev_n = 0;                   // events the last enqueued block records
    pts_inclusion* d_incl = nullptr;  // inclusion list of pts_init_inclusions
    int incl_cap = 0;
    std::string err;
};

namespace {

int fail(pts_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_err = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(c, PTS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct FInfo {
    double** ptr;
    int64_t e[3];  // the reference's extents
    int s[3];      // unified start of the reference's element [1,1,1]
};

// Momentum sources exist for the 3D explicit-index variants on the FP64 two-kernel path.
bool has_sources(const pts_ctx* c) {
    return (c->v == PTS_3D_V || c->v == PTS_3D_VE_PERF) && !c->mixed && !c->fused;
}

// Field table: reference extents (Stokes3D_ve_perf.jl:141-162, Stokes2D_ve_perf.jl:105-118)
// and where each field's first element sits in the unified staggered layout.
bool field_info(pts_ctx* c, int id, FInfo* o) {
    const int nx = c->g.nx, ny = c->g.ny, nz = c->d3 ? c->g.nz : 1;
    Fields64& f = c->f;
    auto set = [&](double** p, int64_t a, int64_t b, int64_t cc, int s0, int s1, int s2) {
        o->ptr = p;
        o->e[0] = a; o->e[1] = b; o->e[2] = cc;
        o->s[0] = s0; o->s[1] = s1; o->s[2] = s2;
    };
    const bool d3 = c->d3, el = c->elastic;
    switch (id) {
        case PTS_F_PT: set(&f.Pt, nx, ny, nz, 0, 0, 0); break;
        case PTS_F_MUS: set(&f.Mus, nx, ny, nz, 0, 0, 0); break;
        case PTS_F_MUS_TAU: set(&f.Must, nx, ny, nz, 0, 0, 0); break;
        case PTS_F_GDTAU: set(&f.Gdt, nx, ny, nz, 0, 0, 0); break;
        case PTS_F_DTAU_RHO: set(&f.dtRho, nx, ny, nz, 0, 0, 0); break;
        case PTS_F_DIVV: set(&f.divV, nx, ny, nz, 0, 0, 0); break;
        case PTS_F_VX: set(&f.Vx, nx + 1, ny, nz, 0, 0, 0); break;
        case PTS_F_VY: set(&f.Vy, nx, ny + 1, nz, 0, 0, 0); break;
        case PTS_F_VZ: if (!d3) return false; set(&f.Vz, nx, ny, nz + 1, 0, 0, 0); break;
        case PTS_F_TXX: case PTS_F_TXX_O:
            if (id == PTS_F_TXX_O && !el) return false;
            if (d3) set(id == PTS_F_TXX ? &f.txx : &f.txx_o, nx, ny - 2, nz - 2, 0, 1, 1);
            else set(id == PTS_F_TXX ? &f.txx : &f.txx_o, nx, ny, 1, 0, 0, 0);
            break;
        case PTS_F_TYY: case PTS_F_TYY_O:
            if (id == PTS_F_TYY_O && !el) return false;
            if (d3) set(id == PTS_F_TYY ? &f.tyy : &f.tyy_o, nx - 2, ny, nz - 2, 1, 0, 1);
            else set(id == PTS_F_TYY ? &f.tyy : &f.tyy_o, nx, ny, 1, 0, 0, 0);
            break;
        case PTS_F_TZZ: case PTS_F_TZZ_O:
            if (!d3 || (id == PTS_F_TZZ_O && !el)) return false;
            set(id == PTS_F_TZZ ? &f.tzz : &f.tzz_o, nx - 2, ny - 2, nz, 1, 1, 0);
            break;
        case PTS_F_TXY: case PTS_F_TXY_O:
            if (id == PTS_F_TXY_O && !el) return false;
            if (d3) set(id == PTS_F_TXY ? &f.txy : &f.txy_o, nx - 1, ny - 1, nz - 2, 1, 1, 1);
            else set(id == PTS_F_TXY ? &f.txy : &f.txy_o, nx - 1, ny - 1, 1, 1, 1, 0);
            break;
        case PTS_F_TXZ: case PTS_F_TXZ_O:
            if (!d3 || (id == PTS_F_TXZ_O && !el)) return false;
            set(id == PTS_F_TXZ ? &f.txz : &f.txz_o, nx - 1, ny - 2, nz - 1, 1, 1, 1);
            break;
        case PTS_F_TYZ: case PTS_F_TYZ_O:
            if (!d3 || (id == PTS_F_TYZ_O && !el)) return false;
            set(id == PTS_F_TYZ ? &f.tyz : &f.tyz_o, nx - 2, ny - 1, nz - 1, 1, 1, 1);
            break;
        case PTS_F_RX: case PTS_F_DVX:
            set(id == PTS_F_RX ? &f.Rx : &f.dVx, nx - 1, ny - 2, d3 ? nz - 2 : 1, 1, 1, d3 ? 1 : 0);
            break;
        case PTS_F_RY: case PTS_F_DVY:
            set(id == PTS_F_RY ? &f.Ry : &f.dVy, nx - 2, ny - 1, d3 ? nz - 2 : 1, 1, 1, d3 ? 1 : 0);
            break;
        case PTS_F_RZ: case PTS_F_DVZ:
            if (!d3) return false;
            set(id == PTS_F_RZ ? &f.Rz : &f.dVz, nx - 2, ny - 2, nz - 1, 1, 1, 1);
            break;
        case PTS_F_FX: if (!has_sources(c)) return false; set(&f.Fx, nx - 1, ny - 2, nz - 2, 1, 1, 1); break;
        case PTS_F_FY: if (!has_sources(c)) return false; set(&f.Fy, nx - 2, ny - 1, nz - 2, 1, 1, 1); break;
        case PTS_F_FZ: if (!has_sources(c)) return false; set(&f.Fz, nx - 2, ny - 2, nz - 1, 1, 1, 1); break;
        case PTS_F_GRAD:
            if (c->v != PTS_3D_V && c->v != PTS_3D_VE_PERF) return false;
            set(&f.grad, nx, ny, nz, 0, 0, 0);
            break;
        // pseudo-time steps of the damped variants (Stokes2D_ve0.jl:123-124,106)
        // pseudo-time steps of the damped variants: the extents of Rx, Ry, Rz and of the cells
        // (Stokes2D_ve0.jl:106,123-124; Stokes3D0_multixpu.jl:123,138-140)
        case PTS_F_DTAU_VX:
            if (!variant_damped(c->v)) return false;
            set(&f.dtVx, nx - 1, ny - 2, d3 ? nz - 2 : 1, 1, 1, d3 ? 1 : 0);
            break;
        case PTS_F_DTAU_VY:
            if (!variant_damped(c->v)) return false;
            set(&f.dtVy, nx - 2, ny - 1, d3 ? nz - 2 : 1, 1, 1, d3 ? 1 : 0);
            break;
        case PTS_F_DTAU_VZ:
            if (!variant_damped(c->v) || !d3) return false;
            set(&f.dtVz, nx - 2, ny - 2, nz - 1, 1, 1, 1);
            break;
        case PTS_F_DTAU_PT: if (!variant_damped(c->v)) return false; set(&f.dtPt, nx, ny, nz, 0, 0, 0); break;
        default: return false;
    }
    return true;
}

int alloc_field(pts_ctx* c, double** p) {
    if (*p) return PTS_OK;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, (size_t)c->g.n * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, PTS_E_NOMEM, std::string("cudaMalloc of a field failed: ") + cudaGetErrorString(e));
    }
    CK(cudaMemsetAsync(q, 0, (size_t)c->g.n * sizeof(double), c->stream));
    *p = (double*)q;
    c->owned.push_back(*p);
    return PTS_OK;
}

void drop_graph(pts_ctx* c) {
    for (auto& g : c->chunk)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// The first source set allocates all three (zero) and switches the V update and the check
// to their source-adding forms (the captured graphs are dropped).
int ensure_sources(pts_ctx* c, int id) {
    if (id != PTS_F_FX && id != PTS_F_FY && id != PTS_F_FZ) return PTS_OK;
    if (!has_sources(c)) return fail(c, PTS_E_INVAL, "momentum sources need 3D_V or 3D_VE_PERF on the FP64 two-kernel path");
    if (c->f.Fx) return PTS_OK;
    int rc;
    if ((rc = alloc_field(c, &c->f.Fx)) != PTS_OK || (rc = alloc_field(c, &c->f.Fy)) != PTS_OK ||
        (rc = alloc_field(c, &c->f.Fz)) != PTS_OK)
        return rc;
    drop_graph(c);
    return PTS_OK;
}

// The ten fields one PT iteration rewrites (Pt, τ, V): the single-pass kernel reads them
// from one buffer and writes the next iterate into the other.
double** iterated(Fields64& f, int q) {
    double** p[] = {&f.Pt, &f.Vx, &f.Vy, &f.Vz, &f.txx, &f.tyy, &f.tzz, &f.txy, &f.txz, &f.tyz};
    return p[q];
}

void swap_buffers(pts_ctx* c) {
    for (int q = 0; q < 10; ++q) std::swap(*iterated(c->f, q), *iterated(c->alt, q));
    c->parity ^= 1;
}

// Numerics of the damped scheme and what derives from them (Stokes2D_ve0.jl:95-105,
// Stokes3D0_multixpu.jl:105-120): dampX = 1.0-Vdmp/nx (Y, Z alike), min_dxy2 =
// min(dx,dy[,dz])^2, max_nxy = max(nx,ny[,nz]).
void set_damping(pts_ctx* c, double Vdmp, double beta_n, double Vsc, double Ptsc) {
    Num& n = c->n;
    n.Vdmp = Vdmp;
    n.beta_n = beta_n;
    n.Vsc = Vsc;
    n.Ptsc = Ptsc;
    n.dampX = 1.0 - Vdmp / (double)c->g.nx;
    n.dampY = 1.0 - Vdmp / (double)c->g.ny;
    n.dampZ = 1.0 - Vdmp / (double)c->g.nz;
    const double m = c->d3 ? std::min(std::min(n.dx, n.dy), n.dz) : std::min(n.dx, n.dy);
    n.min_dxy2 = m * m;
    n.max_nxy = (double)(c->d3 ? std::max(std::max(c->g.nx, c->g.ny), c->g.nz) : std::max(c->g.nx, c->g.ny));
}

int enter(pts_ctx* c) {
    if (!c) return PTS_E_INVAL;
    CK(cudaSetDevice(c->device));
    return PTS_OK;
}

// Wait for the stream, then report a kernel whose bounded wait gave up (its results are
// not to be trusted; the flag is cleared so the context stays usable).
int synced(pts_ctx* c) {
    CK(cudaStreamSynchronize(c->stream));
    int flag = 0;
    CK(cudaMemcpy(&flag, c->d_kerr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        CK(cudaMemset(c->d_kerr, 0, sizeof(int)));
        return fail(c, PTS_E_CUDA, "a bounded shared-memory staging wait in a z-marching kernel timed out");
    }
    return PTS_OK;
}

int copy3d(pts_ctx* c, int id, const double* src_dense, double* dst_dense, int64_t n, cudaMemcpyKind kind) {
    FInfo fi;
    if (!field_info(c, id, &fi)) return fail(c, PTS_E_INVAL, "field not present for this variant: " + std::to_string(id));
    if (*fi.ptr == nullptr) return fail(c, PTS_E_STATE, "field not allocated: " + std::to_string(id));
    const int64_t want = fi.e[0] * fi.e[1] * fi.e[2];
    if (n != want)
        return fail(c, PTS_E_INVAL, "field " + std::to_string(id) + " has " + std::to_string(want) + " elements, got " +
                                        std::to_string(n));
    cudaMemcpy3DParms p;
    memset(&p, 0, sizeof(p));
    cudaPitchedPtr dense = make_cudaPitchedPtr(src_dense ? (void*)src_dense : (void*)dst_dense,
                                               (size_t)fi.e[0] * sizeof(double), (size_t)fi.e[0], (size_t)fi.e[1]);
    cudaPitchedPtr pad = make_cudaPitchedPtr(*fi.ptr, (size_t)c->g.px * sizeof(double), (size_t)c->g.px,
                                             (size_t)c->g.py);
    cudaPos at = make_cudaPos((size_t)fi.s[0] * sizeof(double), (size_t)fi.s[1], (size_t)fi.s[2]);
    if (src_dense) {
        p.srcPtr = dense;
        p.dstPtr = pad;
        p.dstPos = at;
    } else {
        p.srcPtr = pad;
        p.srcPos = at;
        p.dstPtr = dense;
    }
    p.extent = make_cudaExtent((size_t)fi.e[0] * sizeof(double), (size_t)fi.e[1], (size_t)fi.e[2]);
    p.kind = kind;
    CK(cudaMemcpy3DAsync(&p, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PTS_OK;
}

// compute_Pt_τ! (both roles) on the context's fields: the z-marching TMA-staged kernel
// unless the context asked for the one-thread-per-cell form (same bits either way).
int Pt_tau(pts_ctx* c, bool store_divV) {
    if (c->ys)
        CK(launch_Pt_tau_ys(c->v, c->d.stencil_tile, c->g, c->f, c->n, c->d.stencil_kz, store_divV && !c->perf,
                            c->d_kerr, c->stream));
    else if (c->zs)
        CK(launch_Pt_tau_zs(c->v, c->d.stencil_tile, c->g, c->f, c->n, c->d.stencil_kz, store_divV && !c->perf,
                            c->d_kerr, c->stream));
    else
        CK(launch_Pt_tau(c->v, c->g, c->f, c->n, ROLE_P | ROLE_TAU, store_divV && !c->perf, c->stream));
    return PTS_OK;
}

// compute_V! + bc: the z-marching TMA-staged kernel on the plain path (no momentum sources,
// no adjoint folding), else the one-thread-per-face kernel (same bits either way).
int V_bc(pts_ctx* c, bool update) {
    if (c->zs && update && !c->f.Fx && !c->n.adjoint)
        CK(launch_V_bc_zs(c->v, c->d.stencil_vtile, c->g, c->f, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
    else
        CK(launch_V_bc(c->v, c->g, c->f, c->n, update, c->stream));
    return PTS_OK;
}

// With kernel timing on, the next event of the block being enqueued: recorded on the
// context's stream, or, during graph capture, as an event-record node of the graph.
int mark(pts_ctx* c) {
    if (!c->timing) return PTS_OK;
    if (c->tev_n >= (int)c->tev.size()) {
        cudaEvent_t e = nullptr;
        CK(cudaEventCreate(&e));
        c->tev.push_back(e);
    }
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(c->stream, &st));
    if (st == cudaStreamCaptureStatusActive)
        CK(cudaEventRecordWithFlags(c->tev[c->tev_n], c->stream, cudaEventRecordExternal));
    else
        CK(cudaEventRecord(c->tev[c->tev_n], c->stream));
    ++c->tev_n;
    return PTS_OK;
}

// Tile configurations of the TMA-staged compute_Pt_τ! of a context: 3D FP64, 3D FP32
// sweeps, 2D.
int tile_count(bool d3, bool mixed) {
    return mixed ? zstage32_num_configs() : (d3 ? zstage_num_configs() : ystage_num_configs());
}

// The ten FP32 corrections of the current and the second buffer set trade places.
void swap_m(pts_ctx* c) {
    float** a[10] = {&c->m.dPt, &c->m.dVx, &c->m.dVy, &c->m.dVz, &c->m.dtxx,
                     &c->m.dtyy, &c->m.dtzz, &c->m.dtxy, &c->m.dtxz, &c->m.dtyz};
    float** b[10] = {&c->m2.dPt, &c->m2.dVx, &c->m2.dVy, &c->m2.dVz, &c->m2.dtxx,
                     &c->m2.dtyy, &c->m2.dtzz, &c->m2.dtxy, &c->m2.dtxz, &c->m2.dtyz};
    for (int q = 0; q < 10; ++q) std::swap(*a[q], *b[q]);
}

// The second buffer set of the one-pass FP32 sweeps (allocated once, zeroed).
int alloc_m2(pts_ctx* c) {
    if (c->m2.dPt) return PTS_OK;
    float** p[10] = {&c->m2.dPt, &c->m2.dVx, &c->m2.dVy, &c->m2.dVz, &c->m2.dtxx,
                     &c->m2.dtyy, &c->m2.dtzz, &c->m2.dtxy, &c->m2.dtxz, &c->m2.dtyz};
    for (float** q : p) {
        void* d = nullptr;
        if (cudaMalloc(&d, (size_t)c->g.n * sizeof(float)) != cudaSuccess ||
            cudaMemsetAsync(d, 0, (size_t)c->g.n * sizeof(float), c->stream) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, PTS_E_NOMEM, "allocation of the second FP32 correction set failed");
        }
        *q = (float*)d;
        c->owned32.push_back(*q);
    }
    // the stress points the sweeps never update hold -w in both sets (k3_srcw); fill the new
    // set from the current one
    float* src[6] = {c->m.dtxx, c->m.dtyy, c->m.dtzz, c->m.dtxy, c->m.dtxz, c->m.dtyz};
    float* dst[6] = {c->m2.dtxx, c->m2.dtyy, c->m2.dtzz, c->m2.dtxy, c->m2.dtxz, c->m2.dtyz};
    for (int q = 0; q < 6; ++q) {
        CK(cudaMemcpyAsync(dst[q], src[q], (size_t)c->g.n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
        c->m.u2[q] = dst[q];
    }
    return PTS_OK;
}

// One PT iteration with the two-kernel path: compute_Pt_τ! then compute_V! + bc.
int iteration(pts_ctx* c, bool store_divV) {
    int rc = Pt_tau(c, store_divV);
    if (rc || (rc = mark(c))) return rc;
    rc = V_bc(c, true);
    if (rc || (rc = mark(c))) return rc;
    return PTS_OK;
}

// m PT iterations. Single-pass 3D path: compute_Pt_τ! of iteration 1, then m-1 launches
// of the fused kernel (V of iteration q, then Pt/τ of q+1, into the other buffers), then
// compute_V! + bc of iteration m. ∇V of the last iteration is kept for the check of the
// role variants.
int enqueue_block(pts_ctx* c, int64_t m, bool store_last) {
    if (m <= 0) return PTS_OK;
    c->tev_n = 0;
    if (int rc = mark(c)) return rc;
    if (c->mixed && c->fused32) {
        // compute_Pt_τ! of sweep 1 and compute_V! + bc of sweep m in place; in between, one
        // pass per pair (V of sweep q, Pt/τ of q+1) from one buffer set into the other. An
        // even number of passes leaves the current set where it was (the graph of a block
        // is the same for every block); an odd count gives one pair to the two kernels.
        CK(launch_corr_A32_zs(c->v, c->d.stencil_tile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
        int64_t passes = m - 1;
        if (passes & 1) {
            CK(launch_corr_B32_zs(c->v, c->d.stencil_vtile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
            CK(launch_corr_A32_zs(c->v, c->d.stencil_tile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
            --passes;
        }
        for (int64_t q = 0; q < passes; ++q) {
            CK(launch_corr_BA32_zs(c->v, c->ftile, c->g, c->m, c->m2, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
            swap_m(c);
        }
        CK(launch_corr_B32_zs(c->v, c->d.stencil_vtile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
        CK(launch_fold(c->g, c->f, c->m, c->stream));
        return PTS_OK;
    }
    if (c->mixed) {
        // m FP32 sweeps on the correction, then the FP64 fold X += δ (δ = 0 again). The
        // sources must already describe the current X (mixed_prepare or a previous check).
        for (int64_t q = 0; q < m; ++q) {
            if (c->zs)
                CK(launch_corr_A32_zs(c->v, c->d.stencil_tile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
            else
                CK(launch_corr_A32(c->v, c->g, c->m, c->n, c->stream));
            if (int rc = mark(c)) return rc;
            if (c->zs)
                CK(launch_corr_B32_zs(c->v, c->d.stencil_vtile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr,
                                      c->stream));
            else
                CK(launch_corr_B32(c->v, c->g, c->m, c->n, c->stream));
            if (int rc = mark(c)) return rc;
        }
        CK(launch_fold(c->g, c->f, c->m, c->stream));
        if (int rc = mark(c)) return rc;
        return PTS_OK;
    }
    if (!c->fused) {
        for (int64_t q = 0; q < m; ++q) {
            int rc = iteration(c, store_last && q == m - 1);
            if (rc) return rc;
        }
        return PTS_OK;
    }
    CK(launch_Pt_tau(c->v, c->g, c->f, c->n, ROLE_P | ROLE_TAU, store_last && m == 1 && !c->perf, c->stream));
    for (int64_t q = 1; q < m; ++q) {
        CK(launch_fused3(c->v, c->g, c->f, c->alt, c->n, store_last && q == m - 1 && !c->perf, c->d_kerr, c->stream,
                         c->d.single_pass == 2));
        swap_buffers(c);
    }
    CK(launch_V_bc(c->v, c->g, c->f, c->n, true, c->stream));
    return PTS_OK;
}

// The convergence check of the current FP64 iterate. In mixed precision the same pass
// also writes the FP32 residual sources for the next sweeps (the check's R and ∇V are
// two of them).
int enqueue_check(pts_ctx* c) {
    if (c->mixed)
        CK(launch_sources(c->v, c->g, c->f, c->m, c->n, c->partials, c->partials_cap, c->d_result, c->stream));
    else
        CK(launch_check(c->v, c->g, c->f, c->n, c->partials, c->partials_cap, c->d_result, c->stream));
    CK(cudaMemcpyAsync(c->h_result, c->d_result, sizeof(CheckResult), cudaMemcpyDeviceToHost, c->stream));
    return mark(c);
}

// Mixed precision: FP32 copies of the coefficients and the sources of the current iterate
// (called when the FP64 state may have changed outside the sweeps).
int mixed_prepare(pts_ctx* c) {
    CK(launch_coef32(c->g, c->f, c->m, c->stream));
    CK(launch_sources(c->v, c->g, c->f, c->m, c->n, c->partials, c->partials_cap, c->d_result, c->stream));
    return PTS_OK;
}

// Swaps one block of m iterations performs on the host-side buffer pointers.
bool block_swaps_odd(const pts_ctx* c, int64_t m) { return c->fused && m > 1 && ((m - 1) & 1); }

// Capture `nout` iterations + the check as a graph for the current buffer parity. The
// capture itself runs nothing, so the pointer swaps it made are undone afterwards.
int build_chunk(pts_ctx* c) {
    const int p = c->parity;
    if (c->chunk[p]) return PTS_OK;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_block(c, c->d.nout, true);
    if (rc == PTS_OK) rc = enqueue_check(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (c->parity != p) swap_buffers(c);
    if (rc != PTS_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(c, PTS_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->chunk[p], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        c->chunk[p] = nullptr;
        return fail(c, PTS_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    return PTS_OK;
}

int launch_chunk(pts_ctx* c) {
    int rc = build_chunk(c);
    if (rc) return rc;
    CK(cudaGraphLaunch(c->chunk[c->parity], c->stream));
    if (block_swaps_odd(c, c->d.nout)) swap_buffers(c);
    return PTS_OK;
}

void to_check(const CheckResult& r, pts_check* o) {
    o->err = r.err;
    o->norm_Rx = r.nRx;
    o->norm_Ry = r.nRy;
    o->norm_Rz = r.nRz;
    o->norm_divV = r.ndiv;
    o->Vmin = r.vmin;
    o->Vmax = r.vmax;
    o->Pmin = r.pmin;
    o->Pmax = r.pmax;
}

}  // namespace

extern "C" {

int pts_abi_version(void) { return PTS_ABI_VERSION; }

int pts_set_stencil(pts_ctx* c, int32_t stencil, int32_t tile, int32_t kz, int32_t vtile) {
    int rc = enter(c);
    if (rc) return rc;
    if (stencil != 0 && stencil != 1) return fail(c, PTS_E_INVAL, "stencil must be 0 or 1");
    if (tile < 0 || tile >= tile_count(c->d3, c->mixed))
        return fail(c, PTS_E_INVAL, "stencil_tile out of range (pts_stencil_tiles, pts_stencil_tiles_2d)");
    if (vtile < 0 || vtile >= (c->mixed ? zvbc32_num_configs() : zvbc_num_configs()))
        return fail(c, PTS_E_INVAL, "stencil_vtile out of range (pts_stencil_vtiles)");
    if (kz < 0) return fail(c, PTS_E_INVAL, "stencil_kz must be >= 0");
    c->d.stencil = stencil;
    c->d.stencil_tile = tile;
    c->d.stencil_kz = kz;
    c->d.stencil_vtile = vtile;
    c->zs = (c->v == VE3D || c->v == VE3D_PERF || c->v == V3D) && !c->fused && stencil == 0;
    c->ys = (c->v == V2D || c->v == VE2D || c->v == VE2D_PERF) && stencil == 0;
    c->fused32 = c->mixed && c->zs && c->d.mixed_sweep >= 1;
    if (c->fused32 && (rc = alloc_m2(c)) != PTS_OK) return rc;
    CK(cudaStreamSynchronize(c->stream));
    drop_graph(c);  // the captured check blocks hold the previous kernels
    return PTS_OK;
}

int pts_set_mixed_sweep(pts_ctx* c, int32_t mixed_sweep) {
    int rc = enter(c);
    if (rc) return rc;
    if (!c->mixed) return fail(c, PTS_E_STATE, "pts_set_mixed_sweep needs a MIXED context");
    if (mixed_sweep < 0 || mixed_sweep >= 1 + zfused32_num_configs())
        return fail(c, PTS_E_INVAL, "mixed_sweep out of range (0, 1 + tile < 1 + pts_mixed_sweep_tiles())");
    CK(cudaStreamSynchronize(c->stream));
    c->d.mixed_sweep = mixed_sweep;
    c->fused32 = c->zs && mixed_sweep >= 1;
    c->ftile = mixed_sweep >= 1 ? mixed_sweep - 1 : 0;
    if (c->fused32 && (rc = alloc_m2(c)) != PTS_OK) return rc;
    CK(cudaStreamSynchronize(c->stream));
    drop_graph(c);
    return PTS_OK;
}

int pts_mixed_sweep_tiles(void) { return zfused32_num_configs(); }

int pts_set_kernel_timing(pts_ctx* c, int32_t on) {
    int rc = enter(c);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->timing = on != 0;
    c->tev_n = 0;
    drop_graph(c);  // the next check block is captured with (or without) its events
    return PTS_OK;
}

int pts_kernel_times(pts_ctx* c, float* ms, int64_t cap, int64_t* count) {
    int rc = enter(c);
    if (rc) return rc;
    if (!count || (cap > 0 && !ms)) return fail(c, PTS_E_INVAL, "null argument");
    CK(cudaStreamSynchronize(c->stream));
    const int64_t n = c->timing && c->tev_n > 1 ? c->tev_n - 1 : 0;
    for (int64_t q = 0; q < n && q < cap; ++q) CK(cudaEventElapsedTime(&ms[q], c->tev[q], c->tev[q + 1]));
    *count = n;
    return PTS_OK;
}

int pts_stencil_tiles_2d(void) { return ystage_num_configs(); }

int pts_stencil_tiles(int32_t precision) {
    return precision == PTS_MIXED ? zstage32_num_configs() : zstage_num_configs();
}

int pts_stencil_vtiles(int32_t precision) {
    return precision == PTS_MIXED ? zvbc32_num_configs() : zvbc_num_configs();
}

int pts_stencil_tile_info(int32_t precision, int32_t tile, int32_t* tile_y, int32_t* ring_slots) {
    int ty = 0, r = 0;
    const bool ok = precision == PTS_MIXED ? zstage32_tile_info(tile, &ty, &r) : zstage_tile_info(tile, &ty, &r);
    if (!ok) return fail(nullptr, PTS_E_INVAL, "no such stencil tile");
    if (tile_y) *tile_y = ty;
    if (ring_slots) *ring_slots = r;
    return PTS_OK;
}

const char* pts_last_error(const pts_ctx* c) { return c ? c->err.c_str() : g_create_err.c_str(); }

int pts_create(const pts_desc* d, pts_ctx** out) {
    pts_ctx* c = nullptr;
    if (!d || !out) return fail(nullptr, PTS_E_INVAL, "null argument");
    *out = nullptr;
    if (d->variant < PTS_2D_V || d->variant > PTS_3D_V_DAMP) return fail(nullptr, PTS_E_INVAL, "unknown variant");
    if (d->precision != PTS_FP64 && d->precision != PTS_MIXED) return fail(nullptr, PTS_E_INVAL, "unknown precision");
    if (d->precision == PTS_MIXED && d->variant != PTS_3D_VE_PERF && d->variant != PTS_3D_V)
        return fail(nullptr, PTS_E_INVAL, "mixed precision is implemented for PTS_3D_VE_PERF and PTS_3D_V");
    const bool d3 = variant_is3d(d->variant);
    if (d->nx < 3 || d->ny < 3 || (d3 && d->nz < 3)) return fail(nullptr, PTS_E_INVAL, "each of nx, ny(, nz) must be >= 3");
    if ((int64_t)d->nx + 1 > (1 << 20) || (int64_t)d->ny + 1 > (1 << 20) || (d3 && (int64_t)d->nz + 1 > (1 << 20)))
        return fail(nullptr, PTS_E_INVAL, "grid extent too large");
    if (d->nout < 1) return fail(nullptr, PTS_E_INVAL, "nout must be >= 1");
    if (d->mixed_inner != 0 && d->mixed_inner != d->nout)
        return fail(nullptr, PTS_E_INVAL, "mixed_inner: the FP64 correction runs with every check, so it must be 0 or nout");
    if (!(d->lx > 0) || !(d->ly > 0) || (d3 && !(d->lz > 0))) return fail(nullptr, PTS_E_INVAL, "domain extents must be > 0");
    if (d->stencil != 0 && d->stencil != 1) return fail(nullptr, PTS_E_INVAL, "stencil must be 0 or 1");
    if (d->stencil_tile < 0 || d->stencil_tile >= tile_count(d3, d->precision == PTS_MIXED))
        return fail(nullptr, PTS_E_INVAL, "stencil_tile out of range (pts_stencil_tiles, pts_stencil_tiles_2d)");
    if (d->stencil_kz < 0) return fail(nullptr, PTS_E_INVAL, "stencil_kz must be >= 0");
    if (d->stencil_vtile < 0 ||
        d->stencil_vtile >= (d->precision == PTS_MIXED ? zvbc32_num_configs() : zvbc_num_configs()))
        return fail(nullptr, PTS_E_INVAL, "stencil_vtile out of range (pts_stencil_vtiles)");
    if (d->mixed_sweep < 0 || d->mixed_sweep >= 1 + zfused32_num_configs())
        return fail(nullptr, PTS_E_INVAL, "mixed_sweep out of range (0, 1 + tile < 1 + pts_mixed_sweep_tiles())");
    if (d->adjoint && ((d->variant != PTS_3D_V && d->variant != PTS_3D_VE_PERF) || d->precision != PTS_FP64 ||
                       d->single_pass))
        return fail(nullptr, PTS_E_INVAL,
                    "adjoint mode is implemented for PTS_3D_V and PTS_3D_VE_PERF in FP64 on the two-kernel path");
    c = new pts_ctx();
    c->d = *d;
    c->v = d->variant;
    c->d3 = d3;
    c->elastic = variant_elastic(c->v);
    c->perf = variant_perf(c->v);
    Geom& g = c->g;
    g.nx = d->nx;
    g.ny = d->ny;
    g.nz = d3 ? d->nz : 1;
    g.px = ((d->nx + 1) + 15) / 16 * 16;
    g.py = d->ny + 1;
    g.pz = d3 ? d->nz + 1 : 1;
    g.pxy = (int64_t)g.px * g.py;
    g.n = g.pxy * g.pz;
    if (g.n >= ((int64_t)1 << 31)) {
        delete c;
        return fail(nullptr, PTS_E_INVAL, "grid too large: more than 2^31 elements per field");
    }
    Num& n = c->n;
    n.lx = d->lx; n.ly = d->ly; n.lz = d3 ? d->lz : 1.0;
    n.dx = d->lx / d->nx;
    n.dy = d->ly / d->ny;
    n.dz = d3 ? d->lz / d->nz : 1.0;
    n._dx = 1.0 / n.dx;
    n._dy = 1.0 / n.dy;
    n._dz = 1.0 / n.dz;
    n.r = d->r;
    n.G = d->G;
    n.dt = d->dt;
    n.gdt = d->G * d->dt;
    n.Re = d->Re;
    n.Vpdt = (d3 ? std::min(std::min(n.dx, n.dy), n.dz) : std::min(n.dx, n.dy)) * d->CFL;
    n.max_l = d->max_l > 0 ? d->max_l : (d3 ? std::max(std::max(d->lx, d->ly), d->lz) : std::max(d->lx, d->ly));
    n.adjoint = d->adjoint ? 1 : 0;
    for (double& v : n.nsc) v = d->lx;  // norm_R* = ‖R‖/(Pmax-Pmin)*lx/√len (Stokes3D_ve_perf.jl:212-216)
    if (d3) set_damping(c, 4.0, 3.0, 1.0, 5.0);  // Stokes3D0_multixpu.jl:105-108
    else set_damping(c, 4.0, 2.0, 1.0, 3.0);     // Stokes2D_ve0.jl:95-98
    int rc = PTS_OK;
    auto bail = [&](int code) {
        g_create_err = c->err;
        pts_destroy(c);
        return code;
    };
    if (cudaGetDevice(&c->device) != cudaSuccess) {
        cudaGetLastError();
        c->err = "no CUDA device";
        return bail(PTS_E_CUDA);
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        c->err = "cudaStreamCreate failed";
        return bail(PTS_E_CUDA);
    }
    Fields64& f = c->f;
    double** always[] = {&f.Pt, &f.Vx, &f.Vy, &f.txx, &f.tyy, &f.txy, &f.Mus, &f.Must, &f.Gdt, &f.dtRho, &f.divV,
                         &f.Rx, &f.Ry, &f.Mus2};
    for (double** p : always)
        if ((rc = alloc_field(c, p)) != PTS_OK) return bail(rc);
    if (d3) {
        double** more[] = {&f.Vz, &f.tzz, &f.txz, &f.tyz, &f.Rz};
        for (double** p : more)
            if ((rc = alloc_field(c, p)) != PTS_OK) return bail(rc);
    }
    if (c->elastic) {
        double** olds[] = {&f.txx_o, &f.tyy_o, &f.txy_o};
        for (double** p : olds)
            if ((rc = alloc_field(c, p)) != PTS_OK) return bail(rc);
        if (d3) {
            double** olds3[] = {&f.tzz_o, &f.txz_o, &f.tyz_o};
            for (double** p : olds3)
                if ((rc = alloc_field(c, p)) != PTS_OK) return bail(rc);
        }
    }
    if (variant_damped(c->v)) {
        // the damped rates dVxdτ, dVydτ are iteration state (zero at start), and dτV, dτPt
        double** damp[] = {&f.dVx, &f.dVy, &f.dtVx, &f.dtVy, &f.dtPt};
        for (double** p : damp)
            if ((rc = alloc_field(c, p)) != PTS_OK) return bail(rc);
        if (d3) {
            double** damp3[] = {&f.dVz, &f.dtVz};
            for (double** p : damp3)
                if ((rc = alloc_field(c, p)) != PTS_OK) return bail(rc);
        }
    }
    c->mixed = d->precision == PTS_MIXED;
    c->fused = variant_fused(c->v) && d->single_pass != 0 && !c->mixed;
    // z-marching TMA-staged compute_Pt_τ!: the FP64 two-kernel path, and the FP32 sweeps
    c->zs = (c->v == VE3D || c->v == VE3D_PERF || c->v == V3D) && !c->fused && d->stencil == 0;
    c->ys = (c->v == V2D || c->v == VE2D || c->v == VE2D_PERF) && d->stencil == 0;
    if (c->mixed) {
        float** p32[] = {&c->m.dPt, &c->m.dVx, &c->m.dVy, &c->m.dVz, &c->m.dtxx, &c->m.dtyy, &c->m.dtzz, &c->m.dtxy,
                         &c->m.dtxz, &c->m.dtyz, &c->m.aP, &c->m.atxx, &c->m.atyy, &c->m.atzz, &c->m.atxy,
                         &c->m.atxz, &c->m.atyz, &c->m.aVx, &c->m.aVy, &c->m.aVz, &c->m.dtRho};
        for (float** p : p32) {
            void* q = nullptr;
            if (cudaMalloc(&q, (size_t)g.n * sizeof(float)) != cudaSuccess ||
                cudaMemsetAsync(q, 0, (size_t)g.n * sizeof(float), c->stream) != cudaSuccess) {
                cudaGetLastError();
                c->err = "allocation of the FP32 fields failed";
                return bail(PTS_E_NOMEM);
            }
            *p = (float*)q;
            c->owned32.push_back(*p);
        }
        void* q = nullptr;
        if (cudaMalloc(&q, (size_t)g.n * sizeof(float2)) != cudaSuccess ||
            cudaMemsetAsync(q, 0, (size_t)g.n * sizeof(float2), c->stream) != cudaSuccess) {
            cudaGetLastError();
            c->err = "allocation of the FP32 fields failed";
            return bail(PTS_E_NOMEM);
        }
        c->m.GM = (float2*)q;
        c->owned32.push_back((float*)q);
        c->fused32 = c->zs && d->mixed_sweep >= 1;
        c->ftile = d->mixed_sweep >= 1 ? d->mixed_sweep - 1 : 0;
        if (c->fused32 && (rc = alloc_m2(c)) != PTS_OK) return bail(rc);
    }
    if (c->fused) {
        for (int q = 0; q < 10; ++q)
            if ((rc = alloc_field(c, iterated(c->alt, q))) != PTS_OK) return bail(rc);
    }
    c->partials_cap = check_num_blocks(c->v, g);
    if (cudaMalloc((void**)&c->partials, (size_t)c->partials_cap * kCheckSlots * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c->d_result, sizeof(CheckResult)) != cudaSuccess ||
        cudaMalloc((void**)&c->d_kerr, sizeof(int)) != cudaSuccess ||
        cudaMemsetAsync(c->d_kerr, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_result, sizeof(CheckResult)) != cudaSuccess) {
        cudaGetLastError();
        c->err = "allocation of the check buffers failed";
        return bail(PTS_E_NOMEM);
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        c->err = std::string("initialisation: ") + cudaGetErrorString(cudaGetLastError());
        return bail(PTS_E_CUDA);
    }
    *out = c;
    return PTS_OK;
}

int pts_destroy(pts_ctx* c) {
    if (!c) return PTS_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    for (double* p : c->owned) cudaFree(p);
    for (float* p : c->owned32) cudaFree(p);
    if (c->partials) cudaFree(c->partials);
    if (c->d_result) cudaFree(c->d_result);
    if (c->d_kerr) cudaFree(c->d_kerr);
    if (c->d_incl) cudaFree(c->d_incl);
    if (c->h_result) cudaFreeHost(c->h_result);
    for (cudaEvent_t e : c->tev) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PTS_OK;
}

int pts_sync(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    return synced(c);
}

int pts_stream(pts_ctx* c, void** stream) {
    if (!c || !stream) return PTS_E_INVAL;
    *stream = (void*)c->stream;
    return PTS_OK;
}

int pts_field_shape(const pts_ctx* cc, int32_t id, int64_t shape[3]) {
    pts_ctx* c = const_cast<pts_ctx*>(cc);
    if (!c || !shape) return PTS_E_INVAL;
    FInfo fi;
    if (!field_info(c, id, &fi)) return fail(c, PTS_E_INVAL, "field not present for this variant: " + std::to_string(id));
    shape[0] = fi.e[0];
    shape[1] = fi.e[1];
    shape[2] = fi.e[2];
    return PTS_OK;
}

int pts_set_field(pts_ctx* c, int32_t id, const double* host, int64_t n) {
    int rc = enter(c);
    if (rc) return rc;
    if (!host) return fail(c, PTS_E_INVAL, "null host pointer");
    FInfo fi;
    if ((id == PTS_F_DVX || id == PTS_F_DVY || id == PTS_F_DVZ) && field_info(c, id, &fi) &&
        (rc = alloc_field(c, fi.ptr)) != PTS_OK)
        return rc;
    if ((rc = ensure_sources(c, id)) != PTS_OK) return rc;
    return copy3d(c, id, host, nullptr, n, cudaMemcpyHostToDevice);
}

int pts_get_field(pts_ctx* c, int32_t id, double* host, int64_t n) {
    int rc = enter(c);
    if (rc) return rc;
    if (!host) return fail(c, PTS_E_INVAL, "null host pointer");
    return copy3d(c, id, nullptr, host, n, cudaMemcpyDeviceToHost);
}

int pts_set_field_device(pts_ctx* c, int32_t id, const double* dev, int64_t n) {
    int rc = enter(c);
    if (rc) return rc;
    if (!dev) return fail(c, PTS_E_INVAL, "null device pointer");
    if ((rc = ensure_sources(c, id)) != PTS_OK) return rc;
    return copy3d(c, id, dev, nullptr, n, cudaMemcpyDeviceToDevice);
}

int pts_get_field_device(pts_ctx* c, int32_t id, double* dev, int64_t n) {
    int rc = enter(c);
    if (rc) return rc;
    if (!dev) return fail(c, PTS_E_INVAL, "null device pointer");
    return copy3d(c, id, nullptr, dev, n, cudaMemcpyDeviceToDevice);
}

int pts_init_inclusion(pts_ctx* c, double mus0, double musi, double radius2, double ebg) {
    int rc = enter(c);
    if (rc) return rc;
    for (double* p : c->owned) CK(cudaMemsetAsync(p, 0, (size_t)c->g.n * sizeof(double), c->stream));
    CK(launch_init_inclusion(c->v, c->g, c->f, c->n, mus0, musi, radius2, ebg, c->stream));
    return PTS_OK;
}

int pts_init_inclusions(pts_ctx* c, const pts_inclusion* list, int32_t count, double mus0, double ebg) {
    int rc = enter(c);
    if (rc) return rc;
    if (count < 0 || count > PTS_MAX_INCLUSIONS) return fail(c, PTS_E_INVAL, "inclusion count out of range");
    if (count > 0 && !list) return fail(c, PTS_E_INVAL, "null inclusion list");
    for (int32_t q = 0; q < count; ++q)
        if (!std::isfinite(list[q].x) || !std::isfinite(list[q].y) || !std::isfinite(list[q].z) ||
            !std::isfinite(list[q].r2))
            return fail(c, PTS_E_INVAL, "inclusion " + std::to_string(q) + ": centre and r2 must be finite");
    if (count > c->incl_cap) {
        if (c->d_incl) {
            CK(cudaStreamSynchronize(c->stream));
            cudaFree(c->d_incl);
            c->d_incl = nullptr;
            c->incl_cap = 0;
        }
        if (cudaMalloc((void**)&c->d_incl, (size_t)count * sizeof(pts_inclusion)) != cudaSuccess) {
            cudaGetLastError();
            c->d_incl = nullptr;
            return fail(c, PTS_E_NOMEM, "allocation of the inclusion list failed");
        }
        c->incl_cap = count;
    }
    if (count > 0) {
        CK(cudaMemcpyAsync(c->d_incl, list, (size_t)count * sizeof(pts_inclusion), cudaMemcpyHostToDevice, c->stream));
    }
    for (double* p : c->owned) CK(cudaMemsetAsync(p, 0, (size_t)c->g.n * sizeof(double), c->stream));
    CK(launch_init_inclusions(c->v, c->g, c->f, c->n, c->d_incl, count, mus0, ebg, c->stream));
    // the caller's list is borrowed for the call only
    CK(cudaStreamSynchronize(c->stream));
    return PTS_OK;
}

int pts_set_decomposition(pts_ctx* c, int32_t zoff, int32_t nz_global) {
    int rc = enter(c);
    if (rc) return rc;
    if (!c->d3) return fail(c, PTS_E_STATE, "a z-slab decomposition needs a 3D variant");
    if (zoff < 0 || nz_global < c->g.nz || zoff + c->g.nz > nz_global)
        return fail(c, PTS_E_INVAL, "the slab [zoff, zoff+nz) must lie in [0, nz_global)");
    Num& n = c->n;
    n.zoff = zoff;
    n.dz = c->d.lz / nz_global;  // dz = lz/nz_g() (Stokes3D_ve_multixpu.jl:139)
    n._dz = 1.0 / n.dz;
    n.Vpdt = std::min(std::min(n.dx, n.dy), n.dz) * c->d.CFL;
    set_damping(c, n.Vdmp, n.beta_n, n.Vsc, n.Ptsc);
    CK(cudaStreamSynchronize(c->stream));
    drop_graph(c);  // captured launches hold the previous numerics
    return PTS_OK;
}

int pts_compute_V_bc_planes(pts_ctx* c, int32_t k0, int32_t k1, void* stream) {
    int rc = enter(c);
    if (rc) return rc;
    if (!c->d3 || variant_damped(c->v) || c->mixed || c->f.Fx || c->n.adjoint)
        return fail(c, PTS_E_STATE,
                    "pts_compute_V_bc_planes needs an FP64 3D_VE, 3D_VE_PERF or 3D_V context without sources or adjoint mode");
    if (k0 < 0 || k1 > c->g.nz + 1 || k0 > k1)
        return fail(c, PTS_E_INVAL, "face planes [k0, k1) must lie in [0, nz+1]");
    CK(launch_V_bc_planes(c->v, c->g, c->f, c->n, k0, k1, stream ? (cudaStream_t)stream : c->stream));
    return PTS_OK;
}

// One z-plane k of a 3D field (the reference's extents) to or from a dense device buffer.
int plane_copy(pts_ctx* c, int32_t id, int32_t k, double* dev, int64_t n, bool to_field) {
    int rc = enter(c);
    if (rc) return rc;
    FInfo fi;
    if (!c->d3) return fail(c, PTS_E_STATE, "plane copies are for 3D fields");
    if (!field_info(c, id, &fi)) return fail(c, PTS_E_INVAL, "field not present for this variant: " + std::to_string(id));
    if (*fi.ptr == nullptr) return fail(c, PTS_E_STATE, "field not allocated: " + std::to_string(id));
    if (!dev) return fail(c, PTS_E_INVAL, "null device pointer");
    if (k < 0 || k >= fi.e[2]) return fail(c, PTS_E_INVAL, "plane index out of range");
    if (n != fi.e[0] * fi.e[1]) return fail(c, PTS_E_INVAL, "a plane of this field has " + std::to_string(fi.e[0] * fi.e[1]) + " elements");
    double* p = *fi.ptr + gidx(c->g, fi.s[0], fi.s[1], fi.s[2] + k);
    const size_t pitch = (size_t)c->g.px * sizeof(double), w = (size_t)fi.e[0] * sizeof(double);
    if (to_field)
        CK(cudaMemcpy2DAsync(p, pitch, dev, w, w, (size_t)fi.e[1], cudaMemcpyDeviceToDevice, c->stream));
    else
        CK(cudaMemcpy2DAsync(dev, w, p, pitch, w, (size_t)fi.e[1], cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PTS_OK;
}

int pts_get_plane_device(pts_ctx* c, int32_t id, int32_t k, double* dev, int64_t n) {
    return plane_copy(c, id, k, dev, n, false);
}

int pts_set_plane_device(pts_ctx* c, int32_t id, int32_t k, const double* dev, int64_t n) {
    return plane_copy(c, id, k, const_cast<double*>(dev), n, true);
}

int pts_check_partials(pts_ctx* c, double out[8]) {
    int rc = enter(c);
    if (rc) return rc;
    if (!out) return fail(c, PTS_E_INVAL, "null argument");
    if ((rc = enqueue_check(c)) != PTS_OK) return rc;
    if ((rc = synced(c)) != PTS_OK) return rc;
    const CheckResult& r = *c->h_result;
    const double v[8] = {r.sRx, r.sRy, r.sRz, r.sdiv, r.vmin, r.vmax, r.pmin, r.pmax};
    for (int q = 0; q < 8; ++q) out[q] = v[q];
    return PTS_OK;
}

int pts_set_norm_scales(pts_ctx* c, double sRx, double sRy, double sRz, double sdiv) {
    int rc = enter(c);
    if (rc) return rc;
    if (!(sRx > 0) || !(sRy > 0) || !(sRz > 0) || !(sdiv > 0)) return fail(c, PTS_E_INVAL, "scales must be > 0");
    c->n.nsc[0] = sRx;
    c->n.nsc[1] = sRy;
    c->n.nsc[2] = sRz;
    c->n.nsc[3] = sdiv;
    CK(cudaStreamSynchronize(c->stream));
    drop_graph(c);  // the captured check holds the previous scales
    return PTS_OK;
}

int pts_smooth(pts_ctx* c, int32_t nsweeps, double fact) {
    int rc = enter(c);
    if (rc) return rc;
    if (nsweeps < 0) return fail(c, PTS_E_INVAL, "nsweeps < 0");
    // Mus2 .= Mus, then ping-pong (the boundary cells of both stay the initial Mus)
    CK(cudaMemcpyAsync(c->f.Mus2, c->f.Mus, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    for (int s = 0; s < nsweeps; ++s) {
        CK(launch_smooth(c->v, c->g, c->f.Mus2, c->f.Mus, fact, c->stream));
        std::swap(c->f.Mus, c->f.Mus2);
    }
    drop_graph(c);  // the graph captured the old Mus pointer
    return PTS_OK;
}

int pts_compute_maxloc(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    CK(launch_maxloc(c->v, c->g, c->f.Must, c->f.Mus, c->stream));
    return PTS_OK;
}

int pts_compute_iter_params(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    CK(launch_iter_params(c->v, c->g, c->f, c->n, c->stream));
    return PTS_OK;
}

int pts_set_damping(pts_ctx* c, double Vdmp, double beta_n, double Vsc, double Ptsc) {
    int rc = enter(c);
    if (rc) return rc;
    if (!variant_damped(c->v))
        return fail(c, PTS_E_INVAL, "pts_set_damping needs PTS_2D_V_DAMP, PTS_2D_VE_DAMP or PTS_3D_V_DAMP");
    if (!(Vsc > 0) || !(Ptsc > 0) || !std::isfinite(Vdmp) || !std::isfinite(beta_n) || !(beta_n > -1.0))
        return fail(c, PTS_E_INVAL, "damping numerics: Vsc, Ptsc must be > 0, beta_n > -1, Vdmp finite");
    set_damping(c, Vdmp, beta_n, Vsc, Ptsc);
    drop_graph(c);  // the captured launches hold the old numerics
    return PTS_OK;
}

int pts_assign_tau(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    if (!c->elastic) return PTS_OK;  // viscous scripts have no τ_o
    Fields64& f = c->f;
    std::pair<double*, double*> cp[] = {{f.txx_o, f.txx}, {f.tyy_o, f.tyy}, {f.txy_o, f.txy},
                                        {f.tzz_o, f.tzz}, {f.txz_o, f.txz}, {f.tyz_o, f.tyz}};
    for (auto& pr : cp)
        if (pr.first) CK(cudaMemcpyAsync(pr.first, pr.second, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    return PTS_OK;
}

int pts_compute_P(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    CK(launch_Pt_tau(c->v, c->g, c->f, c->n, ROLE_P, !c->perf, c->stream));
    return PTS_OK;
}

int pts_compute_tau(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    CK(launch_Pt_tau(c->v, c->g, c->f, c->n, ROLE_TAU, false, c->stream));
    return PTS_OK;
}

int pts_compute_dV(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    if (c->n.adjoint) return fail(c, PTS_E_INVAL, "adjoint mode iterates with pts_compute_V_bc / pts_iterate / pts_solve");
    double** dv[] = {&c->f.dVx, &c->f.dVy, &c->f.dVz};
    for (int q = 0; q < (c->d3 ? 3 : 2); ++q)
        if ((rc = alloc_field(c, dv[q])) != PTS_OK) return rc;
    CK(launch_dV(c->v, c->g, c->f, c->n, c->stream));
    return PTS_OK;
}

int pts_compute_V(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    if (c->n.adjoint) return fail(c, PTS_E_INVAL, "adjoint mode iterates with pts_compute_V_bc / pts_iterate / pts_solve");
    if (!c->f.dVx) return fail(c, PTS_E_STATE, "compute_V needs dV: call pts_compute_dV first");
    CK(launch_add_dV(c->v, c->g, c->f, c->stream));
    return PTS_OK;
}

int pts_apply_bc(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    if (c->n.adjoint) return fail(c, PTS_E_INVAL, "adjoint mode keeps the ghosts at zero: no free-slip copies");
    CK(launch_V_bc(c->v, c->g, c->f, c->n, false, c->stream));
    return PTS_OK;
}

int pts_compute_Pt_tau(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    return Pt_tau(c, true);
}

int pts_compute_V_bc(pts_ctx* c) {
    int rc = enter(c);
    if (rc) return rc;
    return V_bc(c, true);
}

int pts_sweep32_kernel(pts_ctx* c, int32_t which) {
    int rc = enter(c);
    if (rc) return rc;
    if (!c->mixed) return fail(c, PTS_E_STATE, "pts_sweep32_kernel needs a MIXED context");
    if (which == 0) {
        if (c->zs)
            CK(launch_corr_A32_zs(c->v, c->d.stencil_tile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
        else
            CK(launch_corr_A32(c->v, c->g, c->m, c->n, c->stream));
    } else if (which == 1) {
        if (c->zs)
            CK(launch_corr_B32_zs(c->v, c->d.stencil_vtile, c->g, c->m, c->n, c->d.stencil_kz, c->d_kerr, c->stream));
        else
            CK(launch_corr_B32(c->v, c->g, c->m, c->n, c->stream));
    } else {
        return fail(c, PTS_E_INVAL, "which must be 0 (compute_Pt_τ!) or 1 (compute_V! + bc)");
    }
    return PTS_OK;
}

int pts_compute_res(pts_ctx* c, pts_check* out) {
    int rc = enter(c);
    if (rc) return rc;
    if ((rc = enqueue_check(c)) != PTS_OK) return rc;
    if ((rc = synced(c)) != PTS_OK) return rc;
    if (out) to_check(*c->h_result, out);
    return c->h_result->flag_nan != 0.0 ? fail(c, PTS_E_NAN, "NaN in the residual check") : PTS_OK;
}

int pts_apply_operator(pts_ctx* c, pts_check* out) {
    int rc = enter(c);
    if (rc) return rc;
    if (c->v != PTS_3D_V || c->mixed) return fail(c, PTS_E_INVAL, "pts_apply_operator needs 3D_V in FP64");
    CK(launch_tau_exact(c->g, c->f, c->n, c->stream));
    if ((rc = enqueue_check(c)) != PTS_OK) return rc;
    if ((rc = synced(c)) != PTS_OK) return rc;
    if (out) to_check(*c->h_result, out);
    return PTS_OK;
}

namespace {
int gradient(pts_ctx* fwd, pts_ctx* adj, bool add) {
    pts_ctx* c = fwd;
    int rc = enter(c);
    if (rc) return rc;
    if (!adj) return fail(c, PTS_E_INVAL, "null adjoint context");
    if ((c->v != PTS_3D_V && c->v != PTS_3D_VE_PERF) || adj->v != c->v || c->mixed || adj->mixed)
        return fail(c, PTS_E_INVAL, "the gradient needs two 3D_V or two 3D_VE_PERF contexts in FP64");
    if (add && c->v == PTS_3D_V) return fail(c, PTS_E_INVAL, "pts_gradient_logmu_add is for PTS_3D_VE_PERF");
    if (c->n.adjoint || !adj->n.adjoint)
        return fail(c, PTS_E_INVAL, "pts_gradient_logmu takes a forward context and an adjoint-mode context");
    if (adj->g.nx != c->g.nx || adj->g.ny != c->g.ny || adj->g.nz != c->g.nz || adj->n.dx != c->n.dx ||
        adj->n.dy != c->n.dy || adj->n.dz != c->n.dz || adj->device != c->device)
        return fail(c, PTS_E_INVAL, "forward and adjoint contexts differ in grid, spacing or device");
    if ((rc = alloc_field(c, &c->f.grad)) != PTS_OK) return rc;
    CK(cudaStreamSynchronize(adj->stream));
    if (c->v == PTS_3D_V) CK(launch_grad_logmu(c->g, c->f, adj->f, c->n, c->stream));
    else CK(launch_grad_logmu_ve(c->g, c->f, adj->f, add, c->stream));
    return synced(c);
}
}  // namespace

int pts_gradient_logmu(pts_ctx* fwd, pts_ctx* adj) { return gradient(fwd, adj, false); }
int pts_gradient_logmu_add(pts_ctx* fwd, pts_ctx* adj) { return gradient(fwd, adj, true); }


int pts_iterate(pts_ctx* c, int64_t niter) {
    int rc = enter(c);
    if (rc) return rc;
    if (niter < 0) return fail(c, PTS_E_INVAL, "niter < 0");
    if (c->mixed && niter > 0 && (rc = mixed_prepare(c)) != PTS_OK) return rc;
    return enqueue_block(c, niter, true);
}

int pts_solve(pts_ctx* c, pts_solve_info* info) {
    int rc = enter(c);
    if (rc) return rc;
    if (c->mixed && (rc = mixed_prepare(c)) != PTS_OK) return rc;
    const int64_t nout = c->d.nout;
    const double eps = c->d.eps;
    const int64_t last_iter = (int64_t)std::floor(c->d.iter_max);  // loop runs while iter <= iter_max
    int64_t iter = 0;
    double err = 2 * eps;
    pts_solve_info res;
    memset(&res, 0, sizeof(res));
    res.last.err = err;
    bool converged = false;
    while (err > eps && iter <= last_iter) {
        const int64_t till_check = nout - iter % nout;
        const int64_t remaining = last_iter - iter + 1;
        if (remaining >= till_check) {
            if (till_check == nout) {
                if ((rc = launch_chunk(c)) != PTS_OK) return rc;
            } else {
                if ((rc = enqueue_block(c, till_check, true)) != PTS_OK) return rc;
                if ((rc = enqueue_check(c)) != PTS_OK) return rc;
            }
            if ((rc = synced(c)) != PTS_OK) return rc;
            iter += till_check;
            to_check(*c->h_result, &res.last);
            res.nchecks++;
            err = c->h_result->err;
            if (c->h_result->flag_nan != 0.0) {
                res.iters = iter;
                if (info) *info = res;
                return fail(c, PTS_E_NAN, "NaN");
            }
            if (!(err > eps)) converged = true;
        } else {
            if ((rc = enqueue_block(c, remaining, true)) != PTS_OK) return rc;
            iter += remaining;
            if ((rc = synced(c)) != PTS_OK) return rc;
        }
    }
    res.iters = iter;
    res.converged = converged ? 1 : 0;
    if (info) *info = res;
    return PTS_OK;
}

int pts_run(pts_ctx* c, int32_t nt, int64_t* iters_per_step, pts_solve_info* info) {
    int rc = enter(c);
    if (rc) return rc;
    if (nt < 0) return fail(c, PTS_E_INVAL, "nt < 0");
    pts_solve_info step;
    memset(&step, 0, sizeof(step));
    int64_t ittot = 0;
    for (int32_t it = 0; it < nt; ++it) {
        if ((rc = pts_assign_tau(c)) != PTS_OK) return rc;
        rc = pts_solve(c, &step);
        ittot += step.iters;
        if (iters_per_step) iters_per_step[it] = step.iters;
        if (rc != PTS_OK) {
            step.iters = ittot;
            if (info) *info = step;
            return rc;
        }
    }
    step.iters = ittot;
    if (info) *info = step;
    return PTS_OK;
}

}  // extern "C"
