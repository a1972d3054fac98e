// pts_batch.cu -- host side of the batched 2D viscous sweep: many uneven instances in one
// persistent cooperative launch (kernel k2_batch in pts_kernels64.cu).
//
// Layout: one arena per field holds every instance back to back, each in its own padded
// unified layout (px = round_up(nx+1, 16), py = ny+1) and starting on a 256-byte boundary;
// BInst carries each instance's geometry, numerics, offset and tile range. The tile list
// depends on the tile shape, which the autotuner picks (pts_batch_set_tile).
//
// Numerics are those of the reference's sweep script (scripts/Stokes2D_param.jl): the
// iteration parameters come from Musτ .= μs0 (:190-192), so Gdτ and dτ_Rho are one number
// per instance, computed here in compute_iter_params!'s order and held in BInst; no array
// of Musτ, Gdτ or dτ_Rho is stored or read.
//
// A batch made by pts_batch_create_ve is the visco-elastic aspect-ratio sweep instead
// (scripts/Stokes2D_ve_param.jl over runme_Stokes2D_aspect_ratio.jl's FACT x NSUB x RESOL,
// kernel k2_batch_ve): per-cell iteration parameters from the local-max viscosity, old
// stresses, nt physical steps per instance and a check cadence per instance.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "pts_internal.h"

using namespace pts;

struct pts_batch {
    pts_batch_desc d{};
    bool ve = false;                        // made by pts_batch_create_ve
    std::vector<pts_batch_ve_instance> vin; // its instances
    BStateVE sv{};
    std::vector<pts_batch_instance> in;
    std::vector<BInst> hi;
    int n = 0;
    int tile = 1;
    int ntiles = 0;
    int64_t total = 0;  // elements per arena
    cudaStream_t stream = nullptr;
    Fields64 F{};
    BState st{};
    BInst* d_inst = nullptr;
    std::vector<void*> owned;
    int* h_nactive = nullptr;  // pinned: n, copied to the device at each solve
    cudaGraphExec_t graph = nullptr;
    int64_t graph_iter_last = -1;
    int graph_tile = -1;
    int device = 0;
    std::string err;
};

namespace {

int bfail(pts_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    else set_global_error(m.c_str());
    return code;
}

#define BCK(call)                                                                                              \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return bfail(b, PTS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

Fields64 shifted(const Fields64& F, int64_t off) {
    Fields64 f = F;
    double** p[] = {&f.Pt,  &f.Vx,   &f.Vy,    &f.txx,   &f.tyy,   &f.txy,   &f.Mus,  &f.divV,
                    &f.Rx,  &f.Ry,   &f.Mus2,  &f.rhog,  &f.rhog2, &f.txx_o, &f.tyy_o, &f.txy_o,
                    &f.Must, &f.Gdt, &f.dtRho};
    for (double** q : p)
        if (*q) *q = *q + off;
    return f;
}

void drop_graph(pts_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_iter_last = -1;
    b->graph_tile = -1;
}

int build_tiles(pts_batch* b) {
    int tx, ty;
    batch_tile_dims(b->tile, &tx, &ty);
    int64_t ntiles = 0;
    for (int q = 0; q < b->n; ++q) {
        BInst& I = b->hi[q];
        I.ntx = (I.g.nx + 1 + tx - 1) / tx;
        I.nty = (I.g.ny + 1 + ty - 1) / ty;
        I.tile0 = (int)ntiles;
        ntiles += (int64_t)I.ntx * I.nty;
    }
    if (ntiles >= (int64_t)1 << 31) return bfail(b, PTS_E_INVAL, "too many tiles in the sweep");
    b->ntiles = (int)ntiles;
    if (b->st.partials) cudaFree(b->st.partials);
    b->st.partials = nullptr;
    BCK(cudaMalloc((void**)&b->st.partials, sizeof(double) * kCheckSlots * ntiles));
    BCK(cudaMemcpy(b->d_inst, b->hi.data(), sizeof(BInst) * b->n, cudaMemcpyHostToDevice));
    drop_graph(b);
    return PTS_OK;
}

}  // namespace

extern "C" {

const char* pts_batch_last_error(const pts_batch* b) { return b ? b->err.c_str() : pts_last_error(nullptr); }

int pts_batch_create(const pts_batch_desc* d, const pts_batch_instance* inst, int32_t n, pts_batch** out) {
    pts_batch* b = nullptr;
    if (!d || !inst || !out || n < 1) return bfail(nullptr, PTS_E_INVAL, "null argument or n < 1");
    *out = nullptr;
    if (d->nout < 1) return bfail(nullptr, PTS_E_INVAL, "nout must be >= 1");
    if (d->tile < 0 || d->tile >= kBatchTileShapes) return bfail(nullptr, PTS_E_INVAL, "tile shape must be 0..3");
    int64_t total = 0;
    for (int q = 0; q < n; ++q) {
        if (inst[q].nx < 3 || inst[q].ny < 3) return bfail(nullptr, PTS_E_INVAL, "each instance needs nx, ny >= 3");
        if (!(inst[q].lx > 0) || !(inst[q].ly > 0)) return bfail(nullptr, PTS_E_INVAL, "box extents must be > 0");
        const int64_t px = ((inst[q].nx + 1) + 15) / 16 * 16;
        total += (px * (inst[q].ny + 1) + 31) / 32 * 32;
    }
    b = new pts_batch();
    b->d = *d;
    b->n = n;
    b->tile = d->tile;
    b->in.assign(inst, inst + n);
    b->hi.resize(n);
    int64_t off = 0;
    for (int q = 0; q < n; ++q) {
        const pts_batch_instance& s = inst[q];
        BInst& I = b->hi[q];
        memset(&I, 0, sizeof(I));
        I.g.nx = s.nx;
        I.g.ny = s.ny;
        I.g.nz = 1;
        I.g.px = ((s.nx + 1) + 15) / 16 * 16;
        I.g.py = s.ny + 1;
        I.g.pz = 1;
        I.g.pxy = (int64_t)I.g.px * I.g.py;
        I.g.n = I.g.pxy;
        Num& m = I.n;
        m.lx = s.lx;
        m.ly = s.ly;
        m.lz = 1.0;
        m.dx = s.lx / s.nx;
        m.dy = s.ly / s.ny;
        m.dz = 1.0;
        m._dx = 1.0 / m.dx;
        m._dy = 1.0 / m.dy;
        m._dz = 1.0;
        m.r = d->r;
        m.Re = d->Re;
        m.G = 1.0;
        m.dt = 1.0;
        m.gdt = 1.0;
        m.Vpdt = std::min(m.dx, m.dy) * d->CFL;
        m.max_l = std::max(s.lx, s.ly);
        I.off = off;
        I.ly = s.ly;
        I.lenRx = (double)(s.nx - 1) * (s.ny - 2);
        I.lenRy = (double)(s.nx - 2) * (s.ny - 1);
        I.lenDiv = (double)s.nx * s.ny;
        // compute_iter_params! with Musτ = μs0 = 1 (Stokes2D_param.jl:36-40,190-192)
        const double mus0 = 1.0;
        I.dR = m.Vpdt * m.max_l / m.Re / mus0;
        I.Gd = (m.Vpdt * m.Vpdt) / I.dR / (m.r + 2.0);
        // iterMax = 100max(nx,ny) (Stokes2D_param.jl:146) unless the descriptor sets one
        I.iter_last = d->iter_max > 0 ? (int64_t)std::floor(d->iter_max) : 100 * (int64_t)std::max(s.nx, s.ny);
        off += (I.g.pxy + 31) / 32 * 32;
    }
    b->total = total;
    auto bail = [&](int code) {
        set_global_error(b->err.c_str());
        pts_batch_destroy(b);
        return code;
    };
    if (cudaGetDevice(&b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        b->err = "no CUDA device / stream";
        return bail(PTS_E_CUDA);
    }
    Fields64& F = b->F;
    double** arenas[] = {&F.Pt, &F.Vx, &F.Vy, &F.txx, &F.tyy, &F.txy, &F.Mus, &F.divV,
                         &F.Rx, &F.Ry, &F.Mus2, &F.rhog, &F.rhog2};
    for (double** p : arenas) {
        void* q = nullptr;
        if (cudaMalloc(&q, sizeof(double) * total) != cudaSuccess ||
            cudaMemsetAsync(q, 0, sizeof(double) * total, b->stream) != cudaSuccess) {
            cudaGetLastError();
            b->err = "allocation of the sweep fields failed";
            return bail(PTS_E_NOMEM);
        }
        *p = (double*)q;
        b->owned.push_back(q);
    }
    void *c1 = nullptr, *c2 = nullptr, *c3 = nullptr, *c4 = nullptr, *c5 = nullptr, *c6 = nullptr, *c7 = nullptr;
    if (cudaMalloc(&c1, sizeof(int) * n) != cudaSuccess || cudaMalloc(&c2, sizeof(int64_t) * n) != cudaSuccess ||
        cudaMalloc(&c3, sizeof(double) * n) != cudaSuccess || cudaMalloc(&c4, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c5, sizeof(int)) != cudaSuccess || cudaMalloc(&c6, sizeof(BInst) * n) != cudaSuccess ||
        cudaMalloc(&c7, sizeof(int) * (2 * (size_t)n + 3)) != cudaSuccess ||
        cudaMallocHost((void**)&b->h_nactive, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        b->err = "allocation of the sweep state failed";
        return bail(PTS_E_NOMEM);
    }
    for (void* p : {c1, c2, c3, c4, c5, c6, c7}) b->owned.push_back(p);
    b->st.converged = (int*)c1;
    b->st.iters = (int64_t*)c2;
    b->st.err = (double*)c3;
    b->st.nactive = (int*)c4;
    b->st.nan_flag = (int*)c5;
    b->d_inst = (BInst*)c6;
    b->st.act = (int*)c7;
    *b->h_nactive = n;
    int rc = build_tiles(b);
    if (rc != PTS_OK) return bail(rc);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->err = std::string("initialisation: ") + cudaGetErrorString(cudaGetLastError());
        return bail(PTS_E_CUDA);
    }
    *out = b;
    return PTS_OK;
}

int pts_batch_create_ve(const pts_batch_desc* d, const pts_batch_ve_instance* inst, int32_t n, pts_batch** out) {
    if (!d || !inst || !out || n < 1) return bfail(nullptr, PTS_E_INVAL, "null argument or n < 1");
    *out = nullptr;
    if (d->tile < 0 || d->tile >= kBatchTileShapes) return bfail(nullptr, PTS_E_INVAL, "tile shape must be 0..3");
    if (!(d->eps > 0) || !(d->CFL > 0) || !(d->Re > 0) || !std::isfinite(d->r))
        return bfail(nullptr, PTS_E_INVAL, "eps, CFL, Re must be > 0 and r finite");
    int64_t total = 0;
    for (int q = 0; q < n; ++q) {
        const pts_batch_ve_instance& s = inst[q];
        if (s.ny < 3 || s.nsub < 1 || (int64_t)s.nsub * (s.ny + 1) - 1 > (1 << 20))
            return bfail(nullptr, PTS_E_INVAL, "each instance needs ny >= 3 and 1 <= nsub*(ny+1) <= 2^20");
        if (s.nt < 1 || s.nt > kBatchMaxSteps)
            return bfail(nullptr, PTS_E_INVAL, "each instance needs 1 <= nt <= " + std::to_string(kBatchMaxSteps));
        if (!(s.fact > 0) || !(s.ly > 0) || !(s.musi > 0) || !std::isfinite(s.fact) || !std::isfinite(s.ly) ||
            !std::isfinite(s.musi))
            return bfail(nullptr, PTS_E_INVAL, "fact, ly and musi must be finite and > 0");
        const int64_t nx = (int64_t)s.nsub * (s.ny + 1) - 1;
        const int64_t px = (nx + 1 + 15) / 16 * 16;
        total += (px * (s.ny + 1) + 31) / 32 * 32;
    }
    pts_batch* b = new pts_batch();
    b->ve = true;
    b->d = *d;
    b->n = n;
    b->tile = d->tile;
    b->vin.assign(inst, inst + n);
    b->hi.resize(n);
    int64_t off = 0;
    for (int q = 0; q < n; ++q) {
        const pts_batch_ve_instance& s = inst[q];
        BInst& I = b->hi[q];
        memset(&I, 0, sizeof(I));
        // Stokes2D_ve_param.jl:99-111: lx = nsub*ly, nx = nsub*(ny+1)-1, dx, dy, Vpdτ, min_lxy
        const int nx = s.nsub * (s.ny + 1) - 1, ny = s.ny;
        const double lx = (double)s.nsub * s.ly, ly = s.ly;
        I.g.nx = nx;
        I.g.ny = ny;
        I.g.nz = 1;
        I.g.px = ((nx + 1) + 15) / 16 * 16;
        I.g.py = ny + 1;
        I.g.pz = 1;
        I.g.pxy = (int64_t)I.g.px * I.g.py;
        I.g.n = I.g.pxy;
        Num& m = I.n;
        m.lx = lx;
        m.ly = ly;
        m.lz = 1.0;
        m.dx = lx / nx;
        m.dy = ly / ny;
        m.dz = 1.0;
        m._dx = 1.0 / m.dx;
        m._dy = 1.0 / m.dy;
        m._dz = 1.0;
        m.r = d->r;
        m.Re = d->Re;
        m.G = 1.0;   // G = 1, ξ = 1, μs0 = 1: dt = μs0/(G*ξ) = 1 (:91-96)
        m.dt = 1.0;
        m.gdt = 1.0;
        m.Vpdt = std::min(m.dx, m.dy) * d->CFL;
        m.max_l = s.fact * std::min(lx, ly);
        m.nsc[0] = lx;
        m.nsc[1] = ly;
        m.nsc[2] = lx;
        m.nsc[3] = ly;
        I.off = off;
        I.lx = lx;
        I.ly = ly;
        I.lenRx = (double)(nx - 1) * (ny - 2);
        I.lenRy = (double)(nx - 2) * (ny - 1);
        I.lenDiv = (double)nx * ny;
        // nout = 1nx and iterMax = 100nx (:103-105) unless the descriptor sets them
        I.nout = d->nout > 0 ? d->nout : nx;
        I.iter_last = d->iter_max > 0 ? (int64_t)std::floor(d->iter_max) : 100 * (int64_t)nx;
        I.nt = s.nt;
        off += (I.g.pxy + 31) / 32 * 32;
    }
    b->total = total;
    auto bail = [&](int code) {
        set_global_error(b->err.c_str());
        pts_batch_destroy(b);
        return code;
    };
    if (cudaGetDevice(&b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        b->err = "no CUDA device / stream";
        return bail(PTS_E_CUDA);
    }
    Fields64& F = b->F;
    double** arenas[] = {&F.Pt,    &F.Vx,    &F.Vy,    &F.txx, &F.tyy, &F.txy,   &F.txx_o, &F.tyy_o, &F.txy_o,
                         &F.Mus,   &F.Mus2,  &F.Must,  &F.Gdt, &F.dtRho, &F.divV, &F.Rx,    &F.Ry};
    for (double** p : arenas) {
        void* q = nullptr;
        if (cudaMalloc(&q, sizeof(double) * total) != cudaSuccess ||
            cudaMemsetAsync(q, 0, sizeof(double) * total, b->stream) != cudaSuccess) {
            cudaGetLastError();
            b->err = "allocation of the sweep fields failed";
            return bail(PTS_E_NOMEM);
        }
        *p = (double*)q;
        b->owned.push_back(q);
    }
    const size_t bytes[] = {sizeof(int) * n,    sizeof(int64_t) * n, sizeof(double) * n,  sizeof(int),
                            sizeof(int),        sizeof(BInst) * n,   sizeof(int) * (2 * (size_t)n + 3),
                            sizeof(int64_t) * n, sizeof(int) * n,    sizeof(int64_t) * n * kBatchMaxSteps,
                            sizeof(int) * n,    sizeof(int64_t)};
    void* c[12] = {};
    for (int q = 0; q < 12; ++q) {
        if (cudaMalloc(&c[q], bytes[q]) != cudaSuccess) {
            cudaGetLastError();
            b->err = "allocation of the sweep state failed";
            return bail(PTS_E_NOMEM);
        }
        b->owned.push_back(c[q]);
    }
    if (cudaMallocHost((void**)&b->h_nactive, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        b->err = "allocation of the sweep state failed";
        return bail(PTS_E_NOMEM);
    }
    b->st.converged = (int*)c[0];
    b->st.iters = (int64_t*)c[1];
    b->st.err = (double*)c[2];
    b->st.nactive = (int*)c[3];
    b->st.nan_flag = (int*)c[4];
    b->d_inst = (BInst*)c[5];
    b->st.act = (int*)c[6];
    b->sv.start = (int64_t*)c[7];
    b->sv.steps = (int*)c[8];
    b->sv.step_iters = (int64_t*)c[9];
    b->sv.assign = (int*)c[10];
    b->sv.next_event = (int64_t*)c[11];
    *b->h_nactive = n;
    int rc = build_tiles(b);
    if (rc != PTS_OK) return bail(rc);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->err = std::string("initialisation: ") + cudaGetErrorString(cudaGetLastError());
        return bail(PTS_E_CUDA);
    }
    *out = b;
    return PTS_OK;
}

int pts_batch_steps(pts_batch* b, int32_t q, int64_t* iters, int32_t max_steps, int32_t* nsteps) {
    if (!b || !iters || !nsteps || max_steps < 0) return PTS_E_INVAL;
    if (!b->ve) return bfail(b, PTS_E_INVAL, "per-step iteration counts exist only for a visco-elastic sweep");
    if (q < 0 || q >= b->n) return bfail(b, PTS_E_INVAL, "instance out of range");
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->stream));
    int done = 0;
    BCK(cudaMemcpy(&done, b->sv.steps + q, sizeof(int), cudaMemcpyDeviceToHost));
    done = std::min(done, kBatchMaxSteps);
    const int k = std::min(done, (int)max_steps);
    if (k > 0)
        BCK(cudaMemcpy(iters, b->sv.step_iters + (int64_t)q * kBatchMaxSteps, sizeof(int64_t) * k,
                       cudaMemcpyDeviceToHost));
    *nsteps = done;
    return PTS_OK;
}

int pts_batch_destroy(pts_batch* b) {
    if (!b) return PTS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (void* p : b->owned) cudaFree(p);
    if (b->st.partials) cudaFree(b->st.partials);
    if (b->h_nactive) cudaFreeHost(b->h_nactive);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return PTS_OK;
}

int pts_batch_stream(pts_batch* b, void** stream) {
    if (!b || !stream) return PTS_E_INVAL;
    *stream = (void*)b->stream;
    return PTS_OK;
}

int pts_batch_set_tile(pts_batch* b, int32_t tile) {
    if (!b) return PTS_E_INVAL;
    if (tile < 0 || tile >= kBatchTileShapes) return bfail(b, PTS_E_INVAL, "tile shape must be 0..3");
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->stream));
    b->tile = tile;
    return build_tiles(b);
}

// Set-up of the visco-elastic sweep, instance by instance as Stokes2D_ve_param.jl:126-150
// does it: pure-shear velocities and every other field zero, Mus with nsub inclusions, 10
// smooth! sweeps, compute_maxloc! + bc on Musτ, compute_iter_params! (with min_lxy).
static int setup_ve(pts_batch* b) {
    Fields64& F = b->F;
    double* zeroed[] = {F.Pt, F.Vx, F.Vy, F.txx, F.tyy, F.txy, F.txx_o, F.tyy_o, F.txy_o,
                        F.Mus, F.Mus2, F.Must, F.Gdt, F.dtRho, F.divV, F.Rx, F.Ry};
    for (double* p : zeroed) BCK(cudaMemsetAsync(p, 0, sizeof(double) * b->total, b->stream));
    for (int q = 0; q < b->n; ++q) {
        const BInst& I = b->hi[q];
        const Fields64 f = shifted(F, I.off);
        BCK(launch_init_inclusion(VE2D, I.g, f, I.n, 1.0, 1.0, 0.0, 1.0, b->stream));  // εbg = 1, Mus = μs0
        BCK(launch_init_ve_param(I.g, f, I.n, b->vin[q].nsub, 1.0, b->vin[q].musi, b->stream));
    }
    BCK(cudaMemcpyAsync(F.Mus2, F.Mus, sizeof(double) * b->total, cudaMemcpyDeviceToDevice, b->stream));
    for (int sweep = 0; sweep < 10; ++sweep) {
        for (int q = 0; q < b->n; ++q)
            BCK(launch_smooth(VE2D, b->hi[q].g, F.Mus2 + b->hi[q].off, F.Mus + b->hi[q].off, 1.0, b->stream));
        std::swap(F.Mus, F.Mus2);
    }
    for (int q = 0; q < b->n; ++q) {
        const BInst& I = b->hi[q];
        BCK(launch_maxloc(VE2D, I.g, F.Must + I.off, F.Mus + I.off, b->stream));
        BCK(launch_iter_params(VE2D, I.g, shifted(F, I.off), I.n, b->stream));
    }
    drop_graph(b);  // the arenas of Mus and Mus2 may have swapped
    BCK(cudaStreamSynchronize(b->stream));
    return PTS_OK;
}

int pts_batch_setup(pts_batch* b) {
    if (!b) return PTS_E_INVAL;
    BCK(cudaSetDevice(b->device));
    if (b->ve) return setup_ve(b);
    Fields64& F = b->F;
    double* zeroed[] = {F.Pt, F.Vx, F.Vy, F.txx, F.tyy, F.txy, F.divV, F.Rx, F.Ry};
    for (double* p : zeroed) BCK(cudaMemsetAsync(p, 0, sizeof(double) * b->total, b->stream));
    for (int q = 0; q < b->n; ++q) {
        const BInst& I = b->hi[q];
        const pts_batch_instance& s = b->in[q];
        BCK(launch_init_sweep(I.g, shifted(F, I.off), I.n, s.musi, s.radius2, s.rhogi, s.ebg, b->stream));
    }
    // Mus2 .= Mus; ρg2 .= ρg; 10 x (smooth!(Mus2, Mus); swap; smooth!(ρg2, ρg); swap)  (Stokes2D_param.jl:182-189)
    BCK(cudaMemcpyAsync(F.Mus2, F.Mus, sizeof(double) * b->total, cudaMemcpyDeviceToDevice, b->stream));
    BCK(cudaMemcpyAsync(F.rhog2, F.rhog, sizeof(double) * b->total, cudaMemcpyDeviceToDevice, b->stream));
    for (int sweep = 0; sweep < 10; ++sweep) {
        for (int q = 0; q < b->n; ++q)
            BCK(launch_smooth(V2D, b->hi[q].g, F.Mus2 + b->hi[q].off, F.Mus + b->hi[q].off, 1.0, b->stream));
        std::swap(F.Mus, F.Mus2);
        for (int q = 0; q < b->n; ++q)
            BCK(launch_smooth(V2D, b->hi[q].g, F.rhog2 + b->hi[q].off, F.rhog + b->hi[q].off, 1.0, b->stream));
        std::swap(F.rhog, F.rhog2);
    }
    drop_graph(b);  // the arenas of Mus and ρg may have swapped
    BCK(cudaStreamSynchronize(b->stream));
    return PTS_OK;
}

int pts_batch_solve(pts_batch* b, int64_t iter_limit, int64_t* iters, double* err, int32_t* converged,
                    int32_t* used_graph) {
    if (!b) return PTS_E_INVAL;
    BCK(cudaSetDevice(b->device));
    int64_t iter_last = iter_limit;  // launch-wide ceiling; each instance also stops at its own
    if (iter_last < 0)
        for (const BInst& I : b->hi) iter_last = std::max(iter_last, I.iter_last);
    if (b->ve) iter_last = iter_limit;  // the graph is keyed by the limit as given
    const int n = b->n;
    // the visco-elastic sweep counts iterations globally: iter_limit >= 0 allows iter_limit + 1
    const int64_t iter_cap = iter_limit < 0 ? INT64_MAX : iter_limit + 1;
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t e;
        if ((e = cudaMemsetAsync(b->st.converged, 0, sizeof(int) * n, b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b->st.iters, 0, sizeof(int64_t) * n, b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b->st.err, 0, sizeof(double) * n, b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b->st.nan_flag, 0, sizeof(int), b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(b->st.nactive, b->h_nactive, sizeof(int), cudaMemcpyHostToDevice, b->stream)) !=
            cudaSuccess)
            return e;
        if (b->ve) {
            if ((e = cudaMemsetAsync(b->sv.start, 0, sizeof(int64_t) * n, b->stream)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(b->sv.steps, 0, sizeof(int) * n, b->stream)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(b->sv.step_iters, 0, sizeof(int64_t) * n * kBatchMaxSteps, b->stream)) !=
                cudaSuccess)
                return e;
            if ((e = cudaMemsetAsync(b->sv.assign, 0, sizeof(int) * n, b->stream)) != cudaSuccess) return e;
            return launch_batch_ve(b->tile, b->d_inst, b->ntiles, n, b->F, b->st, b->sv, iter_cap, b->d.eps,
                                   b->stream);
        }
        return launch_batch(b->tile, b->d_inst, b->ntiles, n, b->F, b->st, b->d.nout, iter_last, b->d.eps,
                            b->stream);
    };
    int graph_ok = 0;
    if (!b->graph || b->graph_iter_last != iter_last || b->graph_tile != b->tile) {
        drop_graph(b);
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            cudaError_t e1 = enqueue();
            cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
            if (e1 == cudaSuccess && e2 == cudaSuccess && g && cudaGraphInstantiate(&b->graph, g, 0) == cudaSuccess) {
                b->graph_iter_last = iter_last;
                b->graph_tile = b->tile;
            } else {
                b->graph = nullptr;
            }
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();  // a driver without cooperative launches in graphs: run directly
    }
    if (b->graph) {
        BCK(cudaGraphLaunch(b->graph, b->stream));
        graph_ok = 1;
    } else {
        BCK(enqueue());
    }
    BCK(cudaStreamSynchronize(b->stream));
    std::vector<int> conv(n);
    int nan_flag = 0;
    BCK(cudaMemcpy(conv.data(), b->st.converged, sizeof(int) * n, cudaMemcpyDeviceToHost));
    BCK(cudaMemcpy(&nan_flag, b->st.nan_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (iters) BCK(cudaMemcpy(iters, b->st.iters, sizeof(int64_t) * n, cudaMemcpyDeviceToHost));
    if (err) BCK(cudaMemcpy(err, b->st.err, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (converged)
        for (int q = 0; q < n; ++q) converged[q] = conv[q] == 1;
    if (used_graph) *used_graph = graph_ok;
    if (nan_flag) return bfail(b, PTS_E_NAN, "NaN in the check of at least one instance");
    return PTS_OK;
}

int pts_batch_get_field(pts_batch* b, int32_t q, int32_t id, double* host, int64_t nel) {
    if (!b || !host) return PTS_E_INVAL;
    if (q < 0 || q >= b->n) return bfail(b, PTS_E_INVAL, "instance out of range");
    BCK(cudaSetDevice(b->device));
    const BInst& I = b->hi[q];
    const int nx = I.g.nx, ny = I.g.ny;
    const Fields64& F = b->F;
    const double* base = nullptr;
    int64_t e0 = 0, e1 = 0;
    int s0 = 0, s1 = 0;
    if (b->ve) {  // the visco-elastic sweep keeps the iteration parameters and old stresses per cell
        switch (id) {
            case PTS_F_MUS_TAU: base = F.Must; e0 = nx; e1 = ny; break;
            case PTS_F_GDTAU: base = F.Gdt; e0 = nx; e1 = ny; break;
            case PTS_F_DTAU_RHO: base = F.dtRho; e0 = nx; e1 = ny; break;
            case PTS_F_TXX_O: base = F.txx_o; e0 = nx; e1 = ny; break;
            case PTS_F_TYY_O: base = F.tyy_o; e0 = nx; e1 = ny; break;
            case PTS_F_TXY_O: base = F.txy_o; e0 = nx - 1; e1 = ny - 1; s0 = s1 = 1; break;
            case PTS_F_RHOG: return bfail(b, PTS_E_INVAL, "field not kept by the sweep");
            default: break;
        }
    }
    if (!base) switch (id) {
        case PTS_F_PT: base = F.Pt; e0 = nx; e1 = ny; break;
        case PTS_F_VX: base = F.Vx; e0 = nx + 1; e1 = ny; break;
        case PTS_F_VY: base = F.Vy; e0 = nx; e1 = ny + 1; break;
        case PTS_F_TXX: base = F.txx; e0 = nx; e1 = ny; break;
        case PTS_F_TYY: base = F.tyy; e0 = nx; e1 = ny; break;
        case PTS_F_TXY: base = F.txy; e0 = nx - 1; e1 = ny - 1; s0 = s1 = 1; break;
        case PTS_F_MUS: base = F.Mus; e0 = nx; e1 = ny; break;
        case PTS_F_MUS_TAU:
        case PTS_F_GDTAU:
        case PTS_F_DTAU_RHO: {  // uniform per instance: the reference's arrays hold one value
            if (nel != (int64_t)nx * ny) return bfail(b, PTS_E_INVAL, "wrong element count for this field");
            const double v = id == PTS_F_MUS_TAU ? 1.0 : id == PTS_F_GDTAU ? I.Gd : I.dR;
            for (int64_t e = 0; e < nel; ++e) host[e] = v;
            return PTS_OK;
        }
        case PTS_F_DIVV: base = F.divV; e0 = nx; e1 = ny; break;
        case PTS_F_RX: base = F.Rx; e0 = nx - 1; e1 = ny - 2; s0 = s1 = 1; break;
        case PTS_F_RY: base = F.Ry; e0 = nx - 2; e1 = ny - 1; s0 = s1 = 1; break;
        case PTS_F_RHOG: base = F.rhog; e0 = nx; e1 = ny; break;
        default: return bfail(b, PTS_E_INVAL, "field not kept by the sweep");
    }
    if (nel != e0 * e1) return bfail(b, PTS_E_INVAL, "wrong element count for this field");
    const double* src = base + I.off + (int64_t)s0 + (int64_t)I.g.px * s1;
    BCK(cudaMemcpy2DAsync(host, sizeof(double) * e0, src, sizeof(double) * I.g.px, sizeof(double) * e0, e1,
                          cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return PTS_OK;
}

}  // extern "C"
