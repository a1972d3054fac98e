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
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pts_internal.h"

using namespace pts;

struct pts_batch {
    pts_batch_desc d{};
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
    double** p[] = {&f.Pt, &f.Vx, &f.Vy, &f.txx, &f.tyy, &f.txy, &f.Mus, &f.divV,
                    &f.Rx, &f.Ry, &f.Mus2, &f.rhog, &f.rhog2};
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

int pts_batch_setup(pts_batch* b) {
    if (!b) return PTS_E_INVAL;
    BCK(cudaSetDevice(b->device));
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
    const int n = b->n;
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t e;
        if ((e = cudaMemsetAsync(b->st.converged, 0, sizeof(int) * n, b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b->st.iters, 0, sizeof(int64_t) * n, b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b->st.err, 0, sizeof(double) * n, b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b->st.nan_flag, 0, sizeof(int), b->stream)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(b->st.nactive, b->h_nactive, sizeof(int), cudaMemcpyHostToDevice, b->stream)) !=
            cudaSuccess)
            return e;
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
    switch (id) {
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
