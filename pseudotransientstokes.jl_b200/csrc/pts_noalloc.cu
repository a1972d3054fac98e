// pts_noalloc.cu -- the convergence check of a PT iterate (norms of Rx, Ry, Rz and ∇V,
// extrema of Vx and Pt) for callers that cannot allocate device memory.
//
// Some callers own every byte of device memory through their own allocator: a Julia
// program whose arrays live in CUDA.jl's memory pool, a PyTorch program whose memory
// belongs to the caching allocator, or an application that partitions the GPU's memory
// up front and forbids later cudaMalloc calls. Such callers pass their own device arrays
// here and get the check written to a device buffer they also own; this file never
// calls cudaMalloc, cudaFree or any allocating library routine.
//
// The reduction needs room for one partial result per thread block. That room is the
// file-scope array below: its size is fixed (kMaxBlocks blocks of 8 doubles, 256 KB), so
// the grid is limited to kMaxBlocks blocks and larger problems are rejected. Every GPU
// that loads the library keeps this array until the process exits. All calls share it
// and it keeps the contents of the last call; each call overwrites every slot it reads,
// so nothing has to start at zero. Calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race on the array and must be serialised by the
// caller.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "pts_internal.h"

namespace pts {
namespace noalloc {

constexpr int kMaxBlocks = 4096;
constexpr int kSlots = 8;
constexpr int kMaxDevices = 64;

// Block partials: Σ Rx², Σ Ry², Σ Rz², Σ ∇V², min/max Vx, min/max Pt.
static __device__ __align__(256) double scratch[kMaxBlocks * kSlots];

// Host-side address of `scratch` per device: the name itself is only a host stand-in.
static double* g_scratch_addr[kMaxDevices] = {nullptr};
static std::mutex g_mutex;

struct Dense {
    const double* p;
    int64_t e1, e2;  // x and y extents of the field (the reference's)
    int s0, s1, s2;  // unified coordinate of the field's first element
    __device__ __forceinline__ double at(int i, int j, int k) const {
        return __ldg(p + ((int64_t)(i - s0) + e1 * ((int64_t)(j - s1) + e2 * (int64_t)(k - s2))));
    }
};

struct Inputs {
    Dense Pt, Vx, Vy, Vz, txx, tyy, tzz, txy, txz, tyz;
};

struct Params {
    int nx, ny, nz, d3;
    double _dx, _dy, _dz, lx;
    double lenRx, lenRy, lenRz, lenDiv;
};

__device__ __forceinline__ void reduce_store(double a[kSlots], double* out) {
    for (int o = 16; o > 0; o >>= 1) {
        for (int q = 0; q < 4; ++q) a[q] += __shfl_down_sync(0xffffffffu, a[q], o);
        a[4] = fmin(a[4], __shfl_down_sync(0xffffffffu, a[4], o));
        a[5] = fmax(a[5], __shfl_down_sync(0xffffffffu, a[5], o));
        a[6] = fmin(a[6], __shfl_down_sync(0xffffffffu, a[6], o));
        a[7] = fmax(a[7], __shfl_down_sync(0xffffffffu, a[7], o));
    }
    __shared__ double sm[8][kSlots];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = tid & 31, warp = tid >> 5;
    if (lane == 0)
        for (int q = 0; q < kSlots; ++q) sm[warp][q] = a[q];
    __syncthreads();
    if (tid == 0) {
        double r[kSlots];
        for (int q = 0; q < kSlots; ++q) r[q] = sm[0][q];
        for (int w = 1; w < 8; ++w) {
            for (int q = 0; q < 4; ++q) r[q] += sm[w][q];
            r[4] = fmin(r[4], sm[w][4]); r[5] = fmax(r[5], sm[w][5]);
            r[6] = fmin(r[6], sm[w][6]); r[7] = fmax(r[7], sm[w][7]);
        }
        const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        for (int q = 0; q < kSlots; ++q) out[(int64_t)b * kSlots + q] = r[q];
    }
}

// compute_Res! of the explicit-index scripts (Stokes3D_ve_perf.jl:90-96,
// Stokes2D_ve_perf.jl:61-66) on dense reference-layout arrays, and the block partials.
__global__ void __launch_bounds__(256) k_check_dense(Inputs in, Params pr, double* partials) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int nx = pr.nx, ny = pr.ny, nz = pr.nz;
    double a[kSlots] = {0.0, 0.0, 0.0, 0.0, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    if (i <= nx && j < ny) {
        for (int k = blockIdx.z; k < nz; k += gridDim.z) {
            const double vx = in.Vx.at(i, j, k);
            a[4] = fmin(a[4], vx);
            a[5] = fmax(a[5], vx);
            if (i < nx) {
                const double p = in.Pt.at(i, j, k);
                a[6] = fmin(a[6], p);
                a[7] = fmax(a[7], p);
                double dv = pr._dx * (in.Vx.at(i + 1, j, k) - vx) + pr._dy * (in.Vy.at(i, j + 1, k) - in.Vy.at(i, j, k));
                if (pr.d3) dv = dv + pr._dz * (in.Vz.at(i, j, k + 1) - in.Vz.at(i, j, k));
                a[3] += dv * dv;
            }
            if (pr.d3) {
                if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
                    const double R = ((pr._dx * (in.txx.at(i, j, k) - in.txx.at(i - 1, j, k)) +
                                       pr._dy * (in.txy.at(i, j + 1, k) - in.txy.at(i, j, k))) +
                                      pr._dz * (in.txz.at(i, j, k + 1) - in.txz.at(i, j, k))) -
                                     pr._dx * (in.Pt.at(i, j, k) - in.Pt.at(i - 1, j, k));
                    a[0] += R * R;
                }
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 2) {
                    const double R = ((pr._dy * (in.tyy.at(i, j, k) - in.tyy.at(i, j - 1, k)) +
                                       pr._dx * (in.txy.at(i + 1, j, k) - in.txy.at(i, j, k))) +
                                      pr._dz * (in.tyz.at(i, j, k + 1) - in.tyz.at(i, j, k))) -
                                     pr._dy * (in.Pt.at(i, j, k) - in.Pt.at(i, j - 1, k));
                    a[1] += R * R;
                }
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 1) {
                    const double R = ((pr._dz * (in.tzz.at(i, j, k) - in.tzz.at(i, j, k - 1)) +
                                       pr._dx * (in.txz.at(i + 1, j, k) - in.txz.at(i, j, k))) +
                                      pr._dy * (in.tyz.at(i, j + 1, k) - in.tyz.at(i, j, k))) -
                                     pr._dz * (in.Pt.at(i, j, k) - in.Pt.at(i, j, k - 1));
                    a[2] += R * R;
                }
            } else {
                if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 2) {
                    const double R = (pr._dx * (in.txx.at(i, j, k) - in.txx.at(i - 1, j, k)) +
                                      pr._dy * (in.txy.at(i, j + 1, k) - in.txy.at(i, j, k))) -
                                     pr._dx * (in.Pt.at(i, j, k) - in.Pt.at(i - 1, j, k));
                    a[0] += R * R;
                }
                if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 1) {
                    const double R = (pr._dy * (in.tyy.at(i, j, k) - in.tyy.at(i, j - 1, k)) +
                                      pr._dx * (in.txy.at(i + 1, j, k) - in.txy.at(i, j, k))) -
                                     pr._dy * (in.Pt.at(i, j, k) - in.Pt.at(i, j - 1, k));
                    a[1] += R * R;
                }
            }
        }
    }
    reduce_store(a, partials);
}

// The norms of the check (Stokes3D_ve_perf.jl:213-218) into the caller's pts_check.
__global__ void k_finalize_dense(const double* partials, int nblocks, Params pr, pts_check* out) {
    __shared__ double sm[256][kSlots];
    const int t = threadIdx.x;
    double r[kSlots] = {0.0, 0.0, 0.0, 0.0, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    for (int b = t; b < nblocks; b += blockDim.x) {
        const double* p = partials + (int64_t)b * kSlots;
        for (int q = 0; q < 4; ++q) r[q] += p[q];
        r[4] = fmin(r[4], p[4]); r[5] = fmax(r[5], p[5]);
        r[6] = fmin(r[6], p[6]); r[7] = fmax(r[7], p[7]);
    }
    for (int q = 0; q < kSlots; ++q) sm[t][q] = r[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) {
            for (int q = 0; q < 4; ++q) sm[t][q] += sm[t + s][q];
            sm[t][4] = fmin(sm[t][4], sm[t + s][4]); sm[t][5] = fmax(sm[t][5], sm[t + s][5]);
            sm[t][6] = fmin(sm[t][6], sm[t + s][6]); sm[t][7] = fmax(sm[t][7], sm[t + s][7]);
        }
        __syncthreads();
    }
    if (t == 0) {
        const double dP = sm[0][7] - sm[0][6], dV = sm[0][5] - sm[0][4];
        pts_check c;
        c.norm_Rx = sqrt(sm[0][0]) / dP * pr.lx / sqrt(pr.lenRx);
        c.norm_Ry = sqrt(sm[0][1]) / dP * pr.lx / sqrt(pr.lenRy);
        c.norm_Rz = pr.d3 ? sqrt(sm[0][2]) / dP * pr.lx / sqrt(pr.lenRz) : 0.0;
        c.norm_divV = sqrt(sm[0][3]) / dV * pr.lx / sqrt(pr.lenDiv);
        c.Vmin = sm[0][4]; c.Vmax = sm[0][5]; c.Pmin = sm[0][6]; c.Pmax = sm[0][7];
        const bool bad = isnan(c.norm_Rx) || isnan(c.norm_Ry) || isnan(c.norm_Rz) || isnan(c.norm_divV);
        c.err = bad ? NAN : fmax(fmax(c.norm_Rx, c.norm_Ry), fmax(c.norm_Rz, c.norm_divV));
        *out = c;
    }
}

// Address of `scratch` on the current device, looked up once per device.
cudaError_t scratch_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace noalloc
}  // namespace pts

using namespace pts;
using namespace pts::noalloc;

extern "C" {

int pts_check_noalloc(const pts_desc* d, const double* const fields[10], pts_check* out, void* stream) {
    char msg[256];
    auto fail = [](int code, const char* m) {
        set_global_error(m);
        return code;
    };
    if (!d || !fields || !out) return fail(PTS_E_INVAL, "null argument");
    const bool d3 = d->variant == PTS_3D_VE_PERF || d->variant == PTS_3D_V;
    if (!d3 && d->variant != PTS_2D_VE_PERF)
        return fail(PTS_E_INVAL, "pts_check_noalloc supports the explicit-index variants (2D VE perf, 3D VE perf, 3D viscous)");
    const int nx = d->nx, ny = d->ny, nz = d3 ? d->nz : 1;
    if (nx < 3 || ny < 3 || (d3 && nz < 3)) return fail(PTS_E_INVAL, "each of nx, ny(, nz) must be >= 3");
    if (!(d->lx > 0) || !(d->ly > 0) || (d3 && !(d->lz > 0)))
        return fail(PTS_E_INVAL, "domain extents must be > 0");
    const int gx = (nx + 1 + 31) / 32, gy = (ny + 7) / 8;
    if ((int64_t)gx * gy > kMaxBlocks) {
        snprintf(msg, sizeof(msg),
                 "grid too large for the no-allocation check: ceil((nx+1)/32)*ceil(ny/8) = %lld tiles, at most %d",
                 (long long)gx * gy, kMaxBlocks);
        return fail(PTS_E_INVAL, msg);
    }
    const int need2d[] = {PTS_F_PT, PTS_F_VX, PTS_F_VY, PTS_F_TXX, PTS_F_TYY, PTS_F_TXY};
    for (int q = 0; q < (d3 ? 10 : 6); ++q) {
        const int id = d3 ? q : need2d[q];
        if (!fields[id]) return fail(PTS_E_INVAL, "null field pointer");
    }
    double* part = nullptr;
    cudaError_t e = scratch_address(&part);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the check scratch: %s", cudaGetErrorString(e));
        return fail(PTS_E_CUDA, msg);
    }
    // dense reference layouts: extents and the unified coordinate of element [1,1,1]
    Inputs in;
    auto dense = [&](int id, int64_t e1, int64_t e2, int s0, int s1, int s2) {
        return Dense{fields[id], e1, e2, s0, s1, s2};
    };
    in.Pt = dense(PTS_F_PT, nx, ny, 0, 0, 0);
    in.Vx = dense(PTS_F_VX, nx + 1, ny, 0, 0, 0);
    in.Vy = dense(PTS_F_VY, nx, ny + 1, 0, 0, 0);
    if (d3) {
        in.Vz = dense(PTS_F_VZ, nx, ny, 0, 0, 0);
        in.txx = dense(PTS_F_TXX, nx, ny - 2, 0, 1, 1);
        in.tyy = dense(PTS_F_TYY, nx - 2, ny, 1, 0, 1);
        in.tzz = dense(PTS_F_TZZ, nx - 2, ny - 2, 1, 1, 0);
        in.txy = dense(PTS_F_TXY, nx - 1, ny - 1, 1, 1, 1);
        in.txz = dense(PTS_F_TXZ, nx - 1, ny - 2, 1, 1, 1);
        in.tyz = dense(PTS_F_TYZ, nx - 2, ny - 1, 1, 1, 1);
    } else {
        in.Vz = in.Vy;
        in.txx = dense(PTS_F_TXX, nx, ny, 0, 0, 0);
        in.tyy = dense(PTS_F_TYY, nx, ny, 0, 0, 0);
        in.txy = dense(PTS_F_TXY, nx - 1, ny - 1, 1, 1, 0);
        in.tzz = in.txz = in.tyz = in.txx;
    }
    Params pr;
    pr.nx = nx; pr.ny = ny; pr.nz = nz; pr.d3 = d3 ? 1 : 0;
    const double dx = d->lx / nx, dy = d->ly / ny, dz = d3 ? d->lz / nz : 1.0;
    pr._dx = 1.0 / dx; pr._dy = 1.0 / dy; pr._dz = 1.0 / dz;
    pr.lx = d->lx;
    pr.lenRx = d3 ? (double)(nx - 1) * (ny - 2) * (nz - 2) : (double)(nx - 1) * (ny - 2);
    pr.lenRy = d3 ? (double)(nx - 2) * (ny - 1) * (nz - 2) : (double)(nx - 2) * (ny - 1);
    pr.lenRz = d3 ? (double)(nx - 2) * (ny - 2) * (nz - 1) : 1.0;
    pr.lenDiv = (double)nx * ny * nz;
    const int gz = d3 ? std::max(1, std::min(nz, kMaxBlocks / (gx * gy))) : 1;
    const int nblocks = gx * gy * gz;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_check_dense<<<dim3(gx, gy, gz), dim3(32, 8, 1), 0, s>>>(in, pr, part);
    k_finalize_dense<<<1, 256, 0, s>>>(part, nblocks, pr, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "launch: %s", cudaGetErrorString(e));
        return fail(PTS_E_CUDA, msg);
    }
    return PTS_OK;
}

}  // extern "C"
