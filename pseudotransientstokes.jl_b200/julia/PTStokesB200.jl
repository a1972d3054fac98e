# PTStokesB200.jl -- Julia `ccall` binding of libptstokes.so (the B200 PT Stokes solver).
#
# Keeps the kernel-role names of the reference scripts (compute_P!, compute_τ!,
# compute_dV!, compute_V!, compute_Pt_τ!, compute_Res!, assign_τ!, bc!) so a script can
# replace its `@parallel` calls with these. Fields live on the device inside the context;
# `set_field!`/`get_field` move Julia Arrays (Float64, the reference's extents), and
# `set_field_device!` takes a CuArray's pointer.
#
# This file is written against include/ptstokes.h; no Julia runtime was available where
# it was written, so it has not been executed.
module PTStokesB200

const libpts = get(ENV, "PTSTOKES_LIB", joinpath(@__DIR__, "..", "lib", "libptstokes.so"))

const PTS_OK = Cint(0)
@enum Variant::Int32 V2D = 0 VE2D = 1 VE2D_PERF = 2 VE3D = 3 VE3D_PERF = 4 V3D = 5 V2D_DAMP = 6 VE2D_DAMP = 7 V3D_DAMP = 8
const FIELDS = (:Pt, :Vx, :Vy, :Vz, :τxx, :τyy, :τzz, :τxy, :τxz, :τyz,
                :τxx_o, :τyy_o, :τzz_o, :τxy_o, :τxz_o, :τyz_o,
                :Mus, :Musτ, :Gdτ, :dτ_Rho, :∇V, :Rx, :Ry, :Rz, :dVx, :dVy, :dVz,
                :ρg, :Fx, :Fy, :Fz, :grad, :dτVx, :dτVy, :dτVz, :dτPt)
field_id(s::Symbol) = Int32(findfirst(==(s), FIELDS) - 1)

# pts_desc (include/ptstokes.h)
struct Desc
    variant::Int32; precision::Int32
    nx::Int32; ny::Int32; nz::Int32; nout::Int32
    lx::Float64; ly::Float64; lz::Float64
    G::Float64; dt::Float64
    r::Float64; Re::Float64; CFL::Float64
    max_l::Float64; eps::Float64; iter_max::Float64
    mixed_inner::Int32; single_pass::Int32; adjoint::Int32
    stencil::Int32; stencil_tile::Int32; stencil_kz::Int32; stencil_vtile::Int32
    mixed_sweep::Int32
end

struct Check
    err::Float64; norm_Rx::Float64; norm_Ry::Float64; norm_Rz::Float64; norm_∇V::Float64
    Vmin::Float64; Vmax::Float64; Pmin::Float64; Pmax::Float64
end

struct SolveInfo
    iters::Int64; converged::Int32; nchecks::Int32; last::Check
end

mutable struct Ctx
    ptr::Ptr{Cvoid}
end

function check(ctx, rc)
    if rc != PTS_OK
        msg = unsafe_string(ccall((:pts_last_error, libpts), Cstring, (Ptr{Cvoid},), ctx === nothing ? C_NULL : ctx.ptr))
        error("ptstokes error $rc: $msg")
    end
    return nothing
end

"""
    Ctx(variant, nx, ny, nz; lx=10, ly=10, lz=10, G=1, dt=1, r=1, Re, CFL, nout, ε=1e-8, iterMax)

A device context for one problem (the scripts' `Stokes2D_()`/`Stokes3D_()` state).
"""
function Ctx(variant::Variant, nx, ny, nz=1; lx=10.0, ly=10.0, lz=10.0, G=1.0, dt=1.0, r=1.0, Re, CFL,
             nout=200, ε=1e-8, iterMax=2e5, max_l=0.0, precision=0, single_pass=0, adjoint=0, stencil=0,
             stencil_tile=0, stencil_kz=0, stencil_vtile=0, mixed_sweep=0)
    d = Desc(Int32(variant), Int32(precision), nx, ny, nz, nout, lx, ly, lz, G, dt, r, Re, CFL, max_l, ε, iterMax,
             0, single_pass, adjoint, stencil, stencil_tile, stencil_kz, stencil_vtile, mixed_sweep)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(nothing, ccall((:pts_create, libpts), Cint, (Ref{Desc}, Ref{Ptr{Cvoid}}), d, out))
    ctx = Ctx(out[])
    finalizer(c -> ccall((:pts_destroy, libpts), Cint, (Ptr{Cvoid},), c.ptr), ctx)
    return ctx
end

function field_shape(ctx::Ctx, f::Symbol)
    s = zeros(Int64, 3)
    check(ctx, ccall((:pts_field_shape, libpts), Cint, (Ptr{Cvoid}, Int32, Ptr{Int64}), ctx.ptr, field_id(f), s))
    return Tuple(s)
end

set_field!(ctx::Ctx, f::Symbol, A::Array{Float64}) =
    check(ctx, ccall((:pts_set_field, libpts), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Int64), ctx.ptr, field_id(f), A, length(A)))

function get_field(ctx::Ctx, f::Symbol)
    s = field_shape(ctx, f)
    A = zeros(Float64, s...)
    check(ctx, ccall((:pts_get_field, libpts), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Int64), ctx.ptr, field_id(f), A, length(A)))
    return A
end

# A CuArray's device pointer (e.g. `pointer(A)` converted with `UInt(pointer(A))`).
set_field_device!(ctx::Ctx, f::Symbol, devptr::UInt, n::Integer) =
    check(ctx, ccall((:pts_set_field_device, libpts), Cint, (Ptr{Cvoid}, Int32, UInt, Int64), ctx.ptr, field_id(f), devptr, n))

for (jl, c) in ((:init_inclusion!, :pts_init_inclusion),)
    @eval $jl(ctx::Ctx; μs0=1.0, μsi=1e-3, radius2=1.0, εbg=1.0) =
        check(ctx, ccall(($(QuoteNode(c)), libpts), Cint, (Ptr{Cvoid}, Float64, Float64, Float64, Float64), ctx.ptr, μs0, μsi, radius2, εbg))
end
# create_inclusions! (Stokes2D_param.jl:83-99) for a list of circles/spheres (pts_inclusion)
struct Inclusion
    x::Float64; y::Float64; z::Float64   # centre relative to the domain centre (the script's Xi, Yi)
    r2::Float64                          # squared radius
    μs::Float64                          # viscosity inside
end
init_inclusions!(ctx::Ctx, list::Vector{Inclusion}; μs0=1.0, εbg=1.0) =
    check(ctx, ccall((:pts_init_inclusions, libpts), Cint, (Ptr{Cvoid}, Ptr{Inclusion}, Int32, Float64, Float64),
                     ctx.ptr, list, length(list), μs0, εbg))
# numerics of the damped variants (previous_damp/Stokes2D_ve0.jl:95-98; the 3D script's are
# Vdmp=4, β_n=3, Vsc=1, Ptsc=5, Stokes3D0_multixpu.jl:105-108), before compute_iter_params!
set_damping!(ctx::Ctx; Vdmp=4.0, β_n=2.0, Vsc=1.0, Ptsc=3.0) =
    check(ctx, ccall((:pts_set_damping, libpts), Cint, (Ptr{Cvoid}, Float64, Float64, Float64, Float64),
                     ctx.ptr, Vdmp, β_n, Vsc, Ptsc))
smooth!(ctx::Ctx, nsweeps=10, fact=1.0) = check(ctx, ccall((:pts_smooth, libpts), Cint, (Ptr{Cvoid}, Int32, Float64), ctx.ptr, nsweeps, fact))

# Roles (each replaces the `@parallel` call of the same name in the scripts)
for (jl, c) in ((:compute_maxloc!, :pts_compute_maxloc), (:compute_iter_params!, :pts_compute_iter_params),
                (:assign_τ!, :pts_assign_tau), (:compute_P!, :pts_compute_P), (:compute_τ!, :pts_compute_tau),
                (:compute_dV!, :pts_compute_dV), (:compute_V!, :pts_compute_V), (:bc!, :pts_apply_bc),
                (:compute_Pt_τ!, :pts_compute_Pt_tau), (:compute_V_bc!, :pts_compute_V_bc))
    @eval $jl(ctx::Ctx) = check(ctx, ccall(($(QuoteNode(c)), libpts), Cint, (Ptr{Cvoid},), ctx.ptr))
end

function compute_Res!(ctx::Ctx)
    r = Ref{Check}()
    check(ctx, ccall((:pts_compute_res, libpts), Cint, (Ptr{Cvoid}, Ref{Check}), ctx.ptr, r))
    return r[]
end

iterate!(ctx::Ctx, n) = check(ctx, ccall((:pts_iterate, libpts), Cint, (Ptr{Cvoid}, Int64), ctx.ptr, n))

"The PT loop of one physical step (`while err > ε && iter <= iterMax`)."
function solve!(ctx::Ctx)
    r = Ref{SolveInfo}()
    check(ctx, ccall((:pts_solve, libpts), Cint, (Ptr{Cvoid}, Ref{SolveInfo}), ctx.ptr, r))
    return r[]
end

"The time loop `for it = 1:nt` (assign_τ! + PT loop per step); returns per-step iterations."
function run!(ctx::Ctx, nt)
    per = zeros(Int64, nt)
    r = Ref{SolveInfo}()
    check(ctx, ccall((:pts_run, libpts), Cint, (Ptr{Cvoid}, Int32, Ptr{Int64}, Ref{SolveInfo}), ctx.ptr, nt, per, r))
    return per, r[]
end

"""
The error measure the 2D scripts keep commented out beside their check (Stokes2D_ve0.jl:166):
max of norm(R)/length(R) over Rx, Ry and ∇V, recovered from a `compute_Res!` result `c` of an
nx × ny context whose norms carry the default scale lx.
"""
function length_error(c::Check, nx, ny, lx)
    lens = ((nx - 1) * (ny - 2), (nx - 2) * (ny - 1), nx * ny)
    dP, dV = c.Pmax - c.Pmin, c.Vmax - c.Vmin
    n = (c.norm_Rx * dP * sqrt(lens[1]) / lx / lens[1],
         c.norm_Ry * dP * sqrt(lens[2]) / lx / lens[2],
         c.norm_∇V * dV * sqrt(lens[3]) / lx / lens[3])
    return any(isnan, n) ? NaN : maximum(n)
end

"""
The damped 2D scripts' time loop checked with `length_error`, the measure the reference's
output/out_Stokes2D_ve0.txt totals were taken with: per step assign_τ! (visco-elastic only),
then `while err > ε && iter <= iterMax` in blocks that end on the multiples of nout.
Returns the per-step iterations.
"""
function run_length_error!(ctx::Ctx, nx, ny; nt=5, nout=200, ε=1e-8, iterMax=2e5, lx=10.0, elastic=true)
    nout >= 1 || throw(ArgumentError("nout must be >= 1"))
    imax = floor(Int, iterMax)
    per = Int[]
    for _ in 1:nt
        err, iter = 2ε, 0
        elastic && assign_τ!(ctx)
        while err > ε && iter <= imax
            k = min(nout - iter % nout, imax - iter + 1)
            iterate!(ctx, k)
            iter += k
            if iter % nout == 0
                err = length_error(compute_Res!(ctx), nx, ny, lx)
                isnan(err) && error("NaN")
            end
        end
        push!(per, iter)
    end
    return per
end

# ---- batched 2D sweeps (pts_batch_*): the runme_Stokes2D_*.jl loops in one launch ----

struct BatchInstance
    nx::Int32; ny::Int32
    lx::Float64; ly::Float64; μsi::Float64; radius2::Float64; ρgi::Float64; εbg::Float64
end

struct BatchDesc
    nout::Int32; tile::Int32
    ε::Float64; iterMax::Float64; r::Float64; Re::Float64; CFL::Float64
    reserved::NTuple{4,Int32}
end

mutable struct Batch
    ptr::Ptr{Cvoid}
    n::Int
end

"""
    Batch(instances; nout=200, ε=1e-8, iterMax=0.0, tile=1, r=1.0, Re=5π, CFL=0.9/sqrt(2))

A sweep of 2D viscous instances (`Stokes2D_param.jl` numerics); `iterMax <= 0` gives each
instance iterMax = 100max(nx,ny).
"""
function Batch(inst::Vector{BatchInstance}; nout=200, ε=1e-8, iterMax=0.0, tile=1, r=1.0, Re=5π, CFL=0.9/sqrt(2))
    d = BatchDesc(nout, tile, ε, iterMax, r, Re, CFL, ntuple(_ -> Int32(0), 4))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:pts_batch_create, libpts), Cint, (Ref{BatchDesc}, Ptr{BatchInstance}, Int32, Ref{Ptr{Cvoid}}),
               d, inst, length(inst), out)
    rc == 0 || error("pts_batch_create: ", unsafe_string(ccall((:pts_last_error, libpts), Cstring, (Ptr{Cvoid},), C_NULL)))
    b = Batch(out[], length(inst))
    finalizer(x -> ccall((:pts_batch_destroy, libpts), Cint, (Ptr{Cvoid},), x.ptr), b)
    return b
end

function batch_check(b::Batch, rc)
    rc == 0 || error("ptstokes batch error $rc: ", unsafe_string(ccall((:pts_batch_last_error, libpts), Cstring, (Ptr{Cvoid},), b.ptr)))
    return nothing
end

setup!(b::Batch) = batch_check(b, ccall((:pts_batch_setup, libpts), Cint, (Ptr{Cvoid},), b.ptr))

"Runs the sweep; returns per-instance iterations, last err and convergence flags."
function solve!(b::Batch; iter_limit=-1)
    iters = zeros(Int64, b.n); err = zeros(Float64, b.n); conv = zeros(Int32, b.n); graph = Ref{Int32}(0)
    batch_check(b, ccall((:pts_batch_solve, libpts), Cint,
                         (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Float64}, Ptr{Int32}, Ref{Int32}),
                         b.ptr, iter_limit, iters, err, conv, graph))
    return iters, err, conv .== 1
end

# ---- the visco-elastic aspect-ratio sweep in one launch (pts_batch_create_ve) ----
# runme_Stokes2D_aspect_ratio.jl starts one Julia process of Stokes2D_ve_param.jl per
# (FACT, NSUB, RESOL); here every instance runs its nt Maxwell steps in one persistent launch.

struct BatchVEInstance
    ny::Int32; nsub::Int32; nt::Int32; reserved::Int32
    fact::Float64; ly::Float64; μsi::Float64
end
BatchVEInstance(ny, nsub, fact; nt=5, ly=10.0, μsi=1e-3) = BatchVEInstance(ny, nsub, nt, 0, fact, ly, μsi)

"""
    BatchVE(instances; ε=1e-6, tile=1, r=1.0, Re=5π, CFL=0.87/sqrt(2), nout=0, iterMax=0.0)

The aspect-ratio sweep; `nout <= 0` and `iterMax <= 0` give each instance the script's
nout = nx and iterMax = 100nx. `setup!` and `solve!` as for `Batch` (solve! returns each
instance's ittot); `steps(b, q)` the iterations of each Maxwell step of instance q.
"""
function BatchVE(inst::Vector{BatchVEInstance}; ε=1e-6, tile=1, r=1.0, Re=5π, CFL=0.87/sqrt(2), nout=0, iterMax=0.0)
    d = BatchDesc(nout, tile, ε, iterMax, r, Re, CFL, ntuple(_ -> Int32(0), 4))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:pts_batch_create_ve, libpts), Cint, (Ref{BatchDesc}, Ptr{BatchVEInstance}, Int32, Ref{Ptr{Cvoid}}),
               d, inst, length(inst), out)
    rc == 0 || error("pts_batch_create_ve: ", unsafe_string(ccall((:pts_last_error, libpts), Cstring, (Ptr{Cvoid},), C_NULL)))
    b = Batch(out[], length(inst))
    finalizer(x -> ccall((:pts_batch_destroy, libpts), Cint, (Ptr{Cvoid},), x.ptr), b)
    return b
end

"Iterations of each finished Maxwell step of instance q (1-based)."
function steps(b::Batch, q::Integer)
    buf = zeros(Int64, 64); k = Ref{Int32}(0)
    batch_check(b, ccall((:pts_batch_steps, libpts), Cint, (Ptr{Cvoid}, Int32, Ptr{Int64}, Int32, Ref{Int32}),
                         b.ptr, q - 1, buf, 64, k))
    return buf[1:min(k[], 64)]
end

# ---- adjoint of the 3D viscous solve (pts_apply_operator, pts_gradient_logmu) ----

"One application of the operator (or of its transpose on an adjoint context)."
function apply_operator!(ctx::Ctx)
    r = Ref{Check}()
    check(ctx, ccall((:pts_apply_operator, libpts), Cint, (Ptr{Cvoid}, Ref{Check}), ctx.ptr, r))
    return r[]
end

"∂J/∂log μ into the forward context's :grad field from the adjoint context's solution."
gradient_logmu!(fwd::Ctx, adj::Ctx) =
    check(fwd, ccall((:pts_gradient_logmu, libpts), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), fwd.ptr, adj.ptr))

"""
    top_vz(logμ, fwd, adj, Vwall) -> Vz on the top interior face plane

Forward solve of the 3D viscous problem for the cell viscosity exp.(logμ) (the walls and
ICs `Vwall = (Vx, Vy, Vz)` are set first). `fwd` is a PTS_3D_V context, `adj` one created
with `adjoint=1` on the same grid.
"""
function top_vz(logμ::Array{Float64,3}, fwd::Ctx, adj::Ctx, Vwall)
    init_inclusion!(fwd; μs0=1.0, μsi=1.0, radius2=0.0, εbg=0.0)    # every field zero
    set_field!(fwd, :Vx, Vwall[1]); set_field!(fwd, :Vy, Vwall[2]); set_field!(fwd, :Vz, Vwall[3])
    set_field!(fwd, :Mus, exp.(logμ)); compute_maxloc!(fwd); compute_iter_params!(fwd)
    solve!(fwd)
    Vz = get_field(fwd, :Vz)
    return Vz[2:end-1, 2:end-1, end-1]
end

# ---- z-slab decomposition (the ImplicitGlobalGrid part of Stokes3D_ve_multixpu.jl) ----
# The caller owns the transport (MPI from Julia): these move planes and reduce nothing.

"Make `ctx` the z-slab [zoff, zoff+nz) of a global grid of nz_g cells (before the set-up)."
set_decomposition!(ctx::Ctx, zoff::Integer, nz_g::Integer) =
    check(ctx, ccall((:pts_set_decomposition, libpts), Cint, (Ptr{Cvoid}, Int32, Int32), ctx.ptr, zoff, nz_g))

"z-plane k (0-based) of a field to/from a CuArray's device memory (`pointer(A)` as UInt)."
get_plane_device!(ctx::Ctx, f::Symbol, k::Integer, devptr::UInt, n::Integer) =
    check(ctx, ccall((:pts_get_plane_device, libpts), Cint, (Ptr{Cvoid}, Int32, Int32, UInt, Int64),
                     ctx.ptr, field_id(f), k, devptr, n))
set_plane_device!(ctx::Ctx, f::Symbol, k::Integer, devptr::UInt, n::Integer) =
    check(ctx, ccall((:pts_set_plane_device, libpts), Cint, (Ptr{Cvoid}, Int32, Int32, UInt, Int64),
                     ctx.ptr, field_id(f), k, devptr, n))

"""
    compute_V_bc_planes!(ctx, k0, k1, stream=C_NULL)

compute_V! + bc on the face planes [k0, k1) only, on `stream` (a CuStream's handle; C_NULL: the
context's stream). `@hide_communication b_width` is: the end regions [0, b) and [nz+1-b, nz+1)
on the context's stream, the inner region on another stream, then update_halo! of the
end planes while the inner region runs.
"""
compute_V_bc_planes!(ctx::Ctx, k0::Integer, k1::Integer, stream::Ptr{Cvoid}=C_NULL) =
    check(ctx, ccall((:pts_compute_V_bc_planes, libpts), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Cvoid}),
                     ctx.ptr, k0, k1, stream))

"{Σ Rx², Σ Ry², Σ Rz², Σ ∇V², min Vx, max Vx, min Pt, max Pt} of this slab, for MPI.Allreduce."
function check_partials(ctx::Ctx)
    out = zeros(Float64, 8)
    check(ctx, ccall((:pts_check_partials, libpts), Cint, (Ptr{Cvoid}, Ptr{Float64}), ctx.ptr, out))
    return out
end

"MIXED contexts: 0 = two kernels per FP32 sweep (default), 1 + tile = the one-pass sweep."
set_mixed_sweep!(ctx::Ctx, mixed_sweep::Integer) =
    check(ctx, ccall((:pts_set_mixed_sweep, libpts), Cint, (Ptr{Cvoid}, Int32), ctx.ptr, mixed_sweep))

"A CUDA event after each kernel of every block of PT iterations (inside the check-block graphs)."
set_kernel_timing!(ctx::Ctx, on::Bool) =
    check(ctx, ccall((:pts_set_kernel_timing, libpts), Cint, (Ptr{Cvoid}, Int32), ctx.ptr, on ? 1 : 0))

"Per-kernel times (ms) of the last block, in launch order."
function kernel_times(ctx::Ctx; cap::Integer=1 << 16)
    ms = zeros(Float32, cap)
    n = Ref{Int64}(0)
    check(ctx, ccall((:pts_kernel_times, libpts), Cint, (Ptr{Cvoid}, Ptr{Float32}, Int64, Ref{Int64}),
                     ctx.ptr, ms, cap, n))
    return ms[1:min(n[], cap)]
end

"Lengths scaling norm_Rx, norm_Ry, norm_Rz, norm_∇V (Stokes2D_ve_param.jl:175-177: lx, ly, -, ly)."
set_norm_scales!(ctx::Ctx, sRx, sRy, sRz, sdiv) =
    check(ctx, ccall((:pts_set_norm_scales, libpts), Cint, (Ptr{Cvoid}, Float64, Float64, Float64, Float64),
                     ctx.ptr, sRx, sRy, sRz, sdiv))

# Reverse rules for top_vz (and its visco-elastic time-loop twin top_vz_ve) are the
# ChainRulesCore.rrule methods of PTStokesB200ChainRules.jl, next to this file.

end # module
