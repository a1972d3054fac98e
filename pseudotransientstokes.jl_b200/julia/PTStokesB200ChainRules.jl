# PTStokesB200ChainRules.jl -- ChainRulesCore reverse rules for the adjoint entry points of
# the PTStokesB200 shim (libptstokes.so: pts_solve on a context created with adjoint = 1,
# pts_gradient_logmu, pts_gradient_logmu_add).
#
# The reference has no adjoint. The forward maps differentiated here are
#   top_vz(logμ, fwd, adj, Vwall)          one 3D viscous PT solve (PTS_3D_V)
#   top_vz_ve(logμ, fwd, adj, Vwall, nt)   nt Maxwell visco-elastic steps (PTS_3D_VE_PERF),
#                                          each PT loop converged, per-step stress checkpoints
# and their value is Vz on the top interior face plane. A pullback runs the transposed PT
# solve on the adjoint context with the incoming cotangent as momentum source on that plane
# (field :Fz, the extent of Rz), then the pointwise ∂/∂log μ kernel on the device. The
# Python twin is ptstokes.adjoint (TopVz, a torch.autograd.Function).
#
# Use:  include("PTStokesB200.jl"); include("PTStokesB200ChainRules.jl")
#       using .PTStokesB200, .PTStokesB200ChainRules, Zygote
#       g = Zygote.gradient(l -> 0.5sum(abs2, top_vz(l, fwd, adj, Vwall) .- vobs), logμ)[1]
module PTStokesB200ChainRules

using ChainRulesCore
using ..PTStokesB200: PTStokesB200, Ctx, top_vz, init_inclusion!, set_field!, get_field, field_shape,
                      compute_maxloc!, compute_iter_params!, assign_τ!, solve!, gradient_logmu!, check, libpts

export top_vz_ve

const TAU = (:τxx, :τyy, :τzz, :τxy, :τxz, :τyz)

"∂J/∂log μ of one visco-elastic step added to the forward context's :grad (pts_gradient_logmu_add)."
gradient_logmu_add!(fwd::Ctx, adj::Ctx) =
    check(fwd, ccall((:pts_gradient_logmu_add, libpts), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), fwd.ptr, adj.ptr))

"Zero state, viscosity exp.(logμ), local-max viscosity and iteration parameters (adjoint: no walls)."
function prepare_adjoint!(adj::Ctx, logμ)
    init_inclusion!(adj; μs0=1.0, μsi=1.0, radius2=0.0, εbg=0.0)   # every field zero
    set_field!(adj, :Mus, exp.(logμ))
    compute_maxloc!(adj)
    compute_iter_params!(adj)
    return adj
end

"The momentum source of the transposed solve: ∂J/∂Vz on the top interior face plane."
function top_source(adj::Ctx, v̄)
    Fz = zeros(field_shape(adj, :Fz)...)
    Fz[:, :, end] .= v̄
    return Fz
end

function ChainRulesCore.rrule(::typeof(top_vz), logμ::Array{Float64,3}, fwd::Ctx, adj::Ctx, Vwall)
    v = top_vz(logμ, fwd, adj, Vwall)
    function top_vz_pullback(v̄)
        prepare_adjoint!(adj, logμ)
        set_field!(adj, :Fz, top_source(adj, unthunk(v̄)))
        solve!(adj)
        gradient_logmu!(fwd, adj)
        return NoTangent(), get_field(fwd, :grad), NoTangent(), NoTangent(), NoTangent()
    end
    return v, top_vz_pullback
end

"""
    top_vz_ve(logμ, fwd, adj, Vwall, nt) -> (Vz on the top interior face plane, checkpoints)

nt Maxwell visco-elastic steps (assign_τ! + a converged PT loop each) from the walls and ICs
`Vwall = (Vx, Vy, Vz)` with cell viscosity exp.(logμ); `fwd` and `adj` are PTS_3D_VE_PERF
contexts of one grid, `adj` created with `adjoint=1`. The six stresses after each step are
kept on the host for the pullback.
"""
function top_vz_ve(logμ::Array{Float64,3}, fwd::Ctx, adj::Ctx, Vwall, nt::Integer)
    init_inclusion!(fwd; μs0=1.0, μsi=1.0, radius2=0.0, εbg=0.0)
    set_field!(fwd, :Vx, Vwall[1]); set_field!(fwd, :Vy, Vwall[2]); set_field!(fwd, :Vz, Vwall[3])
    set_field!(fwd, :Mus, exp.(logμ)); compute_maxloc!(fwd); compute_iter_params!(fwd)
    ckpt = Vector{Vector{Array{Float64,3}}}(undef, nt)
    for t in 1:nt
        assign_τ!(fwd)
        solve!(fwd)
        ckpt[t] = [get_field(fwd, s) for s in TAU]
    end
    Vz = get_field(fwd, :Vz)
    return Vz[2:end-1, 2:end-1, end-1], ckpt
end

# The backward time loop: the adjoint steps run in reverse order on the adjoint context with
# assign_τ! between steps (as forward), the source only in the first adjoint step; after
# adjoint step s the forward stresses of step nt-s are restored and that step's gradient
# term is accumulated.
function ChainRulesCore.rrule(::typeof(top_vz_ve), logμ::Array{Float64,3}, fwd::Ctx, adj::Ctx, Vwall, nt::Integer)
    v, ckpt = top_vz_ve(logμ, fwd, adj, Vwall, nt)
    function top_vz_ve_pullback(ȳ)
        v̄ = unthunk(ȳ)[1]
        v̄ isa AbstractZero && return NoTangent(), ZeroTangent(), NoTangent(), NoTangent(), NoTangent(), NoTangent()
        prepare_adjoint!(adj, logμ)
        Fz = top_source(adj, v̄)
        set_field!(adj, :Fz, Fz)
        for s in 0:nt-1
            assign_τ!(adj)
            solve!(adj)
            for (name, τ) in zip(TAU, ckpt[nt - s])
                set_field!(fwd, name, τ)
            end
            s == 0 ? gradient_logmu!(fwd, adj) : gradient_logmu_add!(fwd, adj)
            s == 0 && set_field!(adj, :Fz, zero(Fz))
        end
        return NoTangent(), get_field(fwd, :grad), NoTangent(), NoTangent(), NoTangent(), NoTangent()
    end
    return (v, ckpt), top_vz_ve_pullback
end

end # module
