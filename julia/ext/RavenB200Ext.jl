# RavenB200Ext -- Raven.jl's DGSEM tendency and LSRK stepping on libravenb200.so.
#
# A package extension for Raven.jl (hooked in through Raven's Project.toml [weakdeps] /
# [extensions], like RavenCUDAExt: see julia/Project.extension.toml).  It keeps Raven's
# Grid, GridArray{SVector{Ns,FT}} (CuArray-backed) and balance laws; only the device work
# behind these calls is redirected to the C ABI of include/raven_b200.h:
#   (dg::DGSEM)(dq, q, t; increment)            src/balancelaws/dgsem.jl:84-126, with the
#     DGSEM's directions (dgsem.jl:46-81)
#   solve!(q, timeend, solver; after_step,       src/balancelaws/odesolvers.jl:9-30
#          after_stage, adjust_final)
#   dostep!(q, ::LSRK / ::RLSRK, after_stage)    odesolvers.jl:51-61, 118-151, for the
#     5-stage (LSRK54, RLSRK54) and 14-stage (LSRK144, RLSRK144) tables
#   weightednorm(dg, q, p; componentwise)        src/balancelaws/measures.jl:6-21
#   entropyintegral, entropyproduct              measures.jl:23-33
#
# Stage callbacks.  The reference calls after_stage(stagetime, q) after every stage.  The
# fused step (all five stages as device kernels, one call) cannot do that, so:
#   * solve! on a B200 solver passes `nothing` as after_stage unless the caller gives a
#     callback, and dostep!(q, solver, nothing) runs the fused step;
#   * dostep!(q, solver, f::Function) runs the five stages one by one (rb200_lsrk54_stage),
#     writes each stage's result back into q and calls f(stagetime, q) after each, as the
#     reference does; a callback that changes q in place is seen by the next stage;
#   * any LSRK table (LSRK54, LSRK144, LSRK(rhs!, rka, rkb, rkc, ...)) runs both ways;
#     RLSRK runs its stages, entropy products and relaxation fused in the library, so for
#     it a stage callback raises an error instead of being ignored.
#
# Not run in this repository: no Julia exists on its build or GPU machines.  The Python
# binding (raven.jl_b200/_lib.py) drives the same entry points in the GPU tests.
module RavenB200Ext

using Raven, Raven.BalanceLaws, CUDA
import Raven.BalanceLaws: DGSEM, LSRK, RLSRK, dostep!, solve!, weightednorm, entropyintegral, entropyproduct

const lib = get(ENV, "RAVEN_B200_LIB", "libravenb200.so")

# mirrors rb200_desc (include/raven_b200.h); field order and types must match
struct RB200Desc
    abi_version::Int32
    dim::Int32
    nq::Int32
    law::Int32
    num_elements::Int64
    volume_form::Int32
    volume_flux::Int32
    surface_flux::Int32
    precision::Int32
    gamma::Float64
    advection_velocity::NTuple{3,Float64}
    D::Ptr{Float64}
    w::Ptr{Float64}
    volume_metrics::Ptr{Float64}
    surface_metrics::Ptr{Float64}
    vmapM::Ptr{Int64}
    vmapP::Ptr{Int64}
    boundary_codes::Ptr{Int64}
    device::Int32
end

check(st, h) =
    st == 0 || error("raven_b200: ", unsafe_string(ccall((:rb200_last_error, lib), Cstring, (Ptr{Cvoid},), h)))

lawcode(::Raven.BalanceLaws.Advection.AdvectionLaw) = Int32(0)
lawcode(::Raven.BalanceLaws.Euler.EulerLaw) = Int32(1)
formcode(::WeakForm) = (Int32(0), Int32(0))
formcode(f::FluxDifferencingForm) = (Int32(1), fluxcode(f.volume_numericalflux))
fluxcode(::CentralFlux) = Int32(0)
fluxcode(::KennedyGruberFlux) = Int32(1)
fluxcode(::EntropyConservativeFlux) = Int32(2)
fluxcode(::RusanovFlux) = Int32(3)
fluxcode(::RoeFlux) = Int32(4)     # Euler, FP64
fluxcode(::MatrixFlux) = Int32(5)  # Euler, FP64

"""
    B200DGSEM(dg::DGSEM; precision = :fp64)

The device handle of `dg` (rb200_create): the grid's metrics, face maps, boundary codes,
D and w are uploaded once.  `precision = :fp32_bulk` runs the volume and surface
arithmetic in FP32 with FP64 geometry, state and reductions.  Callable like `dg`.
"""
struct B200DGSEM{D}
    dg::D
    handle::Ptr{Cvoid}
end

function B200DGSEM(dg::DGSEM; precision = :fp64)
    grid, cell = dg.grid, referencecell(dg.grid)
    # host copies of what the Grid holds (rb200_create reads them once)
    vm = Array(parent(first(volumemetrics(grid))))      # (Nq^d, d*d+2, E)
    sm = Array(parent(first(surfacemetrics(grid))))     # (d+2, 2d*Nq^(d-1), E)
    fm = facemaps(grid)
    vmapM, vmapP = Array(fm.vmapM), Array(fm.vmapP)
    bc = Array(boundarycodes(grid))
    D, w = Array(derivatives_1d(cell)[1]), Array(vec(weights_1d(cell)[1]))
    form, vflux = formcode(dg.volume_form)
    law = dg.law
    u = law isa Raven.BalanceLaws.Advection.AdvectionLaw ? constants(law).u⃗ : ()
    adv = ntuple(i -> i <= length(u) ? Float64(u[i]) : 0.0, 3)
    gamma = law isa Raven.BalanceLaws.Euler.EulerLaw ? Float64(constants(law).γ) : 1.4
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve vm sm vmapM vmapP bc D w begin
        desc = RB200Desc(1, ndims(cell), size(cell, 1), lawcode(law), length(grid), form, vflux,
                         fluxcode(dg.surface_numericalflux), precision === :fp64 ? 0 : 1, gamma, adv,
                         pointer(D), pointer(w), pointer(vm), pointer(sm), pointer(vmapM), pointer(vmapP),
                         pointer(bc), CUDA.deviceid(CUDA.device()))
        st = ccall((:rb200_create, lib), Cint, (Ref{RB200Desc}, Ref{Ptr{Cvoid}}), desc, h)
        check(st, h[])
    end
    # DGSEM(; directions) (dgsem.jl:46-81): the volume and surface terms of those directions
    dirs = Raven.BalanceLaws.directions(dg)
    if length(dirs) < ndims(cell)
        mask = Int32(sum(1 << (d - 1) for d in dirs))
        check(ccall((:rb200_set_directions, lib), Cint, (Ptr{Cvoid}, Int32), h[], mask), h[])
    end
    b = B200DGSEM(dg, h[])
    finalizer(x -> ccall((:rb200_destroy, lib), Cint, (Ptr{Cvoid},), x.handle), b)
    return b
end

stream() = CUDA.stream().handle  # CUDA.jl's task-local stream keeps Julia's ordering

# boundarystate(law, problem, n, q-, aux-, tag) (balancelaw.jl:22) is a Julia method the
# device kernels cannot call; the two forms the reference's examples use are set per tag
# instead: a prescribed exterior state (examples/balancelaws/euler/sod.jl:15-21) or a
# reflecting wall (euler_gravity/gravitywave.jl:16-21); `nothing` restores q+ = q-.
function set_boundary_condition!(b::B200DGSEM, tag::Integer, cond)
    if cond === nothing
        st = ccall((:rb200_set_boundary_condition, lib), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}),
                   b.handle, tag, 0, C_NULL)
    elseif cond === :wall
        st = ccall((:rb200_set_boundary_condition, lib), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}),
                   b.handle, tag, 2, C_NULL)
    else
        state = Float64.(collect(cond))
        st = ccall((:rb200_set_boundary_condition, lib), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}),
                   b.handle, tag, 1, state)
    end
    check(st, b.handle)
    return b
end

# (dg)(dq, q, t; increment): the signature of DGSEM's call (dgsem.jl:84)
function (b::B200DGSEM)(dq, q, time; increment = true)
    st = ccall((:rb200_tendency, lib), Cint,
               (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Float64, Int32, Ptr{Cvoid}),
               b.handle, pointer(parent(dq)), pointer(parent(q)), time, increment, stream())
    check(st, b.handle)
    return dq
end

const B200LSRK = LSRK{FT,AT,NS,<:B200DGSEM} where {FT,AT,NS}
const B200RLSRK = RLSRK{FT,AT,NS,<:B200DGSEM} where {FT,AT,NS}

# the fused steps take the solver's own coefficient table (any NS up to 32 stages), so
# LSRK54, LSRK144 and LSRK(rhs!, rka, rkb, rkc, q, dt, t0) all run the same entry point
fused_lsrk(h, q, dq, rka, rkb, time, dt) =
    ccall((:rb200_lsrk_step, lib), Cint,
          (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Float64, Int32,
           Ptr{Cvoid}), h, q, dq, rka, rkb, length(rka), time, dt, 1, stream())
fused_rlsrk(h, q, dq, γ, rka, rkb, time, dt) =
    ccall((:rb200_rlsrk_step, lib), Cint,
          (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Ref{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Float64,
           Float64, Int32, Ptr{Cvoid}), h, q, dq, γ, rka, rkb, length(rka), time, dt, 1, stream())

# solve! (odesolvers.jl:9-30) for the B200 solvers: the same loop, with `nothing` as the
# default stage callback so that dostep! can run the fused step
function solve!(q, timeend, solver::Union{B200LSRK,B200RLSRK}; after_step::Function = (x...) -> nothing,
                after_stage::Union{Nothing,Function} = nothing, adjust_final = true)
    finalstep = false
    step = 0
    while true
        step += 1
        time = solver.time
        if time + solver.dt >= timeend
            adjust_final && (solver.dt = timeend - time)
            finalstep = true
        end
        dostep!(q, solver, after_stage)
        after_step(step, time, q)
        finalstep && break
    end
end

# all stages fused on the device (rb200_lsrk_step with the solver's table)
function dostep!(q, lsrk::LSRK{FT,AT,NS,<:B200DGSEM}, ::Nothing) where {FT,AT,NS}
    rka, rkb = Float64[lsrk.rka...], Float64[lsrk.rkb...]
    st = fused_lsrk(lsrk.rhs!.handle, pointer(parent(q)), pointer(parent(lsrk.dq)), rka, rkb, lsrk.time, lsrk.dt)
    check(st, lsrk.rhs!.handle)
    lsrk.time += lsrk.dt
end

# stage by stage (rb200_lsrk_stage with the solver's a_i, b_i), after_stage(stagetime, q)
# after each with stagetime = time + c_i dt (odesolvers.jl:51-60)
function dostep!(q, lsrk::LSRK{FT,AT,NS,<:B200DGSEM}, after_stage::Function) where {FT,AT,NS}
    out = similar(parent(q))
    for stage = 1:NS
        stagetime = lsrk.time + lsrk.rkc[stage] * lsrk.dt
        st = ccall((:rb200_lsrk_stage, lib), Cint,
                   (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, Float64, Float64, Float64, Float64,
                    Ptr{Cvoid}),
                   lsrk.rhs!.handle, pointer(parent(q)), pointer(out), pointer(parent(lsrk.dq)),
                   Float64(lsrk.rka[stage]), Float64(lsrk.rkb[stage]), stagetime, lsrk.dt, stream())
        check(st, lsrk.rhs!.handle)
        copyto!(parent(q), out)
        after_stage(stagetime, q)
    end
    CUDA.unsafe_free!(out)
    lsrk.time += lsrk.dt
end

# RLSRK54 / RLSRK144 (odesolvers.jl:118-151): the stages, entropy products and the
# relaxation solve run in the library; γ is read from and written back to the RLSRK struct
function dostep!(q, r::RLSRK{FT,AT,NS,<:B200DGSEM}, ::Nothing) where {FT,AT,NS}
    γ = Ref(Float64(r.γ))
    rka, rkb = Float64[r.rka...], Float64[r.rkb...]
    st = fused_rlsrk(r.rhs!.handle, pointer(parent(q)), pointer(parent(r.dq)), γ, rka, rkb, r.time, r.dt)
    check(st, r.rhs!.handle)
    r.γ = γ[]
    r.time += r.dt
end

dostep!(q, r::B200RLSRK, ::Function) =
    error("raven_b200: RLSRK runs its stages fused on the device; after_stage is not supported")

function entropyintegral(b::B200DGSEM, q)
    out = Ref(0.0)
    st = ccall((:rb200_entropy_integral, lib), Cint, (Ptr{Cvoid}, CuPtr{Float64}, Ref{Float64}, Ptr{Cvoid}),
               b.handle, pointer(parent(q)), out, stream())
    check(st, b.handle)
    return out[]
end

function entropyproduct(b::B200DGSEM, p, q)
    out = Ref(0.0)
    st = ccall((:rb200_entropy_product, lib), Cint,
               (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Ref{Float64}, Ptr{Cvoid}),
               b.handle, pointer(parent(p)), pointer(parent(q)), out, stream())
    check(st, b.handle)
    return out[]
end

# weightednorm(dg, q, p = 2; componentwise) (measures.jl:6-21), p = Inf included
function weightednorm(b::B200DGSEM, q, p = 2; componentwise = false)
    Ns = length(eltype(q))
    out = zeros(Float64, Ns + 1)
    st = ccall((:rb200_weightednorm_p, lib), Cint, (Ptr{Cvoid}, CuPtr{Float64}, Float64, Ptr{Float64}, Ptr{Cvoid}),
               b.handle, pointer(parent(q)), Float64(p), out, stream())
    check(st, b.handle)
    return componentwise ? ntuple(s -> out[s], Ns) : out[end]
end

end # module
