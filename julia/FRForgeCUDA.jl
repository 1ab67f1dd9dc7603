# FRForgeCUDA: the Julia binding of libfrforge_cuda.so (include/frforge_cuda.h).
#
# A maintainer adds this module next to FRForge's src/methods.  Existing case
# runners keep calling FRForge's own API; they get the GPU path by passing a
# GPUSolutionState made with `gpu(state, eq, method)`:
#
#     g = FRForgeCUDA.gpu(state, eq, method)          # 1D or 2D SolutionState
#     result = integrate!(g, eq, method, t_final; cfl = 0.1)
#     residual!(du, g, eq, method)
#
# What maps to the GPU, and what is refused with ArgumentError (the library's
# FRG_ERR_INVALID_ARG / FRG_ERR_UNSUPPORTED_HOOK, never a silent CPU path):
#   * SolutionState (1D, Mesh1D) and SolutionState2D (2D, Mesh2D);
#   * 2D geometry: an affine mesh goes as FRG_GEOM_AFFINE; a curved mesh
#     (state.metrics.is_curved) passes the state's own MeshMetrics2D arrays
#     (FRG_GEOM_METRICS), so the GPU uses exactly the caller's metrics;
#   * mesh.solid (2D solid-element mask) as a byte mask;
#   * PeriodicBC, TransmissiveBC, ReflectingBC (2D only, as in the reference's
#     1D residual), DirichletBC whose u_func is constant in (x, y, t) (checked
#     by sampling the domain corners and centre at several times; a state
#     that varies is refused), and GhostStateBC only where the case declares
#     its x-split form through `ghost_xsplit` (the double-Mach shape);
#   * NullCapturing, PerssonAVMethod, ScaledPerssonMethod, and any method
#     that declares `gpu_method_form`, with `gpu_hooks` naming the library's
#     device implementations of the hooks it overrides (selected on the
#     solve by `gpu`); other hook overrides are refused.
#
# The structs below mirror the C structs field for field (same names, same
# order); tests/test_julia_layout.py computes their layout under the C rules
# Julia uses for isbits structs and checks it with static assertions against
# include/frforge_cuda.h.
module FRForgeCUDA

using FRForge

const LIB = get(ENV, "FRFORGE_CUDA_LIB",
                joinpath(@__DIR__, "..", "frforge_b200", "libfrforge_cuda.so"))

# C: frg_bc
struct FrgBC
    kind::Cint
    mode::Cint
    state::NTuple{4,Float64}
    state_b::NTuple{4,Float64}
    x0::Float64
    s0::Float64
    s1::Float64
    sdiv::Float64
end

# C: frg_operators
struct FrgOperators
    p::Cint
    points::Cint
    xi::Ptr{Float64}
    w::Ptr{Float64}
    D::Ptr{Float64}
    l_L::Ptr{Float64}
    l_R::Ptr{Float64}
    gL_xi::Ptr{Float64}
    gR_xi::Ptr{Float64}
    V::Ptr{Float64}
end

# C: frg_metrics2d
struct FrgMetrics2D
    x_xi::Ptr{Float64}
    x_eta::Ptr{Float64}
    y_xi::Ptr{Float64}
    y_eta::Ptr{Float64}
    J::Ptr{Float64}
    nx_W::Ptr{Float64}
    ny_W::Ptr{Float64}
    sJ_W::Ptr{Float64}
    nx_E::Ptr{Float64}
    ny_E::Ptr{Float64}
    sJ_E::Ptr{Float64}
    nx_S::Ptr{Float64}
    ny_S::Ptr{Float64}
    sJ_S::Ptr{Float64}
    nx_N::Ptr{Float64}
    ny_N::Ptr{Float64}
    sJ_N::Ptr{Float64}
    h_char::Ptr{Float64}
end

# C: frg_solve_desc
struct FrgSolveDesc
    dim::Cint
    p::Cint
    points::Cint
    flux::Cint
    time_scheme::Cint
    gamma::Float64
    nx::Cint
    ny::Cint
    x_left::Float64
    x_right::Float64
    y_bottom::Float64
    y_top::Float64
    x_vertices::Ptr{Float64}
    y_vertices::Ptr{Float64}
    bc::NTuple{4,FrgBC}
    solid::Ptr{UInt8}
    geometry::Cint
    wavy_amp::Float64
    metrics::Ptr{FrgMetrics2D}
    ops::Ptr{FrgOperators}
    method::Cint
    av_form::Cint
    kappa::Float64
    s0_factor::Float64
    eps_floor::Float64
    c_av::Float64
end

# C: frg_result
struct FrgResult
    status::Cint
    n_steps::Int64
    t::Float64
end

const FRG_ERR_INVALID_ARG = -1
const FRG_ERR_UNSUPPORTED_HOOK = -2
const STATUS = Dict(0 => :ok, 1 => :diverged, 2 => :max_steps)
const BC_PERIODIC, BC_TRANSMISSIVE, BC_DIRICHLET, BC_REFLECTING, BC_XSPLIT = 0, 1, 2, 3, 4
const GEOM_AFFINE, GEOM_METRICS = 0, 2

last_error(ctx) = ctx == C_NULL ? "" :
    unsafe_string(ccall((:frg_last_error, LIB), Cstring, (Ptr{Cvoid},), ctx))

function check(rc, ctx)
    rc >= 0 && return rc
    msg = last_error(ctx)
    (rc == FRG_ERR_INVALID_ARG || rc == FRG_ERR_UNSUPPORTED_HOOK) && throw(ArgumentError(msg))
    error("frforge_cuda status $rc: $msg")
end

# ---------------------------------------------------------------- boundaries

const ZERO4 = (0.0, 0.0, 0.0, 0.0)
plain_bc(kind) = FrgBC(kind, 0, ZERO4, ZERO4, 0.0, 0.0, 0.0, 1.0)

"""
    ghost_xsplit(bc::GhostStateBC) -> nothing | NamedTuple

Extension point for GhostStateBC: a case whose ghost function is the x-split
shape (ghost = `state` for x < x0 + (s0 + s1 t)/sdiv, else the reflected
interior state (mode 0) or `state_b` (mode 1), as the double-Mach case of
src/verification/Cases2D_Optional.jl:72-84) declares it with a method for
its ghost function's type, returning (x0, s0, s1, sdiv, state, mode,
state_b).  Without one the boundary has no GPU form.
"""
ghost_xsplit(::GhostStateBC) = nothing

# a DirichletBC state as 4-tuple (2D) / 3-tuple (1D), refusing one that varies
function dirichlet_state(bc::DirichletBC, neq, box)
    f = bc.u_func
    at(x, y, t) = begin
        ub = applicable(f, x, y, t) ? f(x, y, t) : f(t)
        ntuple(c -> Float64(ub isa Number ? ub : ub[c]), neq)
    end
    (x0, x1, y0, y1) = box
    xm, ym = (x0 + x1) / 2, (y0 + y1) / 2
    ref = at(x0, y0, 0.0)
    for t in (0.0, 0.37, 1.0, 10.0), (x, y) in ((x0, y0), (x1, y0), (x0, y1), (x1, y1), (xm, ym))
        at(x, y, t) == ref || throw(ArgumentError(
            "DirichletBC u_func varies in (x, y, t): no GPU form (the GPU takes a constant state)"))
    end
    return ref
end

function frg_bc(bc, neq, box)
    bc isa PeriodicBC && return plain_bc(BC_PERIODIC)
    bc isa TransmissiveBC && return plain_bc(BC_TRANSMISSIVE)
    if bc isa ReflectingBC
        neq == 3 && throw(ArgumentError("ReflectingBC is not supported by the 1D residual"))
        return plain_bc(BC_REFLECTING)
    end
    if bc isa DirichletBC
        s = dirichlet_state(bc, neq, box)
        return FrgBC(BC_DIRICHLET, 0, ntuple(c -> c <= neq ? s[c] : 0.0, 4), ZERO4, 0.0, 0.0, 0.0, 1.0)
    end
    if bc isa GhostStateBC && neq == 4
        g = ghost_xsplit(bc)
        g === nothing && throw(ArgumentError(
            "GhostStateBC has no GPU form: declare FRForgeCUDA.ghost_xsplit for its ghost function"))
        return FrgBC(BC_XSPLIT, Cint(g.mode), Tuple(Float64.(g.state)), Tuple(Float64.(g.state_b)),
                     g.x0, g.s0, g.s1, g.sdiv)
    end
    throw(ArgumentError("BC $(typeof(bc)) has no GPU form"))
end

# ------------------------------------------------------------------- methods

"""
    gpu_method_form(method) -> (method, av_form, κ, s0_factor, ε_floor, c_av)

The descriptor fields of a capturing method.  A src/methods plugin whose
hooks the library implements (for example, one that only retunes Persson's
parameters) adds a method here; any other method is refused.
"""
gpu_method_form(::NullCapturing) = (0, 0, 4.0, -4.0, 1e-16, 0.0)
gpu_method_form(m::PerssonAVMethod) = (1, m.dissip.av_form == "element_local_DD" ? 1 : 0,
    Float64(m.sensor.κ), Float64(m.sensor.s0_factor), Float64(m.sensor.ε_floor), Float64(m.dissip.c_av))
gpu_method_form(m::ScaledPerssonMethod) = gpu_method_form(m.inner)
gpu_method_form(m::AbstractCapturingMethod) = throw(ArgumentError(
    "$(typeof(m)) overrides hooks with no GPU implementation (FRG_ERR_UNSUPPORTED_HOOK)"))

"""
    gpu_hooks(method) -> Vector{Tuple{String, Vector{Float64}}}

The device implementations a src/methods plugin selects for the hooks it
overrides, by registry name with their parameters (frg_hook_info lists
them: "positivity_zhang_shu" for post_step!, "flux_rusanov" / "flux_hllc"
for numerical_flux_method, "preprocess_positivity_zhang_shu" for
preprocess_state!, "traces_toward_mean" / "traces_positivity_zhang_shu"
for extrapolate_interface!).  The built-in methods select none.  A plugin
adds a `gpu_method_form` method (its descriptor fields, usually those of the
Persson method it wraps) and a `gpu_hooks` method naming its hooks'
implementations; `gpu(...)` selects them on the solve.
"""
gpu_hooks(::AbstractCapturingMethod) = Tuple{String, Vector{Float64}}[]
gpu_hooks(m::ScaledPerssonMethod) = gpu_hooks(m.inner)

function select_hooks!(g, method)
    for (name, params) in gpu_hooks(method)
        sl, id = Ref{Cint}(), Ref{Cint}()
        check(ccall((:frg_hook_lookup, LIB), Cint, (Cstring, Ref{Cint}, Ref{Cint}), name, sl, id), g.ctx)
        p = Vector{Float64}(params)
        check(ccall((:frg_solve_set_hook, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Float64}, Cint),
                    g.solve, sl[], id[], isempty(p) ? Ptr{Float64}(C_NULL) : pointer(p), length(p)), g.ctx)
    end
    return g
end

# ------------------------------------------------------------------- solves

mutable struct GPUSolutionState
    ctx::Ptr{Cvoid}
    solve::Ptr{Cvoid}
    host::Any          # the SolutionState / SolutionState2D it mirrors
    keep::Vector{Any}  # host arrays the descriptor points into
end

function operators_desc(o, keep)
    D = Matrix{Float64}(o.D)           # column-major, as the ABI expects
    V = Matrix{Float64}(o.V_legendre)
    arrs = (Vector{Float64}(o.ξ), Vector{Float64}(o.w), Vector{Float64}(o.ℓ_L), Vector{Float64}(o.ℓ_R),
            Vector{Float64}(o.gL_ξ), Vector{Float64}(o.gR_ξ))
    append!(keep, (D, V, arrs...))
    xi, w, lL, lR, gL, gR = arrs
    r = Ref(FrgOperators(o.p, o.points === :gl ? 0 : 1, pointer(xi), pointer(w), pointer(D),
                         pointer(lL), pointer(lR), pointer(gL), pointer(gR), pointer(V)))
    push!(keep, r)
    return r
end

function metrics_desc(met, keep)
    names = (:x_ξ, :x_η, :y_ξ, :y_η, :J, :nx_W, :ny_W, :sJ_W, :nx_E, :ny_E, :sJ_E,
             :nx_S, :ny_S, :sJ_S, :nx_N, :ny_N, :sJ_N, :h_char)
    arrs = [Array{Float64}(getfield(met, n)) for n in names]
    append!(keep, arrs)
    r = Ref(FrgMetrics2D((pointer(a) for a in arrs)...))
    push!(keep, r)
    return r
end

scheme_ints(s) = (s.points === :gl ? 0 : 1, s.flux === :hllc ? 1 : 0, s.time === :ssp_rk2 ? 1 : 0)

function create(desc::Ref{FrgSolveDesc}, state, keep, device)
    ctx = Ref{Ptr{Cvoid}}()
    check(ccall((:frg_ctx_create, LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), device, ctx), C_NULL)
    solve = Ref{Ptr{Cvoid}}()
    GC.@preserve keep begin
        check(ccall((:frg_solve_create, LIB), Cint, (Ptr{Cvoid}, Ref{FrgSolveDesc}, Ref{Ptr{Cvoid}}),
                    ctx[], desc, solve), ctx[])
    end
    return GPUSolutionState(ctx[], solve[], state, keep)
end

"""gpu(state::SolutionState2D, eq::Euler2D, method; device = 0)"""
function gpu(state::SolutionState2D, eq::Euler2D, method::AbstractCapturingMethod; device::Integer = 0)
    m, keep = state.mesh, Any[]
    m.geom_x === nothing || state.metrics.is_curved ||
        throw(ArgumentError("isoparametric mesh without curved metrics"))
    ops = operators_desc(state.ops, keep)
    xv, yv = Vector{Float64}(m.x_vertices), Vector{Float64}(m.y_vertices)
    append!(keep, (xv, yv))
    box = (xv[1], xv[end], yv[1], yv[end])
    bcs = (frg_bc(m.left_bc, 4, box), frg_bc(m.right_bc, 4, box), frg_bc(m.bottom_bc, 4, box),
           frg_bc(m.top_bc, 4, box))
    solid = Ptr{UInt8}(C_NULL)
    if m.solid !== nothing
        mask = UInt8.(m.solid)
        push!(keep, mask)
        solid = pointer(mask)
    end
    geometry, metrics = GEOM_AFFINE, Ptr{FrgMetrics2D}(C_NULL)
    if state.metrics.is_curved
        r = metrics_desc(state.metrics, keep)
        geometry, metrics = GEOM_METRICS, Base.unsafe_convert(Ptr{FrgMetrics2D}, r)
    end
    pts, flx, tim = scheme_ints(state.scheme)
    desc = Ref(FrgSolveDesc(2, state.p, pts, flx, tim, Float64(eq.γ), m.nx, m.ny, box..., pointer(xv),
                            pointer(yv), bcs, solid, geometry, 0.0, metrics,
                            Base.unsafe_convert(Ptr{FrgOperators}, ops), gpu_method_form(method)...))
    push!(keep, desc)
    return select_hooks!(create(desc, state, keep, device), method)
end

"""gpu(state::SolutionState, eq::Euler1D, method; device = 0)"""
function gpu(state::SolutionState, eq::Euler1D, method::AbstractCapturingMethod; device::Integer = 0)
    m, keep = state.mesh, Any[]
    ops = operators_desc(state.ops, keep)
    xv = Vector{Float64}(m.x_vertices)
    push!(keep, xv)
    box = (xv[1], xv[end], 0.0, 0.0)
    bcs = (frg_bc(m.left_bc, 3, box), frg_bc(m.right_bc, 3, box), plain_bc(BC_PERIODIC), plain_bc(BC_PERIODIC))
    pts, flx, tim = scheme_ints(state.scheme)
    desc = Ref(FrgSolveDesc(1, state.p, pts, flx, tim, Float64(eq.γ), m.n_elements, 1, xv[1], xv[end], 0.0,
                            1.0, pointer(xv), Ptr{Float64}(C_NULL), bcs, Ptr{UInt8}(C_NULL), GEOM_AFFINE,
                            0.0, Ptr{FrgMetrics2D}(C_NULL), Base.unsafe_convert(Ptr{FrgOperators}, ops),
                            gpu_method_form(method)...))
    push!(keep, desc)
    return select_hooks!(create(desc, state, keep, device), method)
end

function upload!(g::GPUSolutionState)
    u = g.host.u
    check(ccall((:frg_upload_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Csize_t, Float64),
                g.solve, u, length(u), g.host.t), g.ctx)
end

function download!(g::GPUSolutionState)
    t = Ref{Float64}()
    check(ccall((:frg_download_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Csize_t, Ref{Float64}),
                g.solve, g.host.u, length(g.host.u), t), g.ctx)
    g.host.t = t[]
end

"""residual!(du, g::GPUSolutionState, eq, method): the residual of g.host's state on the GPU."""
function FRForge.residual!(du, g::GPUSolutionState, eq, method)
    upload!(g)
    check(ccall((:frg_residual, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Csize_t),
                g.solve, du, length(du)), g.ctx)
    return du
end

"""integrate!(g::GPUSolutionState, eq, method, t_final; cfl, dt, max_steps) on the GPU."""
function FRForge.integrate!(g::GPUSolutionState, eq, method, t_final::Real;
                            cfl::Real = 0.2, dt = nothing, max_steps::Int = 10^7, kwargs...)
    upload!(g)
    r = Ref{FrgResult}()
    check(ccall((:frg_advance, LIB), Cint, (Ptr{Cvoid}, Float64, Float64, Float64, Int64, Ref{FrgResult}),
                g.solve, Float64(t_final), Float64(cfl), dt === nothing ? -1.0 : Float64(dt), max_steps, r),
          g.ctx)
    download!(g)
    return (status = STATUS[r[].status], n_steps = r[].n_steps, t = r[].t)
end

function release!(g::GPUSolutionState)
    g.solve == C_NULL || ccall((:frg_solve_destroy, LIB), Cint, (Ptr{Cvoid},), g.solve)
    g.ctx == C_NULL || ccall((:frg_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), g.ctx)
    g.solve, g.ctx = C_NULL, C_NULL
    return nothing
end

end # module
