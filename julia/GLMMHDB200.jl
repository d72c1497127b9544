# GLMMHDB200.jl -- the reference's Julia step API routed to libglmmhd_b200.so (sm_100a).
#
# NOT RUN HERE: this image has no Julia.  The module is the Julia side of the drop-in boundary, the
# binding a GLMMHDTurb maintainer adds next to glmmhd_turb.jl / ct_mhd.jl.  Every `ccall` below
# binds a symbol declared in include/glmmhd_b200.h with the same argument and return types
# (tests/test_julia_glue.py checks each signature against the header on every CPU test run).  The
# Python mirror glmmhdturb_b200/turb.py, ctmhd.py and march_bridge.py binds the same entry points and
# is what the GPU tests exercise.
#
#   step_plm!(uold, unew, afield, p, dt, t; do_turb, nthreads, tb, half, riemann, recon)  glmmhd_turb.jl:878
#   step_tiled!(uold, unew, afield, p, dt, t; use_hlld, do_turb, nthreads, maxregs, lean) glmmhd_turb.jl:746
#   step_fused!(uold, unew, afield, p, dt, t, be; use_hlld, do_turb)                       glmmhd_turb.jl:579
#   step_multi!(uold, unew, rec, flx, ct, afield, p, dt, t, be; use_hlld, do_turb)         glmmhd_turb.jl:1981
#   compute_dt(uold, ct, p, be)                                                            glmmhd_turb.jl:1973
#   diagnostics(u, ct, p, be)                                                              glmmhd_turb.jl:2006
#   Forcing(p, be; amp), ou_advance!(f, p, be)      the 61-mode OU forcing (replaces :2116-2161)
#   CTMHD.step!(U, bxf, byf, bzf, bccx, bccy, bccz, Fx, Fy, Fz, ex, ey, ez, dt, dx, N)      ct_mhd.jl:174
#   step_frozen + ChainRulesCore.rrule              the pullback of one step (gmt_adjoint_step)
#
# States are the reference's (N,N,N,9) Float32 (or Float64) CuArrays: nine contiguous N^3 planes,
# x fastest, exactly the layout the library takes.  `afield` is a `Forcing` (or nothing); the
# scratch arguments (rec, flx, ct, be) are accepted for signature compatibility and unused, since
# each context keeps its own scratch.  Errors are raised as in the reference (`error(...)`) with the
# library's message.
module GLMMHDB200

using CUDA
using ChainRulesCore

const LIB = get(ENV, "GLMMHDB200_LIB", joinpath(@__DIR__, "..", "glmmhdturb_b200", "libglmmhd_b200.so"))

const GMT_ABI_VERSION = Int32(1)
const GMT_F32, GMT_F64 = Int32(0), Int32(1)
const GMT_SCHEME_UNSPLIT, GMT_SCHEME_MARCH1D, GMT_SCHEME_CT = Int32(0), Int32(1), Int32(2)
const GMT_RECON = Dict(:mc => Int32(0), :plm => Int32(0), :minmod => Int32(1), :ppm => Int32(2))
const GMT_RIEMANN = Dict(:hlld => Int32(0), :hll => Int32(1), :llf => Int32(2), :llf_bound => Int32(3))
const GMT_EMF = Dict(:average => Int32(0), :contact => Int32(1))
const NDIM = 3
const TB = 4

# mirrors `gmt_params` (include/glmmhd_b200.h): field order and types must match
mutable struct GmtParams
    abi_version::Int32; nx::Int32; ny::Int32; nz::Int32; dtype::Int32; scheme::Int32
    recon::Int32; riemann::Int32; iflo::Int32; emf::Int32; ct_halfslope::Int32
    tile_x::Int32; tile_y::Int32; tile_z::Int32; nsp::Int32
    boxlen::Float64; gamma::Float64; courant::Float64; smallr::Float64; smallc::Float64; smallp::Float64
    glm_ch_scale::Float64; glm_cp_coef::Float64; llf_dmin::Float64; llf_pmin::Float64
    turb_min_rho::Float64; turb_amp::Float64; turb_T::Float64; turb_ndt::Int32; turb_seed::UInt32
end
GmtParams() = GmtParams(zeros(Int32, 15)..., zeros(Float64, 13)..., Int32(0), UInt32(0))

struct GmtStepArgs
    dt::Float64; t::Float64; ch::Float64; glm_fac::Float64; do_turb::Int32; want_cfl::Int32
end

struct GmtDiag
    mass::Float64; ke2::Float64; vrms::Float64; divbmax::Float64; rhomin::Float64; etot::Float64
    divb_l2::Float64; psi_l2::Float64; finite::Int32; nonfinite_cells::Int32
end
GmtDiag() = GmtDiag(0, 0, 0, 0, 0, 0, 0, 0, 0, 0)

last_error() = unsafe_string(ccall((:gmt_last_error, LIB), Cstring, ()))
check(rc::Integer, what) = rc == 0 ? nothing : error("$what: ", last_error())
stream_handle() = CUDA.stream().handle

# ---------------------------------------------------------------------------------------------
# Params (glmmhd_turb.jl:28-52) and a cache of library contexts, one per configuration
# ---------------------------------------------------------------------------------------------
Base.@kwdef struct Params
    N::Int = 256
    boxlen::Float32 = 1.0f0
    gamma::Float32 = 1.01f0
    courant::Float32 = 0.7f0
    smallr::Float32 = 1.0f-6
    smallc::Float32 = 1.0f-4
    glm_ch_scale::Float32 = 0.25f0
    glm_cp_coef::Float32 = 0.18f0
    switch_llf_dmin::Float32 = 0.0f0
    switch_llf_pmin::Float32 = 0.0f0
    rho0::Float32 = 1.0f0
    cs0::Float32 = 1.0f0
    b0::Float32 = 1.0f0
    turb_rms::Float32 = 130.0f0
    turb_T::Float32 = 0.3f0
    turb_Ndt::Int = 100
    comp_frac::Float32 = 0.5f0
    turb_min_rho::Float32 = 1.0f-5
    turb_seed::UInt32 = 0x00000001
end
dxof(p::Params) = p.boxlen / p.N
pfloor(p::Params) = p.smallr * p.smallc^2 / p.gamma

mutable struct Context
    ptr::Ptr{Cvoid}
    function Context(gp::GmtParams)
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:gmt_create, LIB), Cint, (Ref{GmtParams}, Ref{Ptr{Cvoid}}), gp, out), "gmt_create")
        c = new(out[])
        finalizer(c) do x
            x.ptr == C_NULL || ccall((:gmt_destroy, LIB), Cint, (Ptr{Cvoid},), x.ptr)
            x.ptr = C_NULL
        end
        return c
    end
end

dtype_code(::Type{Float32}) = GMT_F32
dtype_code(::Type{Float64}) = GMT_F64
dtype_code(T) = error("state eltype must be Float32 or Float64, got $T")

function params_for(p::Params, T; scheme=GMT_SCHEME_UNSPLIT, recon=:mc, riemann=:hlld, iflo=true, emf=:average,
                    ct_halfslope=false, smallp=1e-6, gamma=p.gamma)
    gp = GmtParams()
    check(ccall((:gmt_params_init, LIB), Cint, (Ref{GmtParams}, Cint), gp, p.N), "gmt_params_init")
    gp.dtype = dtype_code(T); gp.scheme = scheme
    gp.recon = GMT_RECON[recon]; gp.riemann = GMT_RIEMANN[riemann]; gp.iflo = iflo; gp.emf = GMT_EMF[emf]
    gp.ct_halfslope = ct_halfslope
    gp.boxlen = p.boxlen; gp.gamma = gamma; gp.courant = p.courant; gp.smallr = p.smallr; gp.smallc = p.smallc
    gp.smallp = smallp; gp.glm_ch_scale = p.glm_ch_scale; gp.glm_cp_coef = p.glm_cp_coef
    gp.llf_dmin = p.switch_llf_dmin; gp.llf_pmin = p.switch_llf_pmin; gp.turb_min_rho = p.turb_min_rho
    gp.turb_amp = p.turb_rms; gp.turb_T = p.turb_T; gp.turb_ndt = p.turb_Ndt; gp.turb_seed = p.turb_seed
    return gp
end

const CONTEXTS = Dict{Any,Context}()
function context(p::Params, T; kw...)
    key = (p, T, sort(collect(kw)), CUDA.device())
    get!(CONTEXTS, key) do
        Context(params_for(p, T; kw...))
    end
end

# ---------------------------------------------------------------------------------------------
# Forcing: the library's deterministic 61-mode solenoidal OU (1 <= |k| <= 3), one context per
# Forcing; `next_time` and the cadence turb_T/turb_Ndt follow the reference host loop (:2146-2161)
# ---------------------------------------------------------------------------------------------
mutable struct Forcing
    p::Params
    ctx::Context
    next_time::Float64
    version::Int
end
function Forcing(p::Params, be=nothing; amp=p.turb_rms, T=Float32)
    fields = NamedTuple{fieldnames(Params)}(Tuple(getfield(p, f) for f in fieldnames(Params)))
    q = Params(; merge(fields, (turb_rms=Float32(amp),))...)
    ctx = context(q, T)
    check(ccall((:gmt_forcing_reset, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), ctx.ptr, stream_handle()), "gmt_forcing_reset")
    return Forcing(q, ctx, 0.0, 0)
end
function ou_advance!(f::Forcing, p=nothing, be=nothing)
    check(ccall((:gmt_forcing_advance, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), f.ctx.ptr, stream_handle()),
          "gmt_forcing_advance")
    f.next_time += f.p.turb_T / f.p.turb_Ndt
    f.version += 1
    return f
end
function modes(f::Forcing)
    m = zeros(Float64, 2 * 3 * 61)
    check(ccall((:gmt_forcing_get_modes, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Cvoid}), f.ctx.ptr, m,
                stream_handle()), "gmt_forcing_get_modes")
    return m
end
const FORCING_SEEN = IdDict{Context,Tuple{UInt,Int}}()
function forcing_into(ctx::Context, afield, do_turb::Bool)
    do_turb || return
    afield isa Forcing || error("do_turb=true needs a Forcing as afield")
    afield.ctx === ctx && return
    tag = (objectid(afield), afield.version)
    get(FORCING_SEEN, ctx, nothing) == tag && return
    check(ccall((:gmt_forcing_set_modes, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Cvoid}), ctx.ptr, modes(afield),
                stream_handle()), "gmt_forcing_set_modes")
    FORCING_SEEN[ctx] = tag
end

# ch = courant*dx/dt/3*glm_ch_scale, glm_fac = exp(-(ch^2/(cp*L*ch))*dt) (glmmhd_turb.jl:582-583)
function glm_parameters(p::Params, dt)
    ch = p.courant * dxof(p) / dt / NDIM * p.glm_ch_scale
    fac = p.glm_cp_coef > 0 ? exp(-(ch * ch / (p.glm_cp_coef * p.boxlen * ch)) * dt) : 1.0
    return ch, fac
end

function _step!(uold::CuArray{T}, unew::CuArray{T}, afield, p::Params, dt, t; recon, riemann, iflo, do_turb) where {T}
    size(uold) == (p.N, p.N, p.N, 9) || error("state must be (N,N,N,9), got $(size(uold))")
    uold === unew && error("uold and unew must be different arrays")
    ctx = context(p, T; recon=recon, riemann=riemann, iflo=iflo)
    forcing_into(ctx, afield, do_turb)
    ch, fac = glm_parameters(p, dt)
    a = GmtStepArgs(dt, t, ch, fac, do_turb, 0)
    check(ccall((:gmt_step, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ref{GmtStepArgs}, Ptr{Cvoid}),
                ctx.ptr, uold, unew, a, stream_handle()), "gmt_step")
    return nothing
end

# Production PLM/PPM step (glmmhd_turb.jl:878-908).  `half` selected 16-bit shared tiles in the
# reference; the library always stages FP32/FP64 tiles.  Any (recon, riemann) pair is built.
function step_plm!(uold, unew, afield, p::Params, dt::Real, t::Real; do_turb::Bool=false, nthreads::Int=192,
                   tb::Int=0, half::Bool=true, riemann::Symbol=:hll, recon::Symbol=:plm)
    tb == 0 && (tb = p.N % 6 == 0 ? 6 : 4)
    p.N % tb == 0 || error("N=$(p.N) not divisible by tb=$tb (need N%6==0 for the fast TB=6 path, or N%4==0)")
    recon in (:plm, :ppm) || error("step_plm!: unsupported recon=$recon")
    riemann in (:hll, :llf, :hlld) || error("step_plm!: unsupported riemann=$riemann")
    rs = riemann === :llf ? :llf_bound : riemann
    _step!(uold, unew, afield, p, dt, t; recon=recon === :ppm ? :ppm : :mc, riemann=rs, iflo=true, do_turb=do_turb)
end

# Tiled HLLD step (glmmhd_turb.jl:746-767); lean = minmod slopes + LLF with the bound speed
function step_tiled!(uold, unew, afield, p::Params, dt::Real, t::Real; use_hlld::Bool=true, do_turb::Bool=false,
                     nthreads::Int=192, maxregs::Int=0, lean::Bool=false)
    p.N % TB == 0 || error("N must be a multiple of $TB")
    if lean
        _step!(uold, unew, afield, p, dt, t; recon=:minmod, riemann=:llf_bound, iflo=true, do_turb=do_turb)
    else
        _step!(uold, unew, afield, p, dt, t; recon=:mc, riemann=use_hlld ? :hlld : :llf, iflo=true, do_turb=do_turb)
    end
end

# Recompute step (glmmhd_turb.jl:579-589) and multi-kernel validation step (:1981-1992): no
# interface-state revert
step_fused!(uold, unew, afield, p::Params, dt::Real, t::Real, be=nothing; use_hlld::Bool=true, do_turb::Bool=false) =
    _step!(uold, unew, afield, p, dt, t; recon=:mc, riemann=use_hlld ? :hlld : :llf, iflo=false, do_turb=do_turb)
step_multi!(uold, unew, rec, flx, ct, afield, p::Params, dt::Real, t::Real, be=nothing; use_hlld::Bool=true,
            do_turb::Bool=false) =
    _step!(uold, unew, afield, p, dt, t; recon=:mc, riemann=use_hlld ? :hlld : :llf, iflo=false, do_turb=do_turb)

# dt = courant*dx/max(sum_d(|v_d|+c_f)) (glmmhd_turb.jl:1973-1978); FP64 reduction on the device
function compute_dt(uold::CuArray{T}, ct, p::Params, be=nothing) where {T}
    ctx = context(p, T)
    dt = Ref{Float64}(0)
    check(ccall((:gmt_compute_dt, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, Ref{Float64}, Ptr{Cvoid}),
                ctx.ptr, uold, dt, stream_handle()), "gmt_compute_dt")
    return T(dt[])
end

# mass, vrms, Mach, centred div B max, rhomin, finite (glmmhd_turb.jl:2006-2018)
function diagnostics(u::CuArray{T}, ct, p::Params, be=nothing) where {T}
    ctx = context(p, T)
    d = Ref(GmtDiag())
    check(ccall((:gmt_diagnostics, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, Ref{GmtDiag}, Ptr{Cvoid}),
                ctx.ptr, u, d, stream_handle()), "gmt_diagnostics")
    x = d[]
    return (mass=x.mass, vrms=x.vrms, mach=x.vrms / p.cs0, divbmax=x.divbmax, rhomin=x.rhomin,
            finite=x.finite != 0, etot=x.etot, divb_l2=x.divb_l2)
end

# initial states on the device (glmmhd_turb.jl:2021-2036, 2164-2172)
function ic_ot!(u::CuArray{T}, p::Params) where {T}
    check(ccall((:gmt_ic_orszag_tang, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}), context(p, T).ptr, u,
                stream_handle()), "gmt_ic_orszag_tang")
end
function ic_uniform!(u::CuArray{T}, p::Params; rho0=p.rho0, p0=p.rho0 * p.cs0^2 / p.gamma, b0=(p.b0, 0, 0)) where {T}
    check(ccall((:gmt_ic_uniform, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, Float64, Float64, Float64, Float64, Float64, Ptr{Cvoid}),
                context(p, T).ptr, u, rho0, p0, b0[1], b0[2], b0[3], stream_handle()), "gmt_ic_uniform")
end

# driven turbulence (glmmhd_turb.jl:2191-2240) with the mode-sum OU forcing
function run_turb(; N=128, t_end=0.6f0, amp=130.0f0, use_hlld=true, nstepmax=20000, T=Float32)
    p0 = 1 / 1.01f0
    p = Params(; N=N, turb_rms=amp, switch_llf_dmin=0.01f0, switch_llf_pmin=0.01f0 * p0)
    u1 = CUDA.zeros(T, N, N, N, 9); u2 = similar(u1)
    ic_uniform!(u1, p)
    f = Forcing(p; amp=amp, T=T)
    ou_advance!(f, p)
    t, step = 0.0, 0
    while t < t_end && step < nstepmax
        while t >= f.next_time
            ou_advance!(f, p)
        end
        dt = min(Float64(compute_dt(u1, nothing, p)), f.next_time - t, t_end - t)
        step_tiled!(u1, u2, f, p, dt, t; use_hlld=use_hlld, do_turb=true)
        u1, u2 = u2, u1
        t += dt; step += 1
    end
    return merge(diagnostics(u1, nothing, p), (steps=step, t=t))
end

# ---------------------------------------------------------------------------------------------
# Differentiation: one step with dt, ch, glm_fac and the forcing modes frozen, and its pullback
# (gmt_adjoint_step).  gmt_adjoint_amp_grad returns the accumulated dL/d(turb_amp).
# ---------------------------------------------------------------------------------------------
function step_frozen(ctx::Context, u::CuArray, dt, t, ch, fac, do_turb)
    unew = similar(u)
    a = GmtStepArgs(dt, t, ch, fac, do_turb, 0)
    check(ccall((:gmt_step, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ref{GmtStepArgs}, Ptr{Cvoid}),
                ctx.ptr, u, unew, a, stream_handle()), "gmt_step")
    return unew
end
function ChainRulesCore.rrule(::typeof(step_frozen), ctx::Context, u::CuArray, dt, t, ch, fac, do_turb)
    unew = step_frozen(ctx, u, dt, t, ch, fac, do_turb)
    function step_frozen_pullback(ubar_next)
        ubar = similar(u)
        ub = CuArray(unthunk(ubar_next))
        a = GmtStepArgs(dt, t, ch, fac, do_turb, 0)
        check(ccall((:gmt_adjoint_step, LIB), Cint,
                    (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ref{GmtStepArgs}, Ptr{Cvoid}),
                    ctx.ptr, u, ub, ubar, a, stream_handle()), "gmt_adjoint_step")
        return NoTangent(), NoTangent(), ubar, NoTangent(), NoTangent(), NoTangent(), NoTangent(), NoTangent()
    end
    return unew, step_frozen_pullback
end
function amp_grad(ctx::Context; reset=true)
    g = Ref{Float64}(0)
    check(ccall((:gmt_adjoint_amp_grad, LIB), Cint, (Ptr{Cvoid}, Ref{Float64}, Int32, Ptr{Cvoid}), ctx.ptr, g,
                Int32(reset), stream_handle()), "gmt_adjoint_amp_grad")
    return g[]
end
# band-limited KE loss of the differentiable run and its gradient dL/du
function ke_band_loss(ctx::Context, u::CuArray, kmin, kmax)
    L = Ref{Float64}(0)
    ubar = similar(u)
    check(ccall((:gmt_ke_band_loss, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, Int32, Int32, Ref{Float64}, CuPtr{Cvoid},
                                                   Ptr{Cvoid}),
                ctx.ptr, u, Int32(kmin), Int32(kmax), L, ubar, stream_handle()), "gmt_ke_band_loss")
    return L[], ubar
end

# ---------------------------------------------------------------------------------------------
# CTMHD (ct_mhd.jl): one CT step with fixed dt, in place on (U, bxf, byf, bzf).  Fx and Fy are
# the reference's (N,N,N,8) scratch; here they hold the packed old and new 8-plane states
# [rho, mx, my, mz, E, bxf, byf, bzf] that gmt_ct_step takes.  ct_mhd.jl's constants: gamma = 5/3,
# SMALLR = SMALLP = 1e-6, HLL, Balsara-Spicer average EMF, its extra slope halving (:49-50).
# ---------------------------------------------------------------------------------------------
module CTMHD
using CUDA
import ..GLMMHDB200: LIB, GmtStepArgs, Context, params_for, Params, check, stream_handle, GMT_SCHEME_CT

const GAMMA = 5f0 / 3f0
const CONTEXTS = Dict{Any,Context}()
function ctx_for(N, T, dx)
    get!(CONTEXTS, (N, T, dx, CUDA.device())) do
        p = Params(; N=N, boxlen=Float32(dx * N), smallr=1f-6)
        Context(params_for(p, T; scheme=GMT_SCHEME_CT, recon=:mc, riemann=:hll, emf=:average, ct_halfslope=true,
                           smallp=1e-6, gamma=GAMMA))
    end
end

function step!(U, bxf, byf, bzf, bccx, bccy, bccz, Fx, Fy, Fz, ex, ey, ez, dt, dx, N)
    T = eltype(U)
    n3 = N^3
    q, o = reshape(Fx, n3, 8), reshape(Fy, n3, 8)
    q[:, 1:5] .= reshape(U, n3, 5)
    q[:, 6] .= vec(bxf); q[:, 7] .= vec(byf); q[:, 8] .= vec(bzf)
    a = GmtStepArgs(dt, 0.0, 0.0, 1.0, 0, 0)
    check(ccall((:gmt_ct_step, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ref{GmtStepArgs}, Ptr{Cvoid}),
                ctx_for(N, T, dx).ptr, Fx, Fy, a, stream_handle()), "gmt_ct_step")
    reshape(U, n3, 5) .= o[:, 1:5]
    vec(bxf) .= o[:, 6]; vec(byf) .= o[:, 7]; vec(bzf) .= o[:, 8]
    return
end

scratch(N) = (CUDA.zeros(Float32, N, N, N), CUDA.zeros(Float32, N, N, N), CUDA.zeros(Float32, N, N, N),
              CUDA.zeros(Float32, N, N, N, 8), CUDA.zeros(Float32, N, N, N, 8), CUDA.zeros(Float32, N, N, N, 8),
              CUDA.zeros(Float32, N, N, N), CUDA.zeros(Float32, N, N, N), CUDA.zeros(Float32, N, N, N))

# face div B for cell i = (upper face - lower face)/dx per dim (ct_mhd.jl:190-194)
function divB_max(bxf, byf, bzf, dx)
    db = (circshift(bxf, (-1, 0, 0)) .- bxf .+ circshift(byf, (0, -1, 0)) .- byf .+ circshift(bzf, (0, 0, -1)) .- bzf) ./ dx
    Float64(maximum(abs.(db)))
end
end # module CTMHD

end # module GLMMHDB200
