"""
    ChaoslabB200Ext

B200 device for `Chaoslab.propagate`: installs `B200Device` when libchaoslab_b200 finds a functional sm_100 GPU,
and runs every device chunk of `Tangent._propagate` through the library's C ABI (include/chaoslab_b200.h) instead
of the KernelAbstractions launch of `_orbit_kernel!`. Runs outside the library's compiled menu report
"kernel does not compile for the element type" (FALLBACK_REASONS[3]) and stay on the CPU, as the reference does.
Drop-in next to ext/ChaoslabCUDAExt.jl (same hooks: src/Foundation/Foundation.jl:84-104, src/Tangent/propagate.jl:57-60).
"""
module ChaoslabB200Ext

using Chaoslab, StaticArrays, TOML
using Chaoslab.Foundation: Foundation, NumericalHealthError
using Chaoslab.Tangent: Tangent, STATUS_OK, STATUS_REDUCER
using Chaoslab.Lyapunov: QRSpectrum, Benettin, CGS, MGS, RGS, HouseholderQR, AugmentedQR, GivensQR
using Chaoslab.Indicators: SALI, GALI, MEGNO, FLI, RLI
using Chaoslab.Systems: StandardMap, WrappedStandardMap, FroeschleMap, StandardMapChain, LinearSymplecticMap,
                        HenonHeilesFlow, WrappedFroeschleMap, WrappedStandardMapChain
using Chaoslab.Integrators: IntegratorMap, Gauss, SplittingMethod, CorrectedMethod, coefficients

const libcl = get(ENV, "CHAOSLAB_B200_LIB", joinpath(@__DIR__, "libchaoslab_b200.so"))

# ---- the C structs (include/chaoslab_b200.h), field for field --------------------------------------------------
struct ClSystem
    kind::Int32; n_sites::Int32; ring::Int32; gauss_maxiter::Int32
    K::Float64; eps::Float64; nu::Float64; kappa::Float64; mu::Float64; gauss_tol::Float64; dt::Float64
    A::NTuple{256, Float64}
    n_stages::Int32; corrector::Int32
    stage_c::NTuple{128, Float64}; stage_d::NTuple{128, Float64}
end
struct ClReducer
    kind::Int32; alg::Int32; replace::Int32; pad::Int32; orthogonality_tol::Float64
end
struct ClFrame
    k::Int32; n_reducers::Int32; reducers::NTuple{4, ClReducer}
end
struct ClRun
    abi_version::Int32; d::Int32; s::Int32; tau::Int32
    N::Int64; n0::Int64; steps::Int64
    n_frames::Int32; precision::Int32; seed::UInt64; orbit_base::Int64
    sys::ClSystem; frames::NTuple{3, ClFrame}
end
struct ClBuffers
    x0::Ptr{Float64}; x::Ptr{Float64}
    W0::NTuple{3, Ptr{Float64}}; W::NTuple{3, Ptr{Float64}}; states::NTuple{3, Ptr{Cvoid}}
    code::NTuple{3, Ptr{Int8}}; hstep::NTuple{3, Ptr{Int64}}
end
struct ClProbe
    loadable::Int32; functional::Int32; compiles::Int32; sm::Int32
    free_bytes::Int64; total_bytes::Int64; sm_count::Int32; pad::Int32; device::NTuple{96, UInt8}
end

# The window kinds' reader (cl_window): kind 1 WeightedPhaseAdvance / 2 WeightedBirkhoff, the windows, the order,
# the observables as (kind, a, b): 1 Planar(iq, ip), 2 LiftedAngle(iq, im), 3 Cos(i, k), 4 Sin(i, k),
# 5 Lifted(iq, im), 6 IndCoordinate(i).
struct ClWindow
    kind::Int32; n_windows::Int32; n_observables::Int32; birkhoff_order::Int32
    window::NTuple{4, Int64}
    obs_kind::NTuple{8, Int32}; obs_a::NTuple{8, Int32}; obs_b::NTuple{8, Int32}
end

"A device call that failed; `code` is the library's return code (-2, -3, -4, -9)."
struct ClB200Error <: Exception
    code::Int32
    msg::String
end
Foundation.is_oom(e::ClB200Error) = e.code == -4
Foundation.is_compile_error(e::ClB200Error) = e.code == -3
Foundation.is_device_lost(e::ClB200Error) = e.code == -9

# ---- the menu: system and reducer records ----------------------------------------------------------------------
const ZA = ntuple(_ -> 0.0, 256)
const ZS = ntuple(_ -> 0.0, 128)
clsys(m::StandardMap{Float64}) = ClSystem(1, 0, 0, 0, m.K, 0, 0, 0, 0, NaN, 0, ZA, 0, 0, ZS, ZS)
clsys(m::WrappedStandardMap{Float64}) = ClSystem(2, 0, 0, 0, m.K, 0, 0, 0, 0, NaN, 0, ZA, 0, 0, ZS, ZS)
clsys(m::FroeschleMap{Float64}) = ClSystem(3, 0, 0, 0, 0, 0, m.nu, m.kappa, m.mu, NaN, 0, ZA, 0, 0, ZS, ZS)
clsys(m::StandardMapChain{Float64}) = ClSystem(4, m.N, m.ring, 0, m.K, m.eps, 0, 0, 0, NaN, 0, ZA, 0, 0, ZS, ZS)
clsys(m::WrappedFroeschleMap{Float64}) = ClSystem(8, 0, 0, 0, 0, 0, m.nu, m.kappa, m.mu, NaN, 0, ZA, 0, 0, ZS, ZS)
clsys(m::WrappedStandardMapChain{Float64}) =
    ClSystem(9, m.chain.N, m.chain.ring, 0, m.chain.K, m.chain.eps, 0, 0, 0, NaN, 0, ZA, 0, 0, ZS, ZS)
function clsys(m::LinearSymplecticMap{Float64, D}) where {D}
    return ClSystem(5, 0, 0, 0, 0, 0, 0, 0, 0, NaN, 0, ntuple(l -> l <= D * D ? m.A[l] : 0.0, 256), 0, 0, ZS, ZS)
end
clsys(m::IntegratorMap{<:Gauss{Float64, 3}, HenonHeilesFlow, Float64}) =
    ClSystem(6, 0, 0, m.method.maxiter, 0, 0, 0, 0, 0, m.method.tol, m.tau, ZA, 0, 0, ZS, ZS)
# a table method's weights travel as they are (Integrators/splitting.jl:16-21), at most 128 stages
function clsys(m::IntegratorMap{<:SplittingMethod{Float64, K}, HenonHeilesFlow, Float64}) where {K}
    K <= 128 || throw(ClB200Error(-3, "a splitting table of $K stages is above the compiled limit (128)"))
    c, d = coefficients(m.method)
    return ClSystem(7, 0, 0, 0, 0, 0, 0, 0, 0, NaN, m.tau, ZA, K, 0, ntuple(i -> i <= K ? c[i] : 0.0, 128),
                    ntuple(i -> i <= K ? d[i] : 0.0, 128))
end
# a corrected method (tables_near.jl:113-128): the base table, the corrector flag and its coefficient c in `eps`
function clsys(m::IntegratorMap{<:CorrectedMethod{Float64, <:SplittingMethod{Float64, K}}, HenonHeilesFlow, Float64}) where {K}
    K <= 128 || throw(ClB200Error(-3, "a splitting table of $K stages is above the compiled limit (128)"))
    c, d = coefficients(m.method.base)
    return ClSystem(7, 0, 0, 0, 0, m.method.c, 0, 0, 0, NaN, m.tau, ZA, K, 1, ntuple(i -> i <= K ? c[i] : 0.0, 128),
                    ntuple(i -> i <= K ? d[i] : 0.0, 128))
end
clsys(m) = throw(ClB200Error(-3, "system $(typeof(m)) is not in the compiled menu"))

qralg(::CGS) = 1; qralg(::MGS) = 2; qralg(::RGS) = 3
qralg(::HouseholderQR) = 4; qralg(::AugmentedQR) = 5; qralg(::GivensQR) = 6
clred(r::QRSpectrum) = ClReducer(1, qralg(r.alg), 0, 0, r.orthogonality_tol)
clred(::Benettin) = ClReducer(2, 0, 0, 0, 0)
clred(::SALI) = ClReducer(3, 0, 0, 0, 0)
clred(::GALI) = ClReducer(4, 0, 0, 0, 0)
clred(r::MEGNO) = ClReducer(5, 0, r.replace, 0, 0)
clred(r::FLI) = ClReducer(6, 0, r.replace, 0, 0)
clred(r::RLI) = ClReducer(7, 0, r.replace, 0, 0)          # the pair kind of the indicator recorder only
clred(r) = throw(ClB200Error(-3, "reducer $(typeof(r)) is not in the compiled menu"))

const NOFRAME = ClFrame(0, 0, ntuple(_ -> ClReducer(0, 0, 0, 0, 0), 4))
function clrun(sys, d, s, k, tau, N, n0, steps, reducers, seed, base)
    rs = map(clred, reducers)
    length(rs) <= 4 || throw(ClB200Error(-3, "more than four reducers"))
    fr = ClFrame(k, length(rs), ntuple(i -> i <= length(rs) ? rs[i] : ClReducer(0, 0, 0, 0, 0), 4))
    return ClRun(3, d, s, tau, N, n0, steps, 1, 0, seed % UInt64, base, clsys(sys), (fr, NOFRAME, NOFRAME))
end

function last_error()
    buf = Vector{UInt8}(undef, 1024)
    n = ccall((:cl_b200_last_error, libcl), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
    return String(buf[1:min(n, 1024)])
end

# ---- the device hooks ------------------------------------------------------------------------------------------
struct B200Device <: Foundation.AbstractDevice end
struct B200Backend end   # chunk buffers are host arrays: the library copies them to HBM and back

function __init__()
    isfile(libcl) || return
    p = Ref{ClProbe}()
    rc = ccall((:cl_b200_probe, libcl), Cint, (Ref{ClProbe},), p)
    rc == 0 && (Foundation.DEVICE[] = B200Device())
end

Tangent.device_backend(::B200Device) = B200Backend()
Tangent.workgroup(::B200Backend) = 128
function Foundation.free_memory(::B200Device)
    p = Ref{ClProbe}()
    ccall((:cl_b200_probe, libcl), Cint, (Ref{ClProbe},), p)
    return Int(p[].free_bytes)
end
# the device memory the library's pools keep between calls, back to the driver (as CUDA.reclaim() does for CUDA.jl)
function reclaim()
    rc = ccall((:cl_b200_release_cache, libcl), Cint, ())
    rc == 0 || throw(ClB200Error(rc, last_error()))
    return nothing
end
function Foundation.probe(::B200Device, ::Type{T}) where {T}
    p = Ref{ClProbe}()
    rc = ccall((:cl_b200_probe, libcl), Cint, (Ref{ClProbe},), p)
    name = String(filter(!iszero, collect(p[].device)))
    return (loadable = true, functional = p[].functional == 1, device = name,
            compiles = rc == 0 && T === Float64, gpu_faster = rc == 0 && T === Float64)
end

# Host buffers for the six chunk arrays of `_alloc_bufs` (propagate.jl:76-80).
function Tangent._alloc_bufs(::B200Backend, ::Type{SVector{s, T}}, ::Val{d}, ::Val{k}, ::Type{S}, m, mws) where {s, d, k, T, S}
    return (Vector{SVector{s, T}}(undef, m), Vector{SMatrix{d, k, T, d * k}}(undef, m), Vector{S}(undef, m),
            Vector{Int8}(undef, m), Vector{Int}(undef, m), zeros(UInt32, max(mws, 1), m))
end

# The one-wave record of the launch plan (propagate.jl:183-190): the same per-machine file and table layout as the
# CUDA extension's record (ext/ChaoslabCUDAExt.jl:42-62), written next to the library by the Python host's first
# measurement (chaos_b200/launch_plan.py); no record gives `nothing`, so the plan uses DEFAULT_GPU_NS.
const RECORD = joinpath(dirname(libcl), "data", "gpu-benchmark.toml")
function Foundation.gpu_step_ns(::B200Device, ::Type{T}) where {T}
    T === Float64 || return nothing
    try
        isfile(RECORD) || return nothing
        p = Ref{ClProbe}()
        ccall((:cl_b200_probe, libcl), Cint, (Ref{ClProbe},), p)
        name = String(filter(!iszero, collect(p[].device)))
        v = get(TOML.parsefile(RECORD)[name]["Float64"], "gpu_ns_per_step_wave", nothing)
        return v isa Real && isfinite(v) && v > 0 ? Float64(v) : nothing
    catch
        return nothing
    end
end

# `_run_chunk!` (propagate.jl:92-119) with each launch of `args.L` steps one cl_b200_propagate call on the carried
# host buffers (the first from x0 / W0, every later one continuing from x, W, states, code, hstep), the
# `_before_launch` hook before each; the host-side error and summary handling is the reference's, unchanged.
function Tangent._run_chunk!(out, bufs, Wh, r, args, who::Symbol, backend::B200Backend, ci::Int = 0)
    x, W, so, code, hstep, wsb = bufs
    len = length(r)
    copyto!(x, 1, args.x0, first(r), len)
    Tangent._fill_W!(Wh, r, args.seed, args.W0, args.dims..., args.T)
    copyto!(W, 1, Wh, 1, len)
    d, k = size(eltype(W))
    s = length(eltype(x))
    nul = Ptr{Float64}(0)
    n0, launch = 0, 0
    args.done[] = 0
    while n0 < args.N
        steps = min(args.L, args.N - n0)
        launch += 1
        Tangent._before_launch(Foundation.DEVICE[], ci, launch, (x = x, W = W, states = so, workspace = wsb))
        run = clrun(args.sys, d, s, k, args.tau, args.N, n0, steps, args.reducers, args.seed, first(r) - 1)
        GC.@preserve x W so code hstep begin
            bufsC = ClBuffers(pointer(x) |> Ptr{Float64}, pointer(x) |> Ptr{Float64},
                              (pointer(W) |> Ptr{Float64}, nul, nul), (pointer(W) |> Ptr{Float64}, nul, nul),
                              (sizeof(eltype(so)) == 0 ? Ptr{Cvoid}(0) : Ptr{Cvoid}(pointer(so)), Ptr{Cvoid}(0), Ptr{Cvoid}(0)),
                              (pointer(code), Ptr{Int8}(0), Ptr{Int8}(0)), (pointer(hstep), Ptr{Int64}(0), Ptr{Int64}(0)))
            rc = ccall((:cl_b200_propagate, libcl), Cint, (Ref{ClRun}, Int64, Ref{ClBuffers}, Ptr{Cvoid}),
                       run, len, bufsC, C_NULL)
        end
        rc == 0 || throw(ClB200Error(rc, last_error()))
        args.done[] = launch
        n0 += steps
    end
    i = findfirst(!=(STATUS_OK), view(code, 1:len))
    i === nothing || code[i] != STATUS_REDUCER || throw(Tangent._reducer_error(args.reducers, so[i], first(r) + i - 1, who))
    i === nothing || throw(Tangent._health_error(code[i], x[i], W[i], hstep[i], first(r) + i - 1, who))
    copyto!(out.x, first(r), x, 1, len)
    copyto!(out.W, first(r), W, 1, len)
    for i in 1:len
        out.finals[first(r) + i - 1] = map((rd, st) -> Tangent.reducer_final(rd, st, view(wsb, :, i)), args.reducers, so[i])
    end
end

end
