# B200 backend for DiplodocusTransport.jl's explicit Euler path, over libdtb.so.
#
# Not exercised in this repository (no Julia toolchain here); it shows the exact `ccall`
# bindings of include/dtb.h that the reference would add: the plain method behind the
# reference's stepping struct and Solve, and batched solves of one grid (B200BatchedEuler).
# Loaded after DiplodocusTransport:
#
#     using DiplodocusTransport
#     include("DTB200Backend.jl"); using .DTB200Backend
#     Backend = B200Backend()            # instead of CPUBackend() / CUDABackend()
#     method = ForwardEulerStruct(PhaseSpace, Initial, Injection, BinM, EmiM, FluxM)  # patched reference
#     method = B200ForwardEulerStruct(PhaseSpace, Initial, Injection, BinM, EmiM, FluxM)  # unpatched
#     output = Solve(method, dt, t_save)  # the reference's Solve, unchanged
#
# B200ForwardEulerStruct takes the same arguments as ForwardEulerStruct and carries the
# fields Solve reads; the reference's own types are left untouched.
module DTB200Backend

using DiplodocusTransport
using SparseArrays

import DiplodocusTransport: BackendType, PhaseSpaceStruct

export B200Backend, B200ForwardEulerStruct, b200_solve, b200_step_io!
export B200BatchedEuler, admit!, run!, run_io!, get_f, batch_moments, gemm_plan, set_tune_cache
export B200Server, add_grid!, start!, submit!, wait_request, cancel!, serve_stats

const libdtb = get(ENV, "DTB_LIB", joinpath(@__DIR__, "..", "lib", "libdtb.so"))

# With the reference patched (Backends.jl defines B200Backend and b200_stepping_struct), the
# reference's own ForwardEulerStruct(...) returns the B200 stepping struct under
# Backend = B200Backend(); against an unpatched reference the type is defined here.
if isdefined(DiplodocusTransport, :b200_stepping_struct)
    import DiplodocusTransport: B200Backend
else
    struct B200Backend <: BackendType end  # next to Backends.jl:3-4
end

const DTB_F64 = Int32(0)
const DTB_F32 = Int32(1)
const DTB_MIXED = Int32(2)
const DTB_FLAG_NO_AUTOTUNE = Int32(2)
const DTB_ENOTFOUND = Int32(7)

struct Dims
    n_species::Int32
    n_space::Int32
    species_size::NTuple{16,Int64}
end

struct Opts
    precision::Int32
    device::Int32
    stream::Ptr{Cvoid}
    index_base::Int32
    graph_steps::Int32
    dt0::Float64
    batch::Int32
    flags::Int32
end

mutable struct StepDiag
    cr::Float64
    cr_bin::Float64
    cr_emi::Float64
    cr_flux::Float64
    sum_df::Float64
    sum_f::Float64
    finite::Int32
    pad::Int32
end
StepDiag() = StepDiag(0, 0, 0, 0, 0, 0, 1, 0)

# Device-resident state: Solve's `@. method.f = method.f_init` (Solver.jl:22) uploads through
# dtb_set_f and `copyto!(f, method.f)` (Solver.jl:40) downloads through dtb_get_f.
mutable struct B200State <: AbstractVector{Float64}
    ctx::Ptr{Cvoid}
    n::Int
end
Base.size(v::B200State) = (v.n,)
Base.getindex(v::B200State, i::Int) = Base.copyto!(Vector{Float64}(undef, v.n), v)[i]
function Base.copyto!(dest::Vector{Float64}, src::B200State)
    GC.@preserve dest check(ccall((:dtb_get_f, libdtb), Int32, (Ptr{Cvoid}, Ptr{Float64}), src.ctx, dest))
    return dest
end
function Base.copyto!(dest::B200State, bc::Base.Broadcast.Broadcasted)
    v = Vector{Float64}(Base.materialize(bc))
    GC.@preserve v check(ccall((:dtb_set_f, libdtb), Int32, (Ptr{Cvoid}, Ptr{Float64}), dest.ctx, v))
    return dest
end
Base.BroadcastStyle(::Type{B200State}) = Base.Broadcast.DefaultArrayStyle{1}()

check(rc) = rc == 0 || error("libdtb: ", unsafe_string(ccall((:dtb_last_error, libdtb), Cstring, ())))

function upload_csc!(ctx, A::SparseMatrixCSC)
    nnz(A) == 0 && return
    nz = Float64.(A.nzval)
    GC.@preserve A nz check(ccall((:dtb_add_flux_csc, libdtb), Int32,
        (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}),
        ctx, size(A, 1), A.colptr, A.rowval, nz))
end

# The operators the step reads (SteppingStructs.jl:33-100), uploaded into a fresh context:
# F = X + P, M_Bin (dense or Bin_sparse), BinM.Domain, M_Emi, Ap, Vol, the initial state and
# the injection.
function upload_operators!(ctx::Ptr{Cvoid}, PhaseSpace::PhaseSpaceStruct, Initial::Vector{Float64},
                           Injection::Vector{Float64}, BinM, EmiM, FluxM)
    Momentum = PhaseSpace.Momentum
    sizes = Momentum.px_num_list .* Momentum.py_num_list .* Momentum.pz_num_list
    upload_csc!(ctx, FluxM.X_Flux)   # F = X + P (SteppingStructs.jl:60)
    upload_csc!(ctx, FluxM.P_Flux)
    n_mom = sum(sizes)
    if !isempty(BinM.Binary_list)
        if BinM.M_Bin isa SparseMatrixCSC   # Bin_sparse (BuildBinaryMatrices.jl:44-52), 1-based CSC
            S = SparseMatrixCSC{Float64,Int64}(BinM.M_Bin)
            GC.@preserve S check(ccall((:dtb_upload_mbin_csc, libdtb), Int32,
                                       (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}),
                                       ctx, n_mom, S.colptr, S.rowval, S.nzval))
        else
            M = Matrix{Float64}(BinM.M_Bin)
            GC.@preserve M check(ccall((:dtb_upload_mbin_ref, libdtb), Int32, (Ptr{Cvoid}, Ptr{Float64}, Int64),
                                       ctx, M, n_mom))
        end
        if !isnothing(BinM.Domain)   # Bin_Domain (SteppingStructs.jl:51, SteppingMethods.jl:369)
            D = Vector{Int64}(BinM.Domain)
            GC.@preserve D check(ccall((:dtb_set_bin_domain, libdtb), Int32, (Ptr{Cvoid}, Ptr{Int64}, Int64),
                                       ctx, D, length(D)))
        end
    end
    if !isempty(EmiM.Emission_list)
        E = Matrix{Float64}(EmiM.M_Emi)
        GC.@preserve E check(ccall((:dtb_upload_emi_ref, libdtb), Int32, (Ptr{Cvoid}, Ptr{Float64}, Int64),
                                   ctx, E, size(E, 1)))
    end
    Ap = Float64.(FluxM.Ap_Flux); Vol = Float64.(FluxM.Vol)
    GC.@preserve Ap Vol Initial Injection check(ccall((:dtb_upload_vectors, libdtb), Int32,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), ctx, Ap, Vol, Initial, Injection))
    return nothing
end

# The stepping struct of the B200 backend. Same constructor arguments as ForwardEulerStruct
# (SteppingStructs.jl:33) and the fields Solve reads (PhaseSpace, f_init, f).
mutable struct B200ForwardEulerStruct <: DiplodocusTransport.SteppingMethodType
    PhaseSpace::PhaseSpaceStruct
    dt0::Float64
    f_init::Vector{Float64}
    f::B200State
    ctx::Ptr{Cvoid}

    function B200ForwardEulerStruct(PhaseSpace::PhaseSpaceStruct, Initial::Vector{Float64}, Injection::Vector{Float64},
                                    BinM, EmiM, FluxM; Adaptive::Bool=false, device::Integer=0)
        Precision = getfield(Main, :Precision)
        Momentum = PhaseSpace.Momentum
        sizes = Momentum.px_num_list .* Momentum.py_num_list .* Momentum.pz_num_list
        ns = length(sizes)
        n_space = PhaseSpace.Space.x_num * PhaseSpace.Space.y_num * PhaseSpace.Space.z_num
        dims = Dims(ns, n_space, ntuple(i -> i <= ns ? Int64(sizes[i]) : Int64(0), 16))
        opts = Opts(Precision == Float32 ? DTB_F32 : DTB_F64, device, C_NULL, 1, 0, PhaseSpace.Time.dt0, 1, 0)  # graph_steps 0: the library's default
        ctx = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:dtb_create, libdtb), Int32, (Ref{Dims}, Ref{Opts}, Ref{Ptr{Cvoid}}), dims, opts, ctx))
        upload_operators!(ctx[], PhaseSpace, Initial, Injection, BinM, EmiM, FluxM)
        check(ccall((:dtb_commit, libdtb), Int32, (Ptr{Cvoid},), ctx[]))
        self = new(PhaseSpace, PhaseSpace.Time.dt0, copy(Initial), B200State(ctx[], length(Initial)), ctx[])
        finalizer(m -> ccall((:dtb_destroy, libdtb), Int32, (Ptr{Cvoid},), m.ctx), self)
        return self
    end
end

if isdefined(DiplodocusTransport, :b200_stepping_struct)
    DiplodocusTransport.b200_stepping_struct(args...; kw...) = B200ForwardEulerStruct(args...; kw...)
end

# The functor (SteppingMethods.jl:12-107): one ccall per step; dt truncation happens in the
# library exactly as in :18-23 and the diagnostics are printed like :87-93.
function (method::B200ForwardEulerStruct)(t_start, t_stop, dt, Verbose::Int64)
    dt_out = Ref{Float64}(0.0); save = Ref{Int32}(0); d = Ref(StepDiag())
    check(ccall((:dtb_step, libdtb), Int32,
        (Ptr{Cvoid}, Float64, Float64, Float64, Int32, Ref{Float64}, Ref{Int32}, Ref{StepDiag}),
        method.ctx, t_start, t_stop, dt, Verbose, dt_out, save, d))
    report_step(d[], Verbose, t_start, t_stop, dt_out[])
    return dt_out[], save[] != 0
end

# The functor with the state in a host vector: f is uploaded, stepped and overwritten with the
# new state, with one wait for the round trip (dtb_step_io).
function b200_step_io!(method::B200ForwardEulerStruct, f::Vector{Float64}, t_start, t_stop, dt, Verbose::Int64=0)
    dt_out = Ref{Float64}(0.0); save = Ref{Int32}(0); d = Ref(StepDiag())
    check(ccall((:dtb_step_io, libdtb), Int32,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Float64, Int32, Ref{Float64}, Ref{Int32},
         Ref{StepDiag}),
        method.ctx, f, f, t_start, t_stop, dt, Verbose, dt_out, save, d))
    report_step(d[], Verbose, t_start, t_stop, dt_out[])
    return dt_out[], save[] != 0
end

# SteppingMethods.jl:87-93
function report_step(d::StepDiag, Verbose, t_start, t_stop, dt)
    d.finite == 0 && println("non-finite value in df calculation")
    if Verbose == 1 && d.cr > 1.0
        println("Cr = $(d.cr), t=$t_start, dt=$dt, system may be unstable")
    elseif Verbose == 2
        println("\rCr = $(d.cr), t=$t_start, dt=$dt")
    elseif Verbose == 3
        println("Cr = $(d.cr),Cr_Bin = $(d.cr_bin), Cr_Emi = $(d.cr_emi), Cr_Flux = $(d.cr_flux), t=$t_start, t_save =$t_stop, dt=$dt")
    end
end

# Solve (Solver.jl:1-64) with each save interval replayed from CUDA graphs on the device.
function b200_solve(method::B200ForwardEulerStruct, dt_initial::Float64, t_save::Vector{Float64}; Verbose::Int64=1)
    n = length(method.f_init)
    F = Matrix{Float64}(undef, n, length(t_save))  # column i = state at t_save[i]
    nsteps = Ref{Int64}(0)
    check(ccall((:dtb_solve, libdtb), Int32,
        (Ptr{Cvoid}, Float64, Ptr{Float64}, Int64, Int32, Ptr{Float64}, Ref{Int64}),
        method.ctx, dt_initial, t_save, length(t_save), Verbose, F, nsteps))
    return F, nsteps[]
end

# Solve with the OutputStruct's FP64 number and energy moments (DistributionMoments.jl:33,145,162)
# of every saved state computed on the device; w: energy weight per momentum state. Returns the
# saved states, number and energy as [species, cell, save] arrays, and the step count.
function b200_solve(method::B200ForwardEulerStruct, dt_initial::Float64, t_save::Vector{Float64},
                    w::Vector{Float64}; Verbose::Int64=1)
    n = length(method.f_init)
    ns = length(method.PhaseSpace.Momentum.px_num_list)
    Sp = method.PhaseSpace.Space
    nsp = Sp.x_num * Sp.y_num * Sp.z_num
    F = Matrix{Float64}(undef, n, length(t_save))
    number = zeros(ns, nsp, length(t_save))
    energy = zeros(ns, nsp, length(t_save))
    nsteps = Ref{Int64}(0)
    check(ccall((:dtb_solve_ex, libdtb), Int32,
        (Ptr{Cvoid}, Float64, Ptr{Float64}, Int64, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ref{Int64}),
        method.ctx, dt_initial, t_save, length(t_save), Verbose, F, w, number, energy, nsteps))
    return F, number, energy, nsteps[]
end

# ---------------------------------------------------------------- batched solves
# Many independent solves of one grid (a parameter scan over initial spectra and time steps)
# in one batched context: the shared G, stored as BF16 hi + lo with per-row scales, is
# contracted against every slot's f1 (x) f2 by one tensor-core GEMM per step, f is FP32 with an
# FP32 compensation term and the update is FP64. Slots are 1-based here; states go in and out
# as n_state x capacity matrices (column s = slot s).
mutable struct B200BatchedEuler
    ctx::Ptr{Cvoid}
    n::Int
    capacity::Int
    dt0::Float64
    n_species::Int
    n_space::Int

    function B200BatchedEuler(PhaseSpace::PhaseSpaceStruct, Injection::Vector{Float64}, BinM, EmiM, FluxM,
                              capacity::Integer; device::Integer=0, autotune::Bool=true)
        Momentum = PhaseSpace.Momentum
        sizes = Momentum.px_num_list .* Momentum.py_num_list .* Momentum.pz_num_list
        ns = length(sizes)
        n_space = PhaseSpace.Space.x_num * PhaseSpace.Space.y_num * PhaseSpace.Space.z_num
        dims = Dims(ns, n_space, ntuple(i -> i <= ns ? Int64(sizes[i]) : Int64(0), 16))
        opts = Opts(DTB_MIXED, device, C_NULL, 1, 16, PhaseSpace.Time.dt0, Int32(capacity),
                    autotune ? Int32(0) : DTB_FLAG_NO_AUTOTUNE)
        ctx = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:dtb_create, libdtb), Int32, (Ref{Dims}, Ref{Opts}, Ref{Ptr{Cvoid}}), dims, opts, ctx))
        n = length(Injection)
        upload_operators!(ctx[], PhaseSpace, zeros(n), Injection, BinM, EmiM, FluxM)
        check(ccall((:dtb_commit, libdtb), Int32, (Ptr{Cvoid},), ctx[]))  # plans (autotunes) the gain GEMM
        self = new(ctx[], n, Int(capacity), PhaseSpace.Time.dt0, ns, n_space)
        finalizer(b -> ccall((:dtb_destroy, libdtb), Int32, (Ptr{Cvoid},), b.ctx), self)
        return self
    end
end

# Starts a solve in `slot`: f = f0, step dt (dt/dt0 is applied as in SteppingMethods.jl:27),
# n_steps steps from the current batched step.
admit!(b::B200BatchedEuler, slot::Integer, f0::Vector{Float64}, dt::Float64, n_steps::Integer) =
    check(ccall((:dtb_batch_admit, libdtb), Int32, (Ptr{Cvoid}, Int32, Ptr{Float64}, Float64, Int64),
                b.ctx, slot - 1, f0, dt / b.dt0, n_steps))

# Captures and uploads the step graphs now, so the first run!/b200_solve pays no capture.
prepare!(b::B200BatchedEuler) = check(ccall((:dtb_prepare, libdtb), Int32, (Ptr{Cvoid},), b.ctx))
prepare!(m::B200ForwardEulerStruct) = check(ccall((:dtb_prepare, libdtb), Int32, (Ptr{Cvoid},), m.ctx))

# nsteps batched steps of every slot with steps left (enqueued; errors surface at the next read).
run!(b::B200BatchedEuler, nsteps::Integer) =
    check(ccall((:dtb_batch_run, libdtb), Int32, (Ptr{Cvoid}, Int64), b.ctx, nsteps))

function get_f(b::B200BatchedEuler, slot::Integer)
    f = Vector{Float64}(undef, b.n)
    check(ccall((:dtb_batch_get_f, libdtb), Int32, (Ptr{Cvoid}, Int32, Ptr{Float64}), b.ctx, slot - 1, f))
    return f
end

# The whole batch in, nsteps steps, the whole batch out, under one wait. F_in === nothing keeps
# the device state; F_out may be F_in.
function run_io!(b::B200BatchedEuler, F_in::Union{Nothing,Matrix{Float64}}, nsteps::Integer,
                 F_out::Matrix{Float64}=Matrix{Float64}(undef, b.n, b.capacity))
    @assert size(F_out) == (b.n, b.capacity)
    pin = F_in === nothing ? C_NULL : pointer(F_in)
    GC.@preserve F_in F_out check(ccall((:dtb_batch_run_io, libdtb), Int32,
                                        (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}), b.ctx, pin, nsteps, F_out))
    return F_out
end

# FP64 number and energy of every (species, cell, slot) (DistributionMoments.jl:33,145,162);
# w: energy weight per momentum state.
function batch_moments(b::B200BatchedEuler, w::Vector{Float64})
    number = zeros(b.n_species, b.n_space, b.capacity)
    energy = zeros(b.n_species, b.n_space, b.capacity)
    check(ccall((:dtb_batch_moments, libdtb), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                b.ctx, w, number, energy))
    return number, energy
end

# The gain-GEMM plan of gain group `group` (1-based), or nothing past the last group.
function gemm_plan(b::B200BatchedEuler, group::Integer=1)
    pair = Ref{Int32}(0); bn = Ref{Int32}(0); ns = Ref{Int32}(0); us = Ref{Float64}(0)
    rc = ccall((:dtb_batch_gemm_plan, libdtb), Int32,
               (Ptr{Cvoid}, Int32, Ref{Int32}, Ref{Int32}, Ref{Int32}, Ref{Float64}), b.ctx, group - 1, pair, bn, ns, us)
    rc == DTB_ENOTFOUND && return nothing
    check(rc)
    return (pair=pair[] != 0, bn=Int(bn[]), n_splits=Int(ns[]), tuned_us=us[])
end

# Plans measured in earlier runs are reused from `path`, new ones appended (nothing: forget).
set_tune_cache(path::Union{Nothing,AbstractString}) =
    check(ccall((:dtb_set_tune_cache, libdtb), Int32, (Cstring,), path === nothing ? C_NULL : path))

# ---------------------------------------------------------------- serving
# Continuous batching of solve requests (each a Solve of n_steps steps from its own f0 and dt):
# a library-owned host thread admits queued requests into free slots of their grid's batched
# context as slots free up, runs every grid on its own stream and reads finished requests back.
# Grids are batched contexts (B200BatchedEuler) registered against an HBM budget; the server
# drives them until it is closed, and the caller closes them afterwards.
struct ServeOpts
    hbm_budget_bytes::Int64
    max_chunk_steps::Int32
    flags::Int32
    chunk_ms::Float64
end

struct RequestStats
    t_submit::Float64
    t_admit::Float64
    t_done::Float64
    steps::Int64
    cr_max::Float64
    finite::Int32
    grid::Int32
end

struct ServeStats
    completed::Int64
    instance_steps::Int64
    batched_steps::Int64
    queued::Int64
    running::Int64
    device_bytes::Int64
    busy_s::Float64
    elapsed_s::Float64
end

mutable struct B200Server
    srv::Ptr{Cvoid}
    grids::Vector{B200BatchedEuler}
    function B200Server(; hbm_budget_bytes::Integer=0, max_chunk_steps::Integer=0, chunk_ms::Real=0.0)
        opts = ServeOpts(Int64(hbm_budget_bytes), Int32(max_chunk_steps), Int32(0), Float64(chunk_ms))
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:dtb_serve_create, libdtb), Int32, (Ref{ServeOpts}, Ref{Ptr{Cvoid}}), opts, out))
        self = new(out[], B200BatchedEuler[])
        finalizer(close, self)
        return self
    end
end

# Registers a committed batched context as a grid; returns its grid id (DTB_ENOMEM past the budget).
function add_grid!(s::B200Server, b::B200BatchedEuler)
    id = Ref{Int32}(0)
    check(ccall((:dtb_serve_add_grid, libdtb), Int32, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Int32}), s.srv, b.ctx, id))
    push!(s.grids, b)
    return Int(id[])
end

start!(s::B200Server) = check(ccall((:dtb_serve_start, libdtb), Int32, (Ptr{Cvoid},), s.srv))

# Queues a solve of n_steps steps from f0 with dt (dt/dt0 applied by the caller, as the
# functor's dt_scale); returns the request id. Thread-safe.
function submit!(s::B200Server, grid::Integer, f0::Vector{Float64}, dt_scale::Float64, n_steps::Integer)
    id = Ref{Int64}(0)
    GC.@preserve f0 check(ccall((:dtb_serve_submit, libdtb), Int32,
                                (Ptr{Cvoid}, Int32, Ptr{Float64}, Float64, Int64, Ref{Int64}),
                                s.srv, grid, f0, dt_scale, n_steps, id))
    return id[]
end

# Waits for a request (timeout in seconds, <= 0: no limit) and returns its final f and timings.
function wait_request(s::B200Server, id::Integer, n_state::Integer; timeout_s::Real=0.0)
    f = Vector{Float64}(undef, n_state)
    st = Ref{RequestStats}()
    check(ccall((:dtb_serve_wait, libdtb), Int32, (Ptr{Cvoid}, Int64, Float64, Ptr{Float64}, Ref{RequestStats}),
                s.srv, id, timeout_s, f, st))
    return f, st[]
end

cancel!(s::B200Server, id::Integer) = check(ccall((:dtb_serve_cancel, libdtb), Int32, (Ptr{Cvoid}, Int64), s.srv, id))

function serve_stats(s::B200Server)
    st = Ref{ServeStats}()
    check(ccall((:dtb_serve_get_stats, libdtb), Int32, (Ptr{Cvoid}, Ref{ServeStats}), s.srv, st))
    return st[]
end

function Base.close(s::B200Server)
    if s.srv != C_NULL
        ccall((:dtb_serve_destroy, libdtb), Int32, (Ptr{Cvoid},), s.srv)
        s.srv = C_NULL
    end
    return nothing
end

end # module
