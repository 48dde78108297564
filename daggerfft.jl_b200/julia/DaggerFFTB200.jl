"""
    DaggerFFTB200

Julia front end over libdfft (include/dfft.h) for CuArrays: the README API of
DaggerFFT.jl (`fft`, `ifft`, `rfft`, `irfft` with `decomp`, `transforms`,
`dims`, plus in-place `fft!` / `ifft!` and the `method = :mixed` tensor-core
form), the plan-level `apply_gpu_fft!`, the DArray-level drivers
`create_gpu_workspace` / `gpu_fft!` / `gpu_ifft!` / `gpu_cleanup_workspace!`
over chunked arrays, batches of uneven transforms (`Batch`), the tuning cache
(`wisdom_export` / `wisdom_import`), and the serving loop (`Server`,
`submit`, `serve`), all executed by hand-written sm_100a kernels.  Arrays are
used in Julia's own column-major layout; every call runs on the CuArray's
task-local stream.

This file is the binding a maintainer would add to DaggerFFT.jl; it is not
exercised in this repository's CI (no Julia toolchain), the C ABI it binds is
(tests/ drive the same entry points through ctypes).
"""
module DaggerFFTB200

using CUDA

const libdfft = joinpath(@__DIR__, "..", "lib", "libdfft.so")

# ---- tags (src/fft.jl:13-24) ----------------------------------------------
abstract type Decomposition end
struct Pencil <: Decomposition end
struct Slab <: Decomposition end
code(::Pencil) = Cint(0)
code(::Slab) = Cint(1)

struct FFT end; struct IFFT end; struct RFFT end; struct IRFFT end
struct FFT! end; struct IFFT! end; struct RFFT! end; struct IRFFT! end
struct R2R{N}
    kinds::NTuple{N,Int}
end
code(::FFT) = Cint(0); code(::IFFT) = Cint(1); code(::RFFT) = Cint(2); code(::IRFFT) = Cint(3)
code(::FFT!) = Cint(4); code(::IFFT!) = Cint(5); code(::RFFT!) = Cint(6); code(::IRFFT!) = Cint(7)
code(::R2R) = Cint(8)

# FFTW r2r kind values
# plan flags (dfft.h)
const FLAG_DESTROY_INPUT = Cuint(1); const FLAG_TUNE = Cuint(2); const FLAG_NO_WISDOM = Cuint(4)
const FLAG_NO_FUSE = Cuint(8); const FLAG_FUSE = Cuint(16)
const DHT = 2; const REDFT00 = 3; const REDFT01 = 4; const REDFT10 = 5; const REDFT11 = 6
const RODFT00 = 7; const RODFT01 = 8; const RODFT10 = 9; const RODFT11 = 10

method_code(m::Symbol) = m === :plain ? Cint(0) : m === :mixed ? Cint(1) :
    throw(ArgumentError("method must be :plain or :mixed"))
method_code(m::Integer) = Cint(m)

precision_code(::Type{<:Union{Float32,ComplexF32}}) = Cint(0)
precision_code(::Type{<:Union{Float64,ComplexF64}}) = Cint(1)

function check(st::Cint)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:dfft_last_error, libdfft), Cstring, ()))
    st in (1, 2, 3) && throw(ArgumentError(msg))   # "Unknown transform type" for 2
    error("libdfft: " * msg)
end

mutable struct Plan
    h::Ptr{Cvoid}
    outsize::Tuple
    function Plan(h, outsize)
        p = new(h, outsize)
        finalizer(p) do q
            q.h != C_NULL && ccall((:dfft_plan_destroy, libdfft), Cint, (Ptr{Cvoid},), q.h)
            q.h = C_NULL
        end
        p
    end
end

# plan cache keyed like GPU_PLAN_CACHE (src/fftgpu.jl:83-116)
const GPU_PLAN_CACHE = Dict{Any,Plan}()

function plan_transform(transform, A::CuArray, dims; decomp=Pencil(), n=0, method=:plain, flags=0)
    dims_t = dims isa Tuple ? dims : (dims,)
    key = (eltype(A), size(A), typeof(transform), dims_t, decomp, n, method, flags)
    get!(GPU_PLAN_CACHE, key) do
        shape = Int64[size(A)...]
        d = Int32[dims_t...]
        kinds = transform isa R2R ? Int32[transform.kinds...] : Int32[0]
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:dfft_plan_create, libdfft), Cint,
                    (Ptr{Ptr{Cvoid}}, Cint, Ptr{Int64}, Cint, Cint, Cint, Ptr{Int32}, Ptr{Int32},
                     Int64, Cint, Cint, Cuint),
                    h, ndims(A), shape, precision_code(eltype(A)), code(transform), length(d), d,
                    kinds, Int64(n), code(decomp), method_code(method), Cuint(flags)))
        out = zeros(Int64, ndims(A))
        check(ccall((:dfft_plan_output_shape, libdfft), Cint, (Ptr{Cvoid}, Ptr{Int64}), h[], out))
        Plan(h[], Tuple(out))
    end
end

"One line per kernel launch of a plan (`dfft_plan_describe`)."
function describe(p::Plan)
    buf = Vector{UInt8}(undef, 8192)
    check(ccall((:dfft_plan_describe, libdfft), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), p.h, buf, length(buf)))
    unsafe_string(pointer(buf))
end

function execute!(p::Plan, out::CuArray, in::CuArray)
    check(ccall((:dfft_execute, libdfft), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}),
                p.h, in, out, CUDA.stream().handle))
    out
end

"""
    slab_split_plan(T, L, nslab, zr, nranks; inverse=false, split_dim=1)

The fused 2-D slab pass of a distributed Slab transform with the pack and
unpack of the exchange folded in (`dfft_slab_split_create`): forward writes
each rank's columns (split_dim 1, the Blocks(L, L, c) -> Blocks(c, L, N3)
layouts) or rows (split_dim 2) of every local slab as one contiguous block
(the message to that rank), inverse reads the received blocks.  Run slab
groups with `execute_split!` at element offsets; the blocks then go out
with `MPI.Isend`/`MPI.Irecv!` and the received chunk takes a dims-3 plan.
With split_dim 1 the forward overwrites its input, as the in-place slab
stage does.
"""
function slab_split_plan(::Type{T}, L::Integer, nslab::Integer, zr::Integer, nranks::Integer;
                         inverse::Bool=false, split_dim::Integer=1) where {T}
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:dfft_slab_split_create, libdfft), Cint,
                (Ptr{Ptr{Cvoid}}, Cint, Cint, Int64, Int64, Int64, Cint, Cint, Cuint),
                h, precision_code(T), inverse ? Cint(1) : Cint(0), Int64(L), Int64(nslab), Int64(zr),
                Cint(nranks), Cint(split_dim), Cuint(0)))
    out = zeros(Int64, 3)
    check(ccall((:dfft_plan_output_shape, libdfft), Cint, (Ptr{Cvoid}, Ptr{Int64}), h[], out))
    Plan(h[], Tuple(out))
end

"Run a split slab plan from `in` (element offset `ioff`) to `out` (offset `ooff`)."
function execute_split!(p::Plan, out::CuArray{T}, ooff::Integer, in::CuArray{T}, ioff::Integer) where {T}
    check(ccall((:dfft_execute, libdfft), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}),
                p.h, pointer(in) + ioff * sizeof(T), pointer(out) + ooff * sizeof(T), CUDA.stream().handle))
    out
end

"`apply_gpu_fft!(out, in, transform, dim)`: plan lookup + execute (src/fftgpu.jl:118-124)."
function apply_gpu_fft!(out, in, transform, dim; kw...)
    execute!(plan_transform(transform, in, dim; kw...), out, in)
end

cplx(::Type{Float32}) = ComplexF32
cplx(::Type{Float64}) = ComplexF64
realt(::Type{ComplexF32}) = Float32
realt(::Type{ComplexF64}) = Float64

function fft(A::CuArray; decomp=Pencil(), dims=(1, 2, 3), transforms=nothing, method=:plain)
    if transforms !== nothing && first(transforms) isa R2R
        p = plan_transform(first(transforms), A, dims; decomp)
        return execute!(p, similar(A, p.outsize), A)
    end
    B = eltype(A) <: Complex ? A : CuArray{cplx(eltype(A))}(A)
    p = plan_transform(FFT(), B, dims; decomp, method)
    execute!(p, similar(B, p.outsize), B)
end

function ifft(A::CuArray; decomp=Pencil(), dims=(1, 2, 3), transforms=nothing, method=:plain)
    if transforms !== nothing && first(transforms) isa R2R
        p = plan_transform(first(transforms), A, dims; decomp)
        return execute!(p, similar(A, p.outsize), A)
    end
    p = plan_transform(IFFT(), A, dims; decomp, method)
    execute!(p, similar(A, p.outsize), A)
end

"In-place `fft!(A; decomp, dims, transforms, method)`: `A` is overwritten with its transform."
function fft!(A::CuArray{<:Complex}; decomp=Pencil(), dims=(1, 2, 3), transforms=nothing, method=:plain)
    t = (transforms !== nothing && first(transforms) isa R2R) ? first(transforms) : FFT!()
    execute!(plan_transform(t, A, dims; decomp, method), A, A)
end
function fft!(A::CuArray{<:Real}; decomp=Pencil(), dims=(1, 2, 3), transforms)
    execute!(plan_transform(first(transforms), A, dims; decomp), A, A)
end

"In-place `ifft!(A; decomp, dims, method)` (scaled by 1/prod(size(A, dims)))."
function ifft!(A::CuArray{<:Complex}; decomp=Pencil(), dims=(1, 2, 3), method=:plain)
    execute!(plan_transform(IFFT!(), A, dims; decomp, method), A, A)
end

function rfft(A::CuArray{<:Real}; decomp=Pencil(), dims=(1, 2, 3))
    p = plan_transform(RFFT(), A, dims; decomp)
    execute!(p, CuArray{cplx(eltype(A))}(undef, p.outsize), A)
end

function irfft(F::CuArray{<:Complex}, d::Integer; decomp=Pencil(), dims=(1, 2, 3))
    p = plan_transform(IRFFT(), F, dims; decomp, n=d)
    execute!(p, CuArray{realt(eltype(F))}(undef, p.outsize), F)
end

# ---- tuning cache (FFTW wisdom analogue, src/fft.jl:113-124,162) -----------
wisdom_export(path::AbstractString) = check(ccall((:dfft_wisdom_export, libdfft), Cint, (Cstring,), path))
wisdom_import(path::AbstractString) = check(ccall((:dfft_wisdom_import, libdfft), Cint, (Cstring,), path))
wisdom_forget() = check(ccall((:dfft_wisdom_forget, libdfft), Cint, ()))
function wisdom_size()
    n = Ref{Cint}(0)
    check(ccall((:dfft_wisdom_size, libdfft), Cint, (Ref{Cint},), n))
    Int(n[])
end

"Reads and clears the device error word (0: no kernel gave up a bounded wait)."
function device_error()
    c = Ref{Cint}(0)
    check(ccall((:dfft_device_error, libdfft), Cint, (Ref{Cint},), c))
    Int(c[])
end

# ---- batches of uneven transforms (one CUDA graph launch, or one launch of
# the persistent batch kernel with `persistent = true`) ----------------------
const BATCH_PERSISTENT = Cuint(1) << 1

mutable struct Batch
    h::Ptr{Cvoid}
    plans::Vector{Plan}   # kept alive as long as the batch
    function Batch(plans::Vector{Plan}; persistent::Bool = false, lag::Integer = 0)
        0 <= lag <= 255 || throw(ArgumentError("lag must be in 0..255"))
        h = Ref{Ptr{Cvoid}}(C_NULL)
        hs = Ptr{Cvoid}[p.h for p in plans]
        flags = (persistent ? BATCH_PERSISTENT : Cuint(0)) | (Cuint(lag) << 8)
        check(ccall((:dfft_batch_create_ex, libdfft), Cint,
                    (Ptr{Ptr{Cvoid}}, Cint, Ptr{Ptr{Cvoid}}, Cuint), h, length(hs), hs, flags))
        b = new(h[], plans)
        finalizer(b) do q
            q.h != C_NULL && ccall((:dfft_batch_destroy, libdfft), Cint, (Ptr{Cvoid},), q.h)
            q.h = C_NULL
        end
        b
    end
end

function launches(b::Batch)
    n = Ref{Cint}(0)
    check(ccall((:dfft_batch_launches, libdfft), Cint, (Ptr{Cvoid}, Ref{Cint}), b.h, n))
    Int(n[])
end

"Runs every plan of the batch, `outs[i] = T_i(ins[i])`, as one graph launch."
function execute!(b::Batch, outs::Vector{<:CuArray}, ins::Vector{<:CuArray})
    length(outs) == length(ins) == length(b.plans) || throw(ArgumentError("one input and output per plan"))
    ip = CuPtr{Cvoid}[pointer(x) for x in ins]
    op = CuPtr{Cvoid}[pointer(x) for x in outs]
    check(ccall((:dfft_batch_execute, libdfft), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Ptr{CuPtr{Cvoid}}, Ptr{Cvoid}),
                b.h, ip, op, CUDA.stream().handle))
    outs
end

# ---- serving: continuous batching with HBM-budget admission -----------------
const MEM_DEVICE = Cint(0); const MEM_HOST = Cint(1); const MEM_SERVER = Cint(2)

# layout of dfft_request (include/dfft.h)
struct DfftRequest
    transform::Cint
    precision::Cint
    decomp::Cint
    ndim::Cint
    shape::NTuple{3,Int64}
    ndims::Cint
    dims::NTuple{3,Int32}
    r2r_kinds::NTuple{3,Int32}
    irfft_len::Int64
    in::Ptr{Cvoid}
    in_location::Cint
    out::Ptr{Cvoid}
    out_location::Cint
end

# layout of dfft_server_stats
struct DfftServerStats
    completed::UInt64
    rejected::UInt64
    cancelled::UInt64
    failed::UInt64
    queued::UInt64
    p50_ms::Cdouble
    p99_ms::Cdouble
    max_ms::Cdouble
    bytes_moved::Cdouble
    elapsed_s::Cdouble
    arena_bytes::Csize_t
    arena_peak_bytes::Csize_t
    peak_running::Cint
    resident_plans::Cint
end

mutable struct Server
    h::Ptr{Cvoid}
    pinned::Dict{UInt64,Any}   # inputs / outputs of requests in flight
    function Server(hbm_budget_bytes::Integer; slots::Integer=8, flags::Integer=0)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:dfft_server_create, libdfft), Cint, (Ptr{Ptr{Cvoid}}, Csize_t, Cint, Cuint),
                    h, hbm_budget_bytes, slots, flags))
        s = new(h[], Dict{UInt64,Any}())
        finalizer(close, s)
        s
    end
end

function Base.close(s::Server)
    s.h != C_NULL && ccall((:dfft_server_destroy, libdfft), Cint, (Ptr{Cvoid},), s.h)
    s.h = C_NULL
    empty!(s.pinned)
    nothing
end

"""
    submit(s, transform, A; dims, decomp, n, out) -> id

Queues one transform request.  `A` is a CuArray (device input) or an Array
(host input, copied in by the server); the result goes to `out` (a CuArray
or Array of the output size) or, when `out === nothing`, stays in the
server's arena until `fetch`/`release`.
"""
function submit(s::Server, transform, A::AbstractArray; dims=ntuple(identity, ndims(A)),
                decomp=Pencil(), n=0, out=nothing)
    dims_t = dims isa Tuple ? dims : (dims,)
    kinds = transform isa R2R ? transform.kinds : ()
    pad3(t, T, fill) = ntuple(i -> i <= length(t) ? T(t[i]) : T(fill), 3)
    inloc = A isa CuArray ? MEM_DEVICE : MEM_HOST
    outloc = out === nothing ? MEM_SERVER : out isa CuArray ? MEM_DEVICE : MEM_HOST
    ptr(x) = x === nothing ? C_NULL : x isa CuArray ? reinterpret(Ptr{Cvoid}, pointer(x)) :
             Ptr{Cvoid}(pointer(x))
    req = DfftRequest(code(transform), precision_code(eltype(A)), code(decomp), Cint(ndims(A)),
                      pad3(size(A), Int64, 1), Cint(length(dims_t)), pad3(dims_t, Int32, 0),
                      pad3(kinds, Int32, 0), Int64(n), ptr(A), inloc, ptr(out), outloc)
    id = Ref{UInt64}(0)
    check(ccall((:dfft_server_submit, libdfft), Cint, (Ptr{Cvoid}, Ref{DfftRequest}, Ref{UInt64}),
                s.h, req, id))
    s.pinned[id[]] = (A, out)
    id[]
end

"Ids of finished requests, oldest first."
function poll(s::Server; max::Integer=256)
    ids = Vector{UInt64}(undef, max)
    n = Ref{Cint}(0)
    check(ccall((:dfft_server_poll, libdfft), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Cint, Ref{Cint}),
                s.h, ids, max, n))
    ids[1:n[]]
end

"Bounded wait for request `id`; throws on timeout or on the request's own failure."
function Base.wait(s::Server, id::UInt64; timeout_ms::Integer=60_000)
    st = Ref{Cint}(0)
    check(ccall((:dfft_server_wait, libdfft), Cint, (Ptr{Cvoid}, UInt64, Cint, Ref{Cint}),
                s.h, id, timeout_ms, st))
    check(st[])
    nothing
end

"Copies a server-held result to `dst` (CuArray or Array)."
function Base.fetch(s::Server, id::UInt64, dst::AbstractArray)
    loc = dst isa CuArray ? MEM_DEVICE : MEM_HOST
    p = dst isa CuArray ? reinterpret(Ptr{Cvoid}, pointer(dst)) : Ptr{Cvoid}(pointer(dst))
    check(ccall((:dfft_server_fetch, libdfft), Cint, (Ptr{Cvoid}, UInt64, Ptr{Cvoid}, Cint, Ptr{Cvoid}),
                s.h, id, p, loc, CUDA.stream().handle))
    dst
end

function release(s::Server, id::UInt64)
    check(ccall((:dfft_server_release, libdfft), Cint, (Ptr{Cvoid}, UInt64), s.h, id))
    delete!(s.pinned, id)
    nothing
end

cancel(s::Server, id::UInt64) = check(ccall((:dfft_server_cancel, libdfft), Cint, (Ptr{Cvoid}, UInt64), s.h, id))

function stats(s::Server)
    st = Ref{DfftServerStats}()
    check(ccall((:dfft_server_get_stats, libdfft), Cint, (Ptr{Cvoid}, Ref{DfftServerStats}), s.h, st))
    st[]
end

reset_stats!(s::Server) = check(ccall((:dfft_server_reset_stats, libdfft), Cint, (Ptr{Cvoid},), s.h))

"""
    serve(s, requests) -> results

The request loop: `requests` is an iterable (a Channel, for a live stream)
of `(transform, A, kwargs)` tuples; each is submitted as it arrives, finished
requests are retired while later ones are still arriving, and the results
(host arrays, in submission order) are returned once the stream ends.
Latency percentiles are in `stats(s)`.
"""
function serve(s::Server, requests)
    ids = UInt64[]
    outs = Dict{UInt64,Any}()
    for (transform, A, kw) in requests
        out = Array{eltype_out(transform, eltype(A))}(undef, outsize(transform, A; kw...))
        id = submit(s, transform, A; out=out, kw...)
        push!(ids, id)
        outs[id] = out
        for done in poll(s)   # retire what finished meanwhile
            release(s, done)
        end
    end
    for id in ids
        haskey(s.pinned, id) || continue
        wait(s, id)
        release(s, id)
    end
    [outs[id] for id in ids]
end

eltype_out(::Union{RFFT,RFFT!}, T) = cplx(T)
eltype_out(::Union{IRFFT,IRFFT!}, T) = realt(T)
eltype_out(_, T) = T
function outsize(transform, A; dims=ntuple(identity, ndims(A)), n=0, kw...)
    sz = collect(size(A))
    d1 = first(dims isa Tuple ? dims : (dims,))
    transform isa Union{RFFT,RFFT!} && (sz[d1] = sz[d1] ÷ 2 + 1)
    transform isa Union{IRFFT,IRFFT!} && (sz[d1] = n)
    Tuple(sz)
end

# ---- DArray level: chunked arrays, workspaces, Pencil / Slab drivers --------
#
# A `ChunkedArray` is the GPU-side view of a Dagger DArray: the block
# subdomains (column-major chunk order), the rank owning each chunk and this
# rank's CuArray chunks.  `create_gpu_workspace` walks dst chunks (outer) x
# src chunks (inner) like src/fftgpu.jl:126-318 and compiles the local
# copies, the packing of every send and the unpacking of every receive into
# three libdfft copy plans (one launch each); the exchange between ranks is
# MPI point-to-point on the flat buffers (CUDA-aware MPI), as the reference's.

struct ChunkedArray{T}
    shape::NTuple{3,Int}
    subdomains::Vector{NTuple{3,UnitRange{Int}}}
    owner::Vector{Int}
    chunks::Vector{Union{Nothing,CuArray{T,3}}}
    rank::Int
end

"`distribute(A, blocks; rank, nranks)`: this rank's chunks of `A` in `Blocks(b1,b2,b3)`."
function distribute(A::AbstractArray{T,3}, blocks::NTuple{3,Int}; rank=0, nranks=1) where {T}
    doms = NTuple{3,UnitRange{Int}}[]
    nb = cld.(size(A), blocks)
    for kz in 1:nb[3], ky in 1:nb[2], kx in 1:nb[1]
        push!(doms, ntuple(d -> ((kx, ky, kz)[d]-1)*blocks[d]+1:min((kx, ky, kz)[d]*blocks[d], size(A, d)), 3))
    end
    owner = [(i - 1) % nranks for i in eachindex(doms)]
    chunks = Union{Nothing,CuArray{T,3}}[owner[i] == rank ? CuArray(A[doms[i]...]) : nothing
                                         for i in eachindex(doms)]
    ChunkedArray{T}(size(A), doms, owner, chunks, rank)
end

similar_chunked(D::ChunkedArray{T}, blocks) where {T} =
    distribute_empty(T, D.shape, blocks; rank=D.rank, nranks=maximum(D.owner) + 1)
function distribute_empty(::Type{T}, shape, blocks; rank=0, nranks=1) where {T}
    Z = ChunkedArray{T}(shape, NTuple{3,UnitRange{Int}}[], Int[], Union{Nothing,CuArray{T,3}}[], rank)
    nb = cld.(shape, blocks)
    for kz in 1:nb[3], ky in 1:nb[2], kx in 1:nb[1]
        d = ntuple(i -> ((kx, ky, kz)[i]-1)*blocks[i]+1:min((kx, ky, kz)[i]*blocks[i], shape[i]), 3)
        push!(Z.subdomains, d)
        push!(Z.owner, (length(Z.owner)) % nranks)
        push!(Z.chunks, Z.owner[end] == rank ? CuArray{T}(undef, length.(d)) : nothing)
    end
    Z
end

# layout of dfft_block_copy
struct DfftBlockCopy
    src::Ptr{Cvoid}
    dst::Ptr{Cvoid}
    src_start::NTuple{3,Int64}
    dst_start::NTuple{3,Int64}
    src_dims::NTuple{3,Int64}
    dst_dims::NTuple{3,Int64}
    count::NTuple{3,Int64}
end

mutable struct CopyPlan
    h::Ptr{Cvoid}
    function CopyPlan(blocks::Vector{DfftBlockCopy}, elsize::Integer)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:dfft_copy_plan_create, libdfft), Cint, (Ptr{Ptr{Cvoid}}, Ptr{DfftBlockCopy}, Cint, Cint),
                    h, blocks, length(blocks), elsize))
        c = new(h[])
        finalizer(c) do q
            q.h != C_NULL && ccall((:dfft_copy_plan_destroy, libdfft), Cint, (Ptr{Cvoid},), q.h)
            q.h = C_NULL
        end
        c
    end
end
run!(c::CopyPlan) = check(ccall((:dfft_copy_plan_execute, libdfft), Cint, (Ptr{Cvoid}, Ptr{Cvoid}),
                                c.h, CUDA.stream().handle))

"The overlap of two subdomains (src/fft.jl:176-178)."
compute_overlap(a::NTuple{3,UnitRange{Int}}, b::NTuple{3,UnitRange{Int}}) =
    ntuple(d -> max(first(a[d]), first(b[d])):min(last(a[d]), last(b[d])), 3)

mutable struct GPUWorkspace{T}
    local_copies::CopyPlan
    pack::Union{Nothing,CopyPlan}
    unpack::Union{Nothing,CopyPlan}
    send_buffer::Union{Nothing,CuVector{T}}
    recv_buffer::Union{Nothing,CuVector{T}}
    send_ranks::Vector{Int}; send_sizes::Vector{Int}
    recv_ranks::Vector{Int}; recv_sizes::Vector{Int}
end

function create_gpu_workspace(src::ChunkedArray{T}, dst::ChunkedArray{T}) where {T}
    rank = src.rank
    loc = DfftBlockCopy[]
    sendp = Dict{Int,Vector{Any}}(); recvp = Dict{Int,Vector{Any}}()
    vp(x) = x === nothing ? C_NULL : reinterpret(Ptr{Cvoid}, pointer(x))
    for (di, dd) in enumerate(dst.subdomains), (si, sd) in enumerate(src.subdomains)
        ov = compute_overlap(sd, dd)
        any(isempty, ov) && continue
        s0 = ntuple(d -> first(ov[d]) - first(sd[d]), 3)
        d0 = ntuple(d -> first(ov[d]) - first(dd[d]), 3)
        cnt = ntuple(d -> length(ov[d]), 3)
        sr, dr = src.owner[si], dst.owner[di]
        if sr == rank && dr == rank
            push!(loc, DfftBlockCopy(vp(src.chunks[si]), vp(dst.chunks[di]), s0, d0,
                                     size(src.chunks[si]), size(dst.chunks[di]), cnt))
        elseif sr == rank
            push!(get!(sendp, dr, Any[]), (si, s0, cnt))
        elseif dr == rank
            push!(get!(recvp, sr, Any[]), (di, d0, cnt))
        end
    end
    sranks = sort!(collect(keys(sendp))); rranks = sort!(collect(keys(recvp)))
    ssz = [sum(prod(p[3]) for p in sendp[r]) for r in sranks]
    rsz = [sum(prod(p[3]) for p in recvp[r]) for r in rranks]
    sbuf = isempty(sranks) ? nothing : CuVector{T}(undef, sum(ssz))
    rbuf = isempty(rranks) ? nothing : CuVector{T}(undef, sum(rsz))
    pk = DfftBlockCopy[]; off = 0
    for r in sranks, (si, s0, cnt) in sendp[r]     # x-fastest flat blocks in walk order
        push!(pk, DfftBlockCopy(vp(src.chunks[si]), vp(sbuf) + off * sizeof(T), s0, (0, 0, 0),
                                size(src.chunks[si]), cnt, cnt))
        off += prod(cnt)
    end
    up = DfftBlockCopy[]; off = 0
    for r in rranks, (di, d0, cnt) in recvp[r]
        push!(up, DfftBlockCopy(vp(rbuf) + off * sizeof(T), vp(dst.chunks[di]), (0, 0, 0), d0,
                                cnt, size(dst.chunks[di]), cnt))
        off += prod(cnt)
    end
    GPUWorkspace{T}(CopyPlan(loc, sizeof(T)), isempty(pk) ? nothing : CopyPlan(pk, sizeof(T)),
                    isempty(up) ? nothing : CopyPlan(up, sizeof(T)), sbuf, rbuf, sranks, ssz, rranks, rsz)
end

"""
`gpu_coalesced_redistribute!(dst, src, ws; comm)` (src/fftgpu.jl:320-415):
pack every send (one launch), exchange the flat per-peer buffers with MPI
point-to-point (`comm` an MPI communicator; `nothing` on one rank), run the
local copies (one launch), unpack (one launch).
"""
function gpu_coalesced_redistribute!(dst::ChunkedArray, src::ChunkedArray, ws::GPUWorkspace; comm=nothing)
    ws.pack === nothing || run!(ws.pack)
    reqs = Any[]
    if comm !== nothing && !(isempty(ws.send_ranks) && isempty(ws.recv_ranks))
        CUDA.synchronize()
        mpi = Base.require(Base.PkgId(Base.UUID("da04e1cc-30fd-572f-bb4f-1f8673147195"), "MPI"))
        off = 0
        for (r, n) in zip(ws.recv_ranks, ws.recv_sizes)
            push!(reqs, mpi.Irecv!(view(ws.recv_buffer, off+1:off+n), comm; source=r, tag=0)); off += n
        end
        off = 0
        for (r, n) in zip(ws.send_ranks, ws.send_sizes)
            push!(reqs, mpi.Isend(view(ws.send_buffer, off+1:off+n), comm; dest=r, tag=0)); off += n
        end
    end
    run!(ws.local_copies)
    if !isempty(reqs)
        mpi = Base.require(Base.PkgId(Base.UUID("da04e1cc-30fd-572f-bb4f-1f8673147195"), "MPI"))
        mpi.Waitall(mpi.RequestSet(reqs))
    end
    ws.unpack === nothing || run!(ws.unpack)
    dst
end

function stage!(D::ChunkedArray, transform, dims; method=:plain)
    for c in D.chunks
        c === nothing && continue
        execute!(plan_transform(transform, c, dims; method), c, c)
    end
end
inplace(::Union{FFT,FFT!}) = FFT!()
inplace(::Union{IFFT,IFFT!}) = IFFT!()
inplace(t) = throw(ArgumentError("Unknown transform type"))

"""
    gpu_fft!(C, A, B, wsAB, wsBC, transforms, dims, Pencil(); comm)
    gpu_fft!(B, A, wsAB, transforms, dims, Slab(); comm)

The reference's DArray-level forward drivers (src/fftgpu.jl:498-557): a
per-chunk stage, a redistribution, ... in the reference's stage order.
"""
function gpu_fft!(C::ChunkedArray, A::ChunkedArray, B::ChunkedArray, wsAB, wsBC, transforms, dims,
                  ::Pencil; comm=nothing)
    stage!(A, inplace(transforms[1]), (dims[1],))
    gpu_coalesced_redistribute!(B, A, wsAB; comm)
    stage!(B, inplace(transforms[2]), (dims[2],))
    gpu_coalesced_redistribute!(C, B, wsBC; comm)
    stage!(C, inplace(transforms[3]), (dims[3],))
    C
end
function gpu_fft!(B::ChunkedArray, A::ChunkedArray, wsAB, transforms, dims, ::Slab; comm=nothing)
    stage!(A, inplace(transforms[1]), (dims[1], dims[2]))
    gpu_coalesced_redistribute!(B, A, wsAB; comm)
    stage!(B, inplace(transforms[3]), (dims[3],))
    B
end

"The inverse drivers (src/fftgpu.jl:560-619): transforms[3] on dims[3] first."
function gpu_ifft!(C::ChunkedArray, A::ChunkedArray, B::ChunkedArray, wsAB, wsBC, transforms, dims,
                   ::Pencil; comm=nothing)
    stage!(A, inplace(transforms[3]), (dims[3],))
    gpu_coalesced_redistribute!(B, A, wsAB; comm)
    stage!(B, inplace(transforms[2]), (dims[2],))
    gpu_coalesced_redistribute!(C, B, wsBC; comm)
    stage!(C, inplace(transforms[1]), (dims[1],))
    C
end
function gpu_ifft!(A::ChunkedArray, B::ChunkedArray, wsBA, transforms, dims, ::Slab; comm=nothing)
    stage!(B, inplace(transforms[3]), (dims[3],))
    gpu_coalesced_redistribute!(A, B, wsBA; comm)
    stage!(A, inplace(transforms[1]), (dims[1], dims[2]))
    A
end

# ---- the Slab exchange with pack and unpack folded into the slab pass -----
# (columns split by rank: the Blocks(L, L, c) -> Blocks(c, L, N3) layouts)

"z-slab ranges (start, count) per rank: blocks of cld(n3, P), one per rank."
slab_zsplit(n3, P) = [(min(r * cld(n3, P), n3), min(cld(n3, P), n3 - min(r * cld(n3, P), n3))) for r in 0:P-1]

"Slab groups (offset, count) of `count` local slabs, the same rule on every rank."
function slab_groups(count, ngroups)
    count == 0 && return [(0, 0) for _ in 1:ngroups]
    g = max(1, min(ngroups, count))
    base, extra = divrem(count, g)
    out = Tuple{Int,Int}[]
    z = 0
    for i in 0:ngroups-1
        n = i < g ? base + (i < extra ? 1 : 0) : 0
        push!(out, (z, n))
        z += n
    end
    out
end

"""
    fused_slab_fft!(Bloc, Aloc, L, n3, rank, nranks; comm=nothing, ngroups=2)

Forward 3-D FFT of an L x L x n3 complex array distributed in z-slabs
(`Aloc` = this rank's (L, L, |Z_r|) chunk, overwritten as the in-place
slab stage overwrites it) into x-blocks (`Bloc` = its (L/P, L, n3) chunk)
with no pack or unpack kernel: the slab pass writes each rank's columns of
every local slab as one contiguous block (`slab_split_plan`), the blocks go
out per slab group with MPI point-to-point (CUDA-aware) while the next group
transforms, and the last-axis pass runs on `Bloc` in place.
"""
function fused_slab_fft!(Bloc::CuArray{T,3}, Aloc::CuArray{T,3}, L::Integer, n3::Integer, rank::Integer,
                         nranks::Integer; comm=nothing, ngroups::Integer=2) where {T}
    L % nranks == 0 || throw(ArgumentError("fused Slab exchange needs L % ranks == 0"))
    R = L ÷ nranks
    LR = L * R
    zs = slab_zsplit(n3, nranks)
    Zr = zs[rank+1][2]
    groups = [slab_groups(zs[s+1][2], ngroups) for s in 1:nranks]
    buf = CuArray{T}(undef, LR * Zr * nranks)
    Bv = vec(Bloc)
    mpi = comm === nothing ? nothing :
          Base.require(Base.PkgId(Base.UUID("da04e1cc-30fd-572f-bb4f-1f8673147195"), "MPI"))
    reqs = Any[]
    for g in 1:ngroups
        z0, n = groups[rank+1][g]
        if n > 0
            p = slab_split_plan(T, L, n, Zr, nranks; split_dim=1)
            execute_split!(p, buf, z0 * LR, Aloc, z0 * L * L)
            a = (rank * Zr + z0) * LR
            b = (zs[rank+1][1] + z0) * LR
            copyto!(view(Bv, b+1:b+n*LR), view(buf, a+1:a+n*LR))
        end
        CUDA.synchronize()  # the blocks are written before MPI reads them
        for s in 0:nranks-1
            (s == rank || mpi === nothing) && continue
            zs0, ns = groups[s+1][g]
            if ns > 0
                b = (zs[s+1][1] + zs0) * LR
                push!(reqs, mpi.Irecv!(view(Bv, b+1:b+ns*LR), comm; source=s, tag=g))
            end
            if n > 0
                a = (s * Zr + z0) * LR
                push!(reqs, mpi.Isend(view(buf, a+1:a+n*LR), comm; dest=s, tag=g))
            end
        end
    end
    isempty(reqs) || mpi.Waitall(mpi.RequestSet(reqs))
    execute!(plan_transform(FFT!(), Bloc, (3,)), Bloc, Bloc)
    Bloc
end

"""
    fused_slab_ifft!(Aloc, Bloc, L, n3, rank, nranks; comm=nothing, ngroups=2)

The inverse: the last-axis IFFT on `Bloc` in place, each owner's z-range of
`Bloc` (contiguous) sent to it, and each group of local slabs transformed
out of the received column blocks into `Aloc` as the group arrives.
"""
function fused_slab_ifft!(Aloc::CuArray{T,3}, Bloc::CuArray{T,3}, L::Integer, n3::Integer, rank::Integer,
                          nranks::Integer; comm=nothing, ngroups::Integer=2) where {T}
    L % nranks == 0 || throw(ArgumentError("fused Slab exchange needs L % ranks == 0"))
    R = L ÷ nranks
    LR = L * R
    zs = slab_zsplit(n3, nranks)
    Zr = zs[rank+1][2]
    groups = [slab_groups(zs[s+1][2], ngroups) for s in 1:nranks]
    buf = CuArray{T}(undef, LR * Zr * nranks)
    Bv = vec(Bloc)
    execute!(plan_transform(IFFT!(), Bloc, (3,)), Bloc, Bloc)
    CUDA.synchronize()
    mpi = comm === nothing ? nothing :
          Base.require(Base.PkgId(Base.UUID("da04e1cc-30fd-572f-bb4f-1f8673147195"), "MPI"))
    batches = Vector{Any}[]
    for g in 1:ngroups
        z0, n = groups[rank+1][g]
        reqs = Any[]
        for s in 0:nranks-1
            (s == rank || mpi === nothing) && continue
            zs0, ns = groups[s+1][g]
            if n > 0
                a = (s * Zr + z0) * LR
                push!(reqs, mpi.Irecv!(view(buf, a+1:a+n*LR), comm; source=s, tag=g))
            end
            if ns > 0
                b = (zs[s+1][1] + zs0) * LR
                push!(reqs, mpi.Isend(view(Bv, b+1:b+ns*LR), comm; dest=s, tag=g))
            end
        end
        if n > 0
            a = (rank * Zr + z0) * LR
            b = (zs[rank+1][1] + z0) * LR
            copyto!(view(buf, a+1:a+n*LR), view(Bv, b+1:b+n*LR))
        end
        push!(batches, reqs)
    end
    for g in 1:ngroups
        isempty(batches[g]) || mpi.Waitall(mpi.RequestSet(batches[g]))
        z0, n = groups[rank+1][g]
        n > 0 || continue
        p = slab_split_plan(T, L, n, Zr, nranks; inverse=true, split_dim=1)
        execute_split!(p, Aloc, z0 * L * L, buf, z0 * LR)
    end
    Aloc
end

"`gpu_cleanup_workspace!` (src/fftgpu.jl:630-634)."
function gpu_cleanup_workspace!(ws::GPUWorkspace)
    ws.send_buffer = nothing
    ws.recv_buffer = nothing
    empty!(GPU_PLAN_CACHE)
    nothing
end

export fft, ifft, rfft, irfft, fft!, ifft!, apply_gpu_fft!, Pencil, Slab, R2R
export slab_split_plan, execute_split!, fused_slab_fft!, fused_slab_ifft!
export Batch, launches, wisdom_export, wisdom_import, wisdom_forget, wisdom_size, device_error
export Server, submit, poll, release, cancel, stats, reset_stats!, serve
export ChunkedArray, distribute, distribute_empty, create_gpu_workspace, gpu_coalesced_redistribute!,
       gpu_fft!, gpu_ifft!, gpu_cleanup_workspace!, compute_overlap
export FFT, IFFT, RFFT, IRFFT, FFT!, IFFT!, RFFT!, IRFFT!
export DHT, REDFT00, REDFT01, REDFT10, REDFT11, RODFT00, RODFT01, RODFT10, RODFT11

end # module
