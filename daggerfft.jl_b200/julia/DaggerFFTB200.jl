"""
    DaggerFFTB200

Julia front end over libdfft (include/dfft.h) for CuArrays: the README API of
DaggerFFT.jl (`fft`, `ifft`, `rfft`, `irfft` with `decomp`, `transforms`,
`dims`) and the plan-level `apply_gpu_fft!`, executed by hand-written sm_100a
kernels.  Arrays are used in Julia's own column-major layout; every call runs
on the CuArray's task-local stream.

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

function plan_transform(transform, A::CuArray, dims; decomp=Pencil(), n=0, method=0, flags=0)
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
                    kinds, Int64(n), code(decomp), Cint(method), Cuint(flags)))
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

"`apply_gpu_fft!(out, in, transform, dim)`: plan lookup + execute (src/fftgpu.jl:118-124)."
function apply_gpu_fft!(out, in, transform, dim; kw...)
    execute!(plan_transform(transform, in, dim; kw...), out, in)
end

cplx(::Type{Float32}) = ComplexF32
cplx(::Type{Float64}) = ComplexF64
realt(::Type{ComplexF32}) = Float32
realt(::Type{ComplexF64}) = Float64

function fft(A::CuArray; decomp=Pencil(), dims=(1, 2, 3), transforms=nothing)
    if transforms !== nothing && first(transforms) isa R2R
        p = plan_transform(first(transforms), A, dims; decomp)
        return execute!(p, similar(A, p.outsize), A)
    end
    B = eltype(A) <: Complex ? A : CuArray{cplx(eltype(A))}(A)
    p = plan_transform(FFT(), B, dims; decomp)
    execute!(p, similar(B, p.outsize), B)
end

function ifft(A::CuArray; decomp=Pencil(), dims=(1, 2, 3), transforms=nothing)
    if transforms !== nothing && first(transforms) isa R2R
        p = plan_transform(first(transforms), A, dims; decomp)
        return execute!(p, similar(A, p.outsize), A)
    end
    p = plan_transform(IFFT(), A, dims; decomp)
    execute!(p, similar(A, p.outsize), A)
end

function rfft(A::CuArray{<:Real}; decomp=Pencil(), dims=(1, 2, 3))
    p = plan_transform(RFFT(), A, dims; decomp)
    execute!(p, CuArray{cplx(eltype(A))}(undef, p.outsize), A)
end

function irfft(F::CuArray{<:Complex}, d::Integer; decomp=Pencil(), dims=(1, 2, 3))
    p = plan_transform(IRFFT(), F, dims; decomp, n=d)
    execute!(p, CuArray{realt(eltype(F))}(undef, p.outsize), F)
end

export fft, ifft, rfft, irfft, apply_gpu_fft!, Pencil, Slab, R2R
export FFT, IFFT, RFFT, IRFFT, FFT!, IFFT!, RFFT!, IRFFT!
export DHT, REDFT00, REDFT01, REDFT10, REDFT11, RODFT00, RODFT01, RODFT10, RODFT11

end # module
