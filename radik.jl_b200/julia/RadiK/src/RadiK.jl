# RadiK -- RadiK.jl's public API (src/RadiK.jl:19-22 of the reference exports
# topk_radix_select!, topk, topk! and RadiKWorkspace) over the C ABI of the
# B200 engine, libradik_b200.so (include/radik.h).
#
# The package keeps the reference's UUID so that it replaces RadiK.jl in an
# environment.  KernelAbstractions kernels give way to `ccall`s on CuArray
# device pointers, issued on CUDA.jl's task-local stream.  Arrays keep the
# reference's layout: the input is the concatenation of all tasks, outputs are
# column-major [k, num_tasks], so task t's results are contiguous at t*k --
# the engine's task-major rows, with no conversion.  Errors are Julia
# ErrorExceptions with the reference's messages (error(...), as in
# src/algorithm.jl:492-510).
#
# Not executed in the environment this engine was built in: it has no Julia
# toolchain.  Every `ccall` below is checked mechanically against
# include/radik.h (symbol, argument count, argument and return widths) by the
# engine's CPU test suite.
module RadiK

using CUDA

export topk_radix_select!, topk, topk!, RadiKWorkspace

const LIB = get(ENV, "RADIK_B200_LIB", joinpath(@__DIR__, "..", "..", "..", "libradik_b200.so"))

# Flags of topk_radix_select! (include/radik.h).
const LARGEST = UInt32(0x1)
const ASCEND = UInt32(0x2)
const WITHSCALE = UInt32(0x4)
const WITHIDXIN = UInt32(0x8)
const WITHPACKING = UInt32(0x10)
const ASYNC = UInt32(0x100)
const PLAIN = UInt32(0x200)

function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:radik_last_error, LIB), Cstring, ()))
    error(isempty(msg) ? unsafe_string(ccall((:radik_status_string, LIB), Cstring, (Cint,), rc)) : msg)
end

"""
    RadiKWorkspace(backend, n, num_tasks, I=Int32)

src/algorithm.jl:58-83.  `n` bounds the longest task and `num_tasks` the
batch of every call that uses the workspace; the engine sizes its device
buffers from the calls it serves and frees them with the workspace.
"""
mutable struct RadiKWorkspace{I}
    handle::Ptr{Cvoid}
    n::Int
    num_tasks::Int
end

function RadiKWorkspace(backend, n, num_tasks, ::Type{I}=Int32) where {I}
    sizeof(I) in (4, 8) || error("workspace integer type must be 4 or 8 bytes")
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:radik_ws_create, LIB), Cint, (Int64, Int64, Cint, Ptr{Ptr{Cvoid}}),
                Int64(n), Int64(num_tasks), Cint(sizeof(I)), h))
    ws = RadiKWorkspace{I}(h[], Int(n), Int(num_tasks))
    finalizer(ws) do w
        w.handle == C_NULL || ccall((:radik_ws_destroy, LIB), Cint, (Ptr{Cvoid},), w.handle)
        w.handle = C_NULL
    end
    return ws
end

lens64(task_lens) = Int64[Int64(x) for x in task_lens]

"""
    topk_radix_select!(val_out, idx_out, ws, val_in, idx_in, task_lens, k,
                       Val(LARGEST)=Val(true), Val(ASCEND)=Val(true),
                       Val(WITHSCALE)=Val(false), Val(WITHIDXIN)=Val(false),
                       Val(WITHPACKING)=Val(true), Val(VLOAD_SIZE_BYTES)=Val(32))

src/algorithm.jl:162-368.  Synchronous, like the reference (:353).
WITHPACKING and VLOAD_SIZE_BYTES are accepted for parity: the engine always
loads 128 bits at a time.
"""
function topk_radix_select!(val_out::CuArray{Float32}, idx_out::CuArray{IdxT}, ws::RadiKWorkspace,
                            val_in::CuArray{Float32}, idx_in::CuArray{IdxT},
                            task_lens::AbstractVector{<:Integer}, k::Integer,
                            ::Val{L}=Val(true), ::Val{A}=Val(true), ::Val{S}=Val(false),
                            ::Val{W}=Val(false), ::Val{P}=Val(true),
                            ::Val{V}=Val(32)) where {IdxT,L,A,S,W,P,V}
    flags = (L ? LARGEST : UInt32(0)) | (A ? ASCEND : UInt32(0)) | (S ? WITHSCALE : UInt32(0)) |
            (W ? WITHIDXIN : UInt32(0)) | (P ? WITHPACKING : UInt32(0))
    lens = lens64(task_lens)
    T = length(lens)
    length(val_out) >= T * k || error("val_out must hold $(T * k) elements, got $(length(val_out))")
    length(idx_out) >= T * k || error("idx_out must hold $(T * k) elements, got $(length(idx_out))")
    length(val_in) >= sum(lens; init=0) || error("val_in must hold sum(task_lens) elements")
    !W || length(idx_in) >= sum(lens; init=0) || error("idx_in must hold sum(task_lens) elements")
    check(ccall((:radik_topk_radix_select, LIB), Cint,
                (CuPtr{Float32}, CuPtr{IdxT}, Cint, Ptr{Cvoid}, CuPtr{Float32}, CuPtr{IdxT},
                 Ptr{Int64}, Int64, Int64, UInt32, CUDA.CUstream),
                val_out, idx_out, Cint(sizeof(IdxT)), ws.handle, val_in, idx_in,
                lens, Int64(T), Int64(k), flags, CUDA.stream()))
    return val_out, idx_out
end

"""
    topk!(val_out, idx_out, data, task_lens, k; indices=nothing, largest=true, rev=false)

src/algorithm.jl:477-522: validates the input type, the output sizes and the
index length with the reference's messages, uses a fresh workspace for the
call (:503) and sorts ascending when `rev` is false (ASCEND = !rev, :520).
"""
function topk!(val_out::CuArray{Float32,2}, idx_out::CuArray{IdxT,2}, data::CuArray,
               task_lens::AbstractVector{<:Integer}, k::Integer;
               indices::Union{Nothing,CuArray{IdxT}}=nothing, largest=true, rev=false) where {IdxT}
    eltype(data) == Float32 || error(
        "RadiK.jl only supports Float32 input data. " *
        "Got $(eltype(data)). Convert with: adapt(backend, Float32.(your_data))")
    expected_size = (k, length(task_lens))
    size(val_out) == expected_size || error("val_out must have size $expected_size, got $(size(val_out))")
    size(idx_out) == expected_size || error("idx_out must have size $expected_size, got $(size(idx_out))")
    if indices !== nothing && !isempty(indices)
        length(indices) == length(data) || error(
            "indices length must equal data length. Got $(length(indices)) vs $(length(data))")
    end
    lens = lens64(task_lens)
    nind = indices === nothing ? 0 : length(indices)
    ind = nind == 0 ? CuPtr{IdxT}(0) : pointer(indices)
    check(ccall((:radik_topk, LIB), Cint,
                (CuPtr{Float32}, CuPtr{IdxT}, Cint, CuPtr{Float32}, Int64, CuPtr{IdxT}, Int64,
                 Ptr{Int64}, Int64, Int64, Cint, Cint, CUDA.CUstream),
                val_out, idx_out, Cint(sizeof(IdxT)), data, Int64(length(data)), ind, Int64(nind),
                lens, Int64(length(lens)), Int64(k), Cint(largest), Cint(rev), CUDA.stream()))
    return nothing
end

topk!(val_out, idx_out, data, k::Integer; indices=nothing, largest=true, rev=false) =
    topk!(val_out, idx_out, data, [length(data)], k; indices=indices, largest=largest, rev=rev)

"""
    topk(data, task_lens, k; indices=nothing, largest=true, rev=false) -> (vals[k, T], idxs[k, T])
    topk(data, k; ...) -> (vals[k], idxs[k])

src/algorithm.jl:528-559.  The index type is eltype(indices), else Int32.
"""
function topk(data::CuArray, task_lens::AbstractVector{<:Integer}, k::Integer;
              indices=nothing, largest=true, rev=false)
    eltype(data) == Float32 || error(
        "RadiK.jl only supports Float32 input data. " *
        "Got $(eltype(data)). Convert with: adapt(backend, Float32.(your_data))")
    IdxT = indices === nothing ? Int32 : eltype(indices)
    val_out = CUDA.zeros(Float32, k, length(task_lens))
    idx_out = CUDA.zeros(IdxT, k, length(task_lens))
    topk!(val_out, idx_out, data, task_lens, k; indices=indices, largest=largest, rev=rev)
    return val_out, idx_out
end

function topk(data, k::Integer; indices=nothing, largest=true, rev=false)
    v, i = topk(data, [length(data)], k; indices=indices, largest=largest, rev=rev)
    return v[:, 1], i[:, 1]
end

# ---- Engine-only functions (no reference counterpart; not exported) ---------

"""Builds and caches the launch plan of a batch shape (before CUDA-graph capture)."""
function prepare!(ws::RadiKWorkspace, task_lens, k::Integer; largest=true, ascend=true,
                  idx_type::Type=Int32)
    lens = lens64(task_lens)
    flags = (largest ? LARGEST : UInt32(0)) | (ascend ? ASCEND : UInt32(0))
    check(ccall((:radik_ws_prepare, LIB), Cint, (Ptr{Cvoid}, Ptr{Int64}, Int64, Int64, UInt32, Cint),
                ws.handle, lens, Int64(length(lens)), Int64(k), flags, Cint(sizeof(idx_type))))
    return ws
end

"""Times the fused path's configurations on this batch and keeps the fastest for its shape."""
function autotune!(ws::RadiKWorkspace, val_out::CuArray{Float32}, idx_out::CuArray{IdxT},
                   val_in::CuArray{Float32}, task_lens, k::Integer; largest=true, ascend=true,
                   reps::Integer=5) where {IdxT}
    lens = lens64(task_lens)
    flags = (largest ? LARGEST : UInt32(0)) | (ascend ? ASCEND : UInt32(0))
    best = Ref{Cdouble}(0)
    check(ccall((:radik_ws_autotune, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Float32}, CuPtr{IdxT}, Cint, CuPtr{Float32}, CuPtr{IdxT},
                 Ptr{Int64}, Int64, Int64, UInt32, CUDA.CUstream, Cint, Ptr{Cvoid}, Ptr{Cdouble}),
                ws.handle, val_out, idx_out, Cint(sizeof(IdxT)), val_in, CuPtr{IdxT}(0),
                lens, Int64(length(lens)), Int64(k), flags, CUDA.stream(), Cint(reps), C_NULL, best))
    return best[]
end

"""
    topk_radix_select_noalloc!(val_out, idx_out, val_in, task_lens, k; largest=true, ascend=true)

topk_radix_select! without a workspace: the engine's scratch is a static
8 MiB device array, so the call allocates no device memory -- for callers
inside an out-of-memory handler or under a hard device-memory cap.  k <= 4096
and the batch's scratch must fit in 8 MiB; calls that overlap on one device race.
"""
function topk_radix_select_noalloc!(val_out::CuArray{Float32}, idx_out::CuArray{IdxT},
                                    val_in::CuArray{Float32}, task_lens, k::Integer;
                                    largest=true, ascend=true) where {IdxT}
    lens = lens64(task_lens)
    flags = (largest ? LARGEST : UInt32(0)) | (ascend ? ASCEND : UInt32(0))
    check(ccall((:radik_topk_noalloc, LIB), Cint,
                (CuPtr{Float32}, CuPtr{IdxT}, Cint, CuPtr{Float32}, CuPtr{IdxT}, Ptr{Int64}, Int64, Int64,
                 UInt32, CUDA.CUstream),
                val_out, idx_out, Cint(sizeof(IdxT)), val_in, CuPtr{IdxT}(0), lens, Int64(length(lens)), Int64(k),
                flags, CUDA.stream()))
    return val_out, idx_out
end

"""CUDA allocations (device and pinned host) the engine has made in this process."""
function alloc_count()
    n = Ref{UInt64}(0)
    check(ccall((:radik_alloc_count, LIB), Cint, (Ptr{UInt64},), n))
    return n[]
end

# Tuning table: the autotuner's choices by batch shape, shared by every
# workspace of the process, kept in a text file between processes.
"""Write the process-wide tuning table to `path`."""
tune_save(path::AbstractString) = (check(ccall((:radik_tune_save, LIB), Cint, (Cstring,), path)); nothing)

"""Merge a tuning table written by `tune_save`; returns the entries read."""
function tune_load(path::AbstractString)
    n = Ref{Int64}(0)
    check(ccall((:radik_tune_load, LIB), Cint, (Cstring, Ptr{Int64}), path, n))
    return n[]
end

"""Forget every remembered tuning choice of the process."""
tune_clear() = (check(ccall((:radik_tune_clear, LIB), Cint, ())); nothing)

# Request server: continuous batching of independent top-k requests.
struct ServerConfig
    slots::Cint
    device::Cint
    mem_cap_bytes::Int64
    max_batch_rows::Int64
end

mutable struct Server
    handle::Ptr{Cvoid}
end

function Server(; slots::Integer=4, device::Integer=0, mem_cap_bytes::Integer=32 << 30,
                max_batch_rows::Integer=4096)
    cfg = Ref(ServerConfig(Cint(slots), Cint(device), Int64(mem_cap_bytes), Int64(max_batch_rows)))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:radik_server_create, LIB), Cint, (Ptr{ServerConfig}, Ptr{Ptr{Cvoid}}), cfg, h))
    srv = Server(h[])
    finalizer(srv) do s
        s.handle == C_NULL || ccall((:radik_server_destroy, LIB), Cint, (Ptr{Cvoid},), s.handle)
        s.handle = C_NULL
    end
    return srv
end

"""Queues the k best of every column of `data` (a Julia column is one row of
the request); returns (ticket, vals[k, rows], idxs[k, rows])."""
function submit(srv::Server, data::CuArray{Float32,2}, k::Integer; largest=true, rev=false)
    row_len, rows = size(data)
    v = CuArray{Float32}(undef, k, rows)
    i = CuArray{Int32}(undef, k, rows)
    flags = (largest ? LARGEST : UInt32(0)) | (!rev ? ASCEND : UInt32(0))
    t = Ref{UInt64}(0)
    check(ccall((:radik_server_submit, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Float32}, Int64, Int64, Int64, UInt32, CuPtr{Float32}, CuPtr{Int32}, Cint,
                 Ptr{UInt64}),
                srv.handle, data, Int64(rows), Int64(row_len), Int64(k), flags, v, i, Cint(4), t))
    return t[], v, i
end

"""Waits for a ticket (timeout_us < 0: no limit)."""
function wait_ticket(srv::Server, ticket::UInt64; timeout_us::Integer=-1)
    check(ccall((:radik_server_wait, LIB), Cint, (Ptr{Cvoid}, UInt64, Int64), srv.handle, ticket,
                Int64(timeout_us)))
    return nothing
end

end # module RadiK
