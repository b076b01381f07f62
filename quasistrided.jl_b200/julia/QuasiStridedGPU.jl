# QuasiStridedGPU — Julia binding of libqsgpu.so (include/qsgpu.h).
#
# Device-resident strided operands drop into QuasiStrided's API: the labels
# are resolved by the library's planner (the same rules as
# src/planning/labels.jl), and execution runs on the B200 kernels.  Shipped
# as source; it needs CUDA.jl for device arrays and streams.
module QuasiStridedGPU

using CUDA
import TensorOperations as TO

const libqsgpu = get(ENV, "QSGPU_LIB", joinpath(@__DIR__, "..", "lib", "libqsgpu.so"))

# --- C structs (layout of include/qsgpu.h) ---------------------------------

struct QSView
    data::Ptr{Cvoid}
    length::Int64
    offset::Int64
    size::Ptr{Int64}
    strides::Ptr{Int64}
    ndim::Int32
    eltype::Int32
    op::Int32
    reserved::Int32
end

Base.@kwdef struct QSPlanOptions
    conjA::Int32 = 0
    conjB::Int32 = 0
    accumulator::Int32 = 0
    method::Int32 = 0
    m_block::Int64 = 0
    k_block::Int64 = 0
    n_block::Int64 = 0
    dot_mode::Int32 = 0
    outer_mode::Int32 = 0
    unpacked_b_mode::Int32 = 0
    ozaki_slices::Int32 = 0
    complex_mode::Int32 = 0
    flags::Int32 = 0
    native_tile::Int32 = 0
    allocator::Ptr{Cvoid} = C_NULL   # const qs_allocator*; C_NULL = the library's pool
end

const ELTYPE = Dict(Float32 => Int32(0), Float64 => Int32(1), ComplexF32 => Int32(2), ComplexF64 => Int32(3))
opcode(::typeof(identity)) = Int32(0)
opcode(::typeof(conj)) = Int32(1)
opcode(::typeof(transpose)) = Int32(2)
opcode(::typeof(adjoint)) = Int32(3)
opcode(f) = throw(ArgumentError("unsupported StridedView.op $f"))
accode(::Nothing) = Int32(0)
accode(::Type{Float32}) = Int32(1)
accode(::Type{Float64}) = Int32(2)

"""
    DeviceStridedView(parent::CuArray, size, strides, offset, op = identity)

A StridedView over device memory: the fields StridedViews.jl's `StridedView`
carries (size, strides, offset, op) over a `CuArray` parent.
"""
struct DeviceStridedView{T, N, A <: CuArray{T}, F}
    parent::A
    size::NTuple{N, Int}
    strides::NTuple{N, Int}
    offset::Int
    op::F
end
DeviceStridedView(a::CuArray{T, N}) where {T, N} =
    DeviceStridedView(a, size(a), strides(a), 0, identity)
Base.eltype(::DeviceStridedView{T}) where {T} = T

function check(rc::Cint)
    rc == 0 && return nothing
    buf = Vector{UInt8}(undef, 4096)
    ccall((:qs_last_error, libqsgpu), Csize_t, (Ptr{UInt8}, Csize_t), buf, length(buf))
    msg = unsafe_string(pointer(buf))
    rc == 1 && throw(ArgumentError(msg))
    rc == 2 && throw(DimensionMismatch(msg))
    rc == 3 && throw(BoundsError(msg))
    rc == 7 && throw(ArgumentError(msg))
    error("qsgpu status $rc: $msg")
end

# Build the C view; the size/stride vectors are kept alive by the caller.
function cview(v::DeviceStridedView{T}, keep) where {T}
    sz = collect(Int64, v.size)
    st = collect(Int64, v.strides)
    push!(keep, sz, st)
    return QSView(reinterpret(Ptr{Cvoid}, pointer(v.parent)), length(v.parent), v.offset,
        pointer(sz), pointer(st), Int32(length(v.size)), ELTYPE[T], opcode(v.op), Int32(0))
end

mutable struct ContractPlan
    handle::Ptr{Cvoid}
    C::DeviceStridedView
    A::DeviceStridedView
    B::DeviceStridedView
    allocator::Any   # kept alive while the plan holds its workspace
end

# --- allocators ---------------------------------------------------------------

"""
    DeviceArenaAllocator(nbytes)

TensorOperations' BufferAllocator on the device (qs_arena_*): plan workspace
and `tensoralloc`'d intermediates from one device buffer; `tensorfree!` of the
last block pops it, `allocator_reset!` reclaims everything after a checkpoint.
Reclaimed memory is reused only after the work enqueued before the reclaim on
CUDA.jl's current stream.
"""
mutable struct DeviceArenaAllocator
    handle::Ptr{Cvoid}
    function DeviceArenaAllocator(nbytes::Integer)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:qs_arena_create, libqsgpu), Cint, (Ref{Ptr{Cvoid}}, Ptr{Cvoid}, Csize_t),
            h, C_NULL, nbytes))
        a = new(h[])
        finalizer(a) do a
            a.handle != C_NULL && ccall((:qs_arena_destroy, libqsgpu), Cint, (Ptr{Cvoid},), a.handle)
            a.handle = C_NULL
        end
        return a
    end
end

allocator_ptr(::TO.DefaultAllocator) = C_NULL
allocator_ptr(a::DeviceArenaAllocator) = ccall((:qs_arena_allocator, libqsgpu), Ptr{Cvoid}, (Ptr{Cvoid},), a.handle)
allocator_ptr(a) = throw(ArgumentError("unsupported allocator $(typeof(a)): use DefaultAllocator or DeviceArenaAllocator"))

curstream() = reinterpret(Ptr{Cvoid}, CUDA.stream().handle)

function TO.tensoralloc(::Type{A}, structure, istemp, a::DeviceArenaAllocator) where {T, N, A <: CuArray{T, N}}
    p = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:qs_arena_alloc, libqsgpu), Cint, (Ptr{Cvoid}, Csize_t, Ref{Ptr{Cvoid}}),
        a.handle, prod(structure; init = 1) * sizeof(T), p))
    return unsafe_wrap(CuArray, CuPtr{T}(UInt(p[])), structure; own = false)
end

TO.tensorfree!(t::CuArray, a::DeviceArenaAllocator) =
    (check(ccall((:qs_arena_free, libqsgpu), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Csize_t, Ptr{Cvoid}),
        a.handle, reinterpret(Ptr{Cvoid}, UInt(pointer(t))), sizeof(t), curstream())); nothing)

TO.allocator_checkpoint!(a::DeviceArenaAllocator) =
    ccall((:qs_arena_checkpoint, libqsgpu), Csize_t, (Ptr{Cvoid},), a.handle)

TO.allocator_reset!(a::DeviceArenaAllocator, checkpoint) =
    (check(ccall((:qs_arena_reset, libqsgpu), Cint, (Ptr{Cvoid}, Csize_t, Ptr{Cvoid}),
        a.handle, checkpoint, curstream())); nothing)

release!(p::ContractPlan) = (p.handle != C_NULL && ccall((:qs_plan_destroy, libqsgpu), Cint, (Ptr{Cvoid},), p.handle); p.handle = C_NULL; nothing)

"""
    plan_contract(C, A, indA, B, indB, indC; conjA=false, conjB=false, accumulator=nothing)

QuasiStrided.plan_contract for device views (src/planning/plan.jl:115-133).
"""
function plan_contract(C::DeviceStridedView, A::DeviceStridedView, indA::NTuple{NA, Int},
        B::DeviceStridedView, indB::NTuple{NB, Int}, indC::NTuple{NC, Int};
        conjA::Bool = false, conjB::Bool = false, accumulator = nothing,
        allocator = TO.DefaultAllocator()) where {NA, NB, NC}
    keep = Any[]
    cC, cA, cB = cview(C, keep), cview(A, keep), cview(B, keep)
    opts = QSPlanOptions(; conjA = Int32(conjA), conjB = Int32(conjB), accumulator = accode(accumulator),
        allocator = allocator_ptr(allocator))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep begin
        check(ccall((:qs_plan_contract, libqsgpu), Cint,
            (Ref{Ptr{Cvoid}}, Ref{QSView}, Ref{QSView}, Ptr{Int64}, Ref{QSView}, Ptr{Int64}, Ptr{Int64}, Ref{QSPlanOptions}),
            h, cC, cA, collect(Int64, indA), cB, collect(Int64, indB), collect(Int64, indC), opts))
    end
    p = ContractPlan(h[], C, A, B, allocator)
    finalizer(release!, p)
    return p
end

"""
    execute!(plan, alpha, beta) -> parent(C)

QuasiStrided.execute! (src/execution/execute.jl:11): enqueued on CUDA.jl's
current stream.
"""
function execute!(p::ContractPlan, alpha::Number, beta::Number)
    a = Float64[real(alpha), imag(alpha)]
    b = Float64[real(beta), imag(beta)]
    stream = CUDA.stream().handle
    check(ccall((:qs_execute, libqsgpu), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Cvoid}),
        p.handle, a, b, reinterpret(Ptr{Cvoid}, stream)))
    return p.C.parent
end

"""
    check_status(p::ContractPlan)

Synchronizes CUDA.jl's stream and throws if a bounded device wait of the
plan's tensor-core kernels gave up since the last check (QS_ETIMEOUT): the
kernel stopped without writing C; the plan stays usable.
"""
check_status(p::ContractPlan) =
    check(ccall((:qs_plan_check_status, libqsgpu), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), p.handle,
        reinterpret(Ptr{Cvoid}, CUDA.stream().handle)))

"""
    set_wait_limit!(p::ContractPlan, limit_ns = 0; hold_loads = false)

Bound every device wait of the plan's tensor-core kernels (0: the default
2 s); `hold_loads` makes a wait run out with nothing in flight, for tests of
the failure path.
"""
set_wait_limit!(p::ContractPlan, limit_ns::Integer = 0; hold_loads::Bool = false) =
    check(ccall((:qs_plan_set_wait_limit, libqsgpu), Cint, (Ptr{Cvoid}, UInt64, Int32), p.handle,
        UInt64(limit_ns), Int32(hold_loads)))

"""
    contract!(C, alpha, A, indA, B, indB, beta, indC; accumulator = nothing) -> C
"""
function contract!(C::DeviceStridedView, alpha::Number, A::DeviceStridedView, indA, B::DeviceStridedView,
        indB, beta::Number, indC; accumulator = nothing)
    p = plan_contract(C, A, indA, B, indB, indC; accumulator)
    execute!(p, alpha, beta)
    CUDA.synchronize()  # the plan's workspace goes back to the pool below
    release!(p)
    return C
end

"""
    QuasiStridedGPUBackend(; accumulator = nothing)

The device counterpart of QuasiStridedBackend
(src/integrations/tensoroperations.jl:24-32).
"""
struct QuasiStridedGPUBackend{A} <: TO.AbstractBackend
    function QuasiStridedGPUBackend{A}() where {A}
        A in (nothing, Float32, Float64) ||
            throw(ArgumentError("QuasiStridedGPUBackend: accumulator must be nothing, Float32 or Float64, got $A"))
        return new{A}()
    end
end
QuasiStridedGPUBackend(; accumulator = nothing) = QuasiStridedGPUBackend{accumulator}()

function TO.tensorcontract!(C::CuArray, A::CuArray, pA::TO.Index2Tuple, conjA::Bool,
        B::CuArray, pB::TO.Index2Tuple, conjB::Bool, pAB::TO.Index2Tuple,
        α::Number, β::Number, ::QuasiStridedGPUBackend{AC}, allocator = TO.DefaultAllocator()) where {AC}
    # prepare_contraction's checks (src/integrations/tensoroperations.jl:61-70)
    TO.argcheck_tensorcontract(C, A, pA, B, pB, pAB)
    TO.dimcheck_tensorcontract(C, A, pA, B, pB, pAB)
    NoA, Nk, NoB = length(pA[1]), length(pA[2]), length(pB[2])
    lin(p) = Int64[p[1]..., p[2]...]
    indA = Vector{Int64}(undef, NoA + Nk)
    indB = Vector{Int64}(undef, Nk + NoB)
    indC = Vector{Int64}(undef, NoA + NoB)
    check(ccall((:qs_contraction_labels, libqsgpu), Cint,
        (Int32, Int32, Int32, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}),
        NoA, Nk, NoB, lin(pA), lin(pB), lin(pAB), indA, indB, indC))
    # Bracketed with checkpoint/reset like the reference (tensoroperations.jl:84-86).
    checkpoint = TO.allocator_checkpoint!(allocator)
    p = plan_contract(DeviceStridedView(C), DeviceStridedView(A), Tuple(indA), DeviceStridedView(B),
        Tuple(indB), Tuple(indC); conjA, conjB, accumulator = AC, allocator)
    execute!(p, α, β)
    allocator isa DeviceArenaAllocator || CUDA.synchronize()
    release!(p)
    TO.allocator_reset!(allocator, checkpoint)
    return C
end

"""
    add_trace!(C, alpha, A, indA, beta, indC; conjA = false) -> C

`C[indC] = alpha * (sum over traced labels of op(A)[indA]) + beta * C` on the
device (qs_tensoradd_trace): labels of indC appear once in indA, the other
labels of indA exactly twice. Runs on CUDA.jl's current stream.
"""
function add_trace!(C::DeviceStridedView, alpha::Number, A::DeviceStridedView, indA, beta::Number, indC;
        conjA::Bool = false)
    keep = Any[]
    cC, cA = cview(C, keep), cview(A, keep)
    iA, iC = collect(Int64, indA), collect(Int64, indC)
    GC.@preserve keep iA iC begin
        check(ccall((:qs_tensoradd_trace, libqsgpu), Cint,
            (Ref{QSView}, Ptr{Float64}, Ref{QSView}, Ptr{Int64}, Int32, Ptr{Float64}, Ptr{Int64}, Ptr{Cvoid}),
            cC, Float64[real(alpha), imag(alpha)], cA, iA, Int32(conjA), Float64[real(beta), imag(beta)], iC,
            reinterpret(Ptr{Cvoid}, CUDA.stream().handle)))
    end
    return C
end

# TO.tensoradd!: C = β C + α permutedims(op(A), linearize(pA)); the reference
# forwards this to StridedNative on the host (tensoroperations.jl:91-98).
function TO.tensoradd!(C::CuArray, A::CuArray, pA::TO.Index2Tuple, conjA::Bool, α::Number, β::Number,
        ::QuasiStridedGPUBackend, allocator = TO.DefaultAllocator())
    perm = (pA[1]..., pA[2]...)
    indA = zeros(Int64, ndims(A))
    for (i, ax) in enumerate(perm)
        indA[ax] = i
    end
    add_trace!(DeviceStridedView(C), α, DeviceStridedView(A), indA, β, 1:ndims(C); conjA)
    return C  # stream-ordered: later work on CUDA.jl's stream sees C
end

# TO.tensortrace!: C = β C + α (trace of op(A) over the pairs (q[1][j], q[2][j]),
# the kept axes linearize(p) in C's order) (tensoroperations.jl:100-107).
function TO.tensortrace!(C::CuArray, A::CuArray, p::TO.Index2Tuple, q::TO.Index2Tuple, conjA::Bool,
        α::Number, β::Number, ::QuasiStridedGPUBackend, allocator = TO.DefaultAllocator())
    indA = zeros(Int64, ndims(A))
    for (i, ax) in enumerate((p[1]..., p[2]...))
        indA[ax] = i
    end
    for (j, (x, y)) in enumerate(zip(q[1], q[2]))
        indA[x] = indA[y] = -j
    end
    add_trace!(DeviceStridedView(C), α, DeviceStridedView(A), indA, β, 1:ndims(C); conjA)
    return C  # stream-ordered: later work on CUDA.jl's stream sees C
end

end # module
