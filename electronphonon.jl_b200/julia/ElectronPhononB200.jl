"""
    ElectronPhononB200

`ccall` glue that routes ElectronPhonon.jl's device methods to libepb200.so (B200, sm_100a).
Loaded after `ElectronPhonon` and `CUDA`, it replaces the methods that the reference's CUDA
extension defines on `CuArray` (ext/ElectronPhononCUDAExt.jl) and adds device methods for the
batched Fourier and e-ph drivers, so that every caller above them is unchanged. Device buffers
stay CUDA.jl `CuArray`s; the library reads and writes them through their pointers, in order on
the task's CUDA stream.

This file is the binding a maintainer adds to the reference; it is written against the reference's
public API (`WannierObject`, `BatchedWannierInterpolator`, the `wannier_to_bloch_batched.jl`
drivers) and has not been executed in this repository's environment (no Julia toolchain).
"""
module ElectronPhononB200

using CUDA
using ElectronPhonon
using ElectronPhonon: WannierObject, Vec3

const LIB = Ref(joinpath(@__DIR__, "..", "lib", "libepb200.so"))
# Precision of the methods that replace the reference's own (fourier, eigensolves, e-ph chain, rotations,
# batched_gemm!): plain FP64 by default, the reference's semantics (cuBLAS ZGEMM + cuSOLVER heevj in
# FP64, ext/ElectronPhononCUDAExt.jl:80-126). `set_precision!(:mixed)` opts into the split-precision
# tensor-core path (FP32-level sums, FP32 eigensolve + FP64 refinement).
const PREC = Ref{Cint}(0)
# Precision of this library's own drivers (eph_pass, serta, eph_outer_q, the band / window calls, the
# surrogate screen), which have no FP64 counterpart in the reference to match: mixed by default.
const DRIVER_PREC = Ref{Cint}(1)
function set_precision!(p::Symbol; drivers::Bool = false)
    v = p === :fp64 ? Cint(0) : p === :mixed ? Cint(1) : throw(ArgumentError("precision :fp64 or :mixed"))
    drivers ? (DRIVER_PREC[] = v) : (PREC[] = v)
    v
end
const NULLDEV = CuPtr{Cvoid}(0)  # an absent optional device buffer

last_error() = unsafe_string(ccall((:epb_last_error, LIB[]), Cstring, ()))
check(st::Integer) = st == 0 || error("libepb200: status $st: $(last_error())")

# ---- context: one per (device, host thread); bound to the calling task's stream on every call ----
# The library's workspace lives in the context, so one per device and thread is enough; CUDA.jl gives
# each task its own stream, which `ctx()` installs (epb_set_stream) before the call, so a context never
# holds a stream handle past the call that used it.
mutable struct Ctx
    h::Ptr{Cvoid}
end
const CTX = Dict{Tuple{Int,Int},Ctx}()
const CTX_LOCK = ReentrantLock()
function ctx()
    dev = CUDA.deviceid(CUDA.device())
    s = CUDA.stream()
    c = lock(CTX_LOCK) do
        get!(CTX, (dev, Threads.threadid())) do
            r = Ref{Ptr{Cvoid}}(C_NULL)
            check(ccall((:epb_create, LIB[]), Cint, (Ptr{Ptr{Cvoid}}, Cint, Ptr{Cvoid}), r, dev, s.handle))
            c = Ctx(r[])
            finalizer(x -> ccall((:epb_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), c)
            c
        end
    end
    check(ccall((:epb_set_stream, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), c.h, s.handle))
    c
end

# ---- device operands as the reference's loop passes them ---------------------------------------
# The batched loop hands over contiguous device VIEWS (view(epkq_dev, :,:,:, rng_q), view(P_kq, :, rng_q),
# view(ep_ekpR_all, :, :, ik_ind); run_eph_over_k_and_kq.jl:821-869) and reshapes of them
# (reshape(view(ws.g, :, 1:nq), ...), wannier_to_bloch_batched.jl:270), so the overrides are typed
# DenseCuArray / StridedCuArray / AnyCuArray like the extension's own methods (ext:172-179), never a bare
# CuArray. `devptr` is the device address of such an operand; `colstride` its column stride.
function assert_dense(a)
    c = a isa Base.ReshapedArray ? Base.iscontiguous(parent(a)) : Base.iscontiguous(a)
    c || throw(ArgumentError("libepb200: this operand must be contiguous (got $(typeof(a)))"))
    a
end
function devptr(a)
    a === nothing && return NULLDEV
    assert_dense(a)
    p = a isa Base.ReshapedArray && !(a isa DenseCuArray) ? parent(a) : a  # reshape(view(...)): the view's address
    p isa StridedCuArray || throw(ArgumentError("libepb200: expected a device array, got $(typeof(a))"))
    Base.unsafe_convert(CuPtr{eltype(p)}, p)  # the conversion ccall applies to a device array argument
end
function colstride(a::AbstractArray)
    stride(a, 1) == 1 || throw(ArgumentError("libepb200: the first axis of a device operand must be contiguous"))
    ndims(a) >= 2 ? stride(a, 2) : length(a)
end
colstride(a::Base.ReshapedArray) = size(a, 1)  # a reshape of a contiguous array is contiguous

# ---- lattice-vector sets (BatchedFourierCore's irvec_mat, WannierObject.jl:148-152) ---------
mutable struct RSet
    h::Ptr{Cvoid}
end
const RSETS = IdDict{Any,RSet}()
function rset(irvec::Vector{Vec3{Int}})
    get!(RSETS, irvec) do
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:epb_rset_create, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Int64}, Int64, Ptr{Ptr{Cvoid}}),
                    ctx().h, reinterpret(Int64, irvec), length(irvec), r))
        s = RSet(r[])
        finalizer(x -> ccall((:epb_rset_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), s)
        s
    end
end

# k lists: a host Vector{Vec3} (or a view of one) is uploaded; a (3 x nk) device matrix is used in place
xk_device(xks) = CuArray(reinterpret(reshape, Float64, collect(Vec3{Float64}, xks)))  # 3 x nk
xk_device(xks::DenseCuMatrix{Float64}) = xks

# ---- backend (ext:34-37) -----------------------------------------------------------------------
function ElectronPhonon.free_bytes(::ElectronPhonon.GPUBackend)
    f = Ref{UInt64}(0); t = Ref{UInt64}(0)
    check(ccall((:epb_free_bytes, LIB[]), Cint, (Ptr{Cvoid}, Ref{UInt64}, Ref{UInt64}), ctx().h, f, t))
    Int(f[])
end
ElectronPhonon.synchronize(::ElectronPhonon.GPUBackend) =
    check(ccall((:epb_synchronize, LIB[]), Cint, (Ptr{Cvoid},), ctx().h))

# ---- Fourier (batched_fourier_core.jl:24-30, 117-139) ----------------------------------------
# fourier_phase!(phase, irvec_mat, xkmat): the reference's own operands, the (nr x 3) FP64 R matrix of
# _irvec_to_device_matrix and a (3 x nk) coordinate matrix, views included (P_mk[:, 1:nk_batch] and
# mxk_dev[:, iks_batch] at run_eph_over_k_and_kq.jl:821; batched_fourier_core.jl:104).
function ElectronPhonon.fourier_phase!(phase::StridedCuMatrix{ComplexF64}, irvec_mat::StridedCuMatrix{Float64},
        xkmat::StridedCuMatrix{Float64})
    nr, nk = size(phase)
    @assert size(irvec_mat) == (nr, 3) && size(xkmat) == (3, nk)
    check(ccall((:epb_fourier_phase_mat, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, Int64, Int64, CuPtr{Float64}, Int64, Int64, CuPtr{ComplexF64}, Int64),
                ctx().h, irvec_mat, colstride(irvec_mat), nr, xkmat, colstride(xkmat), nk, phase, colstride(phase)))
    phase
end

function ElectronPhonon.get_fourier_batched!(out::DenseCuMatrix{ComplexF64},
        itp::ElectronPhonon.BatchedWannierInterpolator, xks)
    p = itp.parent
    xk = xk_device(xks)
    @assert size(out) == (p.ndata, size(xk, 2))
    check(ccall((:epb_fourier, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{ComplexF64}, Cint),
                ctx().h, p.op_r, size(p.op_r, 1), p.ndata, rset(p.irvec).h, xk, size(xk, 2), out, PREC[]))
    out
end

# batched_gemm! (src/common/gpu_utils.jl:71-78; CUDA method ext:122-126): strided-batched, alpha = 1, beta = 0
function ElectronPhonon.batched_gemm!(transA::Char, transB::Char, A::StridedCuArray{ComplexF64,3},
        B::StridedCuArray{ComplexF64,3}, C::StridedCuArray{ComplexF64,3})
    m, n, nb = size(C)
    k = transA == 'N' ? size(A, 2) : size(A, 1)
    @assert size(A, 3) == size(B, 3) == nb
    @assert (transA == 'N' ? size(A, 1) : size(A, 2)) == m && (transB == 'N' ? size(B, 1) : size(B, 2)) == k &&
            (transB == 'N' ? size(B, 2) : size(B, 1)) == n
    check(ccall((:epb_batched_zgemm, LIB[]), Cint,
                (Ptr{Cvoid}, Cchar, Cchar, Int64, Int64, Int64, CuPtr{ComplexF64}, Int64, Int64, CuPtr{ComplexF64},
                 Int64, Int64, CuPtr{ComplexF64}, Int64, Int64, Int64),
                ctx().h, transA, transB, m, n, k, A, colstride(A), stride(A, 3), B, colstride(B), stride(B, 3),
                C, colstride(C), stride(C, 3), nb))
    C
end

# ---- eigensolves (ext:80-115) -----------------------------------------------------------------
# Hk as the callers pass it: a CuArray or a reshape / contiguous view of one
# (eigen_batched(reshape(Hkq_flat, nw, nw, nk_batch_max)), run_eph_over_q_and_k.jl:578).
function ElectronPhonon.eigvals_batched(Hk::DenseCuArray{ComplexF64,3})
    nw, _, nk = size(Hk)
    E = CuArray{Float64}(undef, nw, nk)
    check(ccall((:epb_eigh_batched, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, CuPtr{Float64}, Cchar, Cint),
                ctx().h, Hk, nw, nk, E, 'N', PREC[]))
    E
end

function ElectronPhonon.eigen_batched(Hk::DenseCuArray{ComplexF64,3})
    nw, _, nk = size(Hk)
    E = CuArray{Float64}(undef, nw, nk)
    check(ccall((:epb_eigh_batched, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, CuPtr{Float64}, Cchar, Cint),
                ctx().h, Hk, nw, nk, E, 'V', PREC[]))
    E, Hk  # eigenvectors overwrite Hk (destroy-input contract)
end

# phonons: D(q) / sqrt(m_i m_j) -> eigen -> omega = sign sqrt, u ./= sqrt(m) (compute_states.jl:293-300)
function phonon_eigen_batched!(Dq::DenseCuArray{ComplexF64,3}, mass::DenseCuVector{Float64})
    nm, _, nq = size(Dq)
    ω = CuArray{Float64}(undef, nm, nq)
    check(ccall((:epb_ph_eigen_batched, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, CuPtr{Float64}, Int64, Int64, CuPtr{Float64}, Cint),
                ctx().h, Dq, mass, nm, nq, ω, PREC[]))
    ω, Dq
end

# ---- e-ph chain (wannier_to_bloch_batched.jl:178-273, 442-455) -------------------------------
# call site: get_eph_RR_to_kR_batched!(ep_ekpR_all, itp_epmat, ks_batch, uks_dev; additional_phase = P_mk)
# (run_eph_over_k_and_kq.jl:822): device buffers, a host k list
function ElectronPhonon.get_eph_RR_to_kR_batched!(ep_ekpR_all::DenseCuArray{ComplexF64,3},
        itp_epmat::ElectronPhonon.BatchedWannierInterpolator, ks, uks::DenseCuArray{ComplexF64,3};
        additional_phase::Union{Nothing,DenseCuMatrix{ComplexF64}} = nothing)
    epmat = itp_epmat.parent
    nr_ep = length(epmat.irvec_next)
    nw, nband, nk = size(uks)
    nmodes = div(epmat.ndata, nw^2 * nr_ep)
    @assert size(ep_ekpR_all) == (nw * nband * nmodes, nr_ep, nk)
    additional_phase === nothing || @assert size(additional_phase) == (nr_ep, nk)
    xk = xk_device(ks)
    check(ccall((:epb_eph_RR_to_kR, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Ptr{Cvoid}, CuPtr{Float64}, Int64,
                 CuPtr{ComplexF64}, Int64, CuPtr{ComplexF64}, CuPtr{ComplexF64}, Cint),
                ctx().h, epmat.op_r, nw, nmodes, nr_ep, rset(epmat.irvec).h, xk, nk, uks, nband,
                devptr(additional_phase), ep_ekpR_all, PREC[]))
    ep_ekpR_all
end

# call site (run_eph_over_k_and_kq.jl:866-869): every array argument a contiguous device view,
#   get_eph_kR_to_kq_batched!(view(epkq_dev, :,:,:, rng_q), view(ep_ekpR_all, :, :, ik_ind), view(P_kq, :, rng_q),
#       view(uphs_dev, :, :, rng_q), view(ukqs_all_dev, :, :, qstart:qend); ws, g2_out = view(g2_dev, ...), ωq = view(ωq_dev, :, rng_q))
function ElectronPhonon.get_eph_kR_to_kq_batched!(ep_kq_all::DenseCuArray{ComplexF64,4},
        ep_kR::StridedCuMatrix{ComplexF64}, phase::StridedCuMatrix{ComplexF64}, u_phs::DenseCuArray{ComplexF64,3},
        ukqs::DenseCuArray{ComplexF64,3}; ws = nothing, g2_out::Union{Nothing,DenseCuArray{Float64,4}} = nothing,
        ωq::Union{Nothing,DenseCuMatrix{Float64}} = nothing)
    nbandkq, nbandk, nmodes, nq = size(ep_kq_all)
    nw = size(ukqs, 1)
    nr_ep = size(ep_kR, 2)
    @assert size(ep_kR, 1) == nw * nbandk * nmodes && size(phase) == (nr_ep, nq)
    @assert size(ukqs) == (nw, nbandkq, nq) && size(u_phs) == (nmodes, nmodes, nq)
    colstride(phase) == nr_ep || throw(ArgumentError("libepb200: the phase columns must be contiguous (stride nr)"))
    check(ccall((:epb_eph_kR_to_kq, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Int64, Int64, CuPtr{ComplexF64}, Int64,
                 CuPtr{ComplexF64}, Int64, CuPtr{ComplexF64}, CuPtr{Float64}, CuPtr{ComplexF64}, CuPtr{Float64}, Cint),
                ctx().h, ep_kR, colstride(ep_kR), nw, nbandk, nmodes, nr_ep, phase, nq, ukqs, nbandkq,
                u_phs, devptr(ωq), ep_kq_all, devptr(g2_out), PREC[]))
    ep_kq_all
end

# g arrives as reshape(view(ws.g, :, 1:nq), nw, nbandk, nmodes, nq) (wannier_to_bloch_batched.jl:270), a
# reshape of a view, hence AnyCuArray (as ext:176); its per-q stride is nw * nbandk * nmodes.
function ElectronPhonon.eph_apply_rotations!(ep_kq_all::DenseCuArray{ComplexF64,4}, g::AnyCuArray{ComplexF64,4},
        ukqs::DenseCuArray{ComplexF64,3}, u_phs::DenseCuArray{ComplexF64,3}, tmp; g2_out = nothing, ωq = nothing)
    nbandkq, nbandk, nmodes, nq = size(ep_kq_all)
    nw = size(ukqs, 1)
    @assert size(g) == (nw, nbandk, nmodes, nq)
    assert_dense(g)
    check(ccall((:epb_eph_apply_rotations, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Int64, Int64, CuPtr{ComplexF64}, Int64,
                 CuPtr{ComplexF64}, CuPtr{Float64}, CuPtr{ComplexF64}, CuPtr{Float64}),
                ctx().h, devptr(g), nw * nbandk * nmodes, nw, nbandk, nmodes, nq, ukqs, nbandkq, u_phs,
                devptr(ωq), ep_kq_all, devptr(g2_out)))
    ep_kq_all
end

# ---- energy window (filter.jl:19,40-72): band ranges and kept k without copying E to the host --
function window_filter(E::DenseCuMatrix{Float64}, wmin::Real, wmax::Real)
    nw, nk = size(E)
    bmin = CuVector{Int32}(undef, nk); bmax = CuVector{Int32}(undef, nk)
    keep = CuVector{Int32}(undef, max(nk, 1)); nkeep = CUDA.zeros(Int64, 1)
    nbelow = CuVector{Float64}(undef, nk)
    check(ccall((:epb_window_filter, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, Int64, Int64, Float64, Float64, CuPtr{Int32}, CuPtr{Int32},
                 CuPtr{Int32}, CuPtr{Int64}, CuPtr{Float64}),
                ctx().h, E, nw, nk, wmin, wmax, bmin, bmax, keep, nkeep, nbelow))
    n = Int(Array(nkeep)[1])
    bmin, bmax, keep[1:n] .+ Int32(1), nbelow   # 1-based k indices for the Julia side
end

# ---- outer-q chain (wannier_to_bloch.jl:277-300, wannier_to_bloch_batched.jl:317-377) -----------
# call site: get_eph_Rq_to_kq_batched!(ep_batch, itp_ep_eRpq, ks_batch, Uk_batch, Ukq_batch; ws = ep_ws)
# (run_eph_over_q_and_k.jl:588)
function ElectronPhonon.get_eph_Rq_to_kq_batched!(ep_kq_all::DenseCuArray{ComplexF64,4},
        itp_epobj_eRpq::ElectronPhonon.BatchedWannierInterpolator, ks, uks::DenseCuArray{ComplexF64,3},
        ukqs::DenseCuArray{ComplexF64,3}; ws = nothing)
    nbandkq, nbandk, nmodes, nk = size(ep_kq_all)
    nw = size(uks, 1)
    parent = itp_epobj_eRpq.parent
    @assert parent.ndata == nw^2 * nmodes
    check(ccall((:epb_eph_Rq_to_kq, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{ComplexF64},
                 Int64, CuPtr{ComplexF64}, Int64, CuPtr{Float64}, CuPtr{ComplexF64}, CuPtr{Float64}, Cint),
                ctx().h, parent.op_r, nw, nmodes, rset(parent.irvec).h, xk_device(ks), nk, uks, nbandk, ukqs, nbandkq,
                NULLDEV, ep_kq_all, NULLDEV, PREC[]))
    ep_kq_all
end

# g(Re, q) for a list of q from the "ph"-layout epmat (rows (i, j, nu, Re)), in the eigenmode basis u_phs
function eph_RR_to_Rq_batched!(ep_Rq_all::DenseCuArray{ComplexF64,3}, epmat::ElectronPhonon.WannierObject, xqs,
        u_phs::DenseCuArray{ComplexF64,3})
    nm = size(u_phs, 1)
    nr_el = length(epmat.irvec_next)
    nw = isqrt(div(epmat.ndata, nm * nr_el))
    check(ccall((:epb_eph_RR_to_Rq, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Ptr{Cvoid}, CuPtr{Float64}, Int64,
                 CuPtr{ComplexF64}, CuPtr{ComplexF64}, Cint),
                ctx().h, epmat.op_r, nw, nm, nr_el, rset(epmat.irvec).h, xk_device(xqs), size(u_phs, 3), u_phs,
                ep_Rq_all, PREC[]))
    ep_Rq_all
end

# ---- calculator hooks (calculator_utils.jl:36-50, boltzmann_calculator.jl:336-362) ----------------
# The extension leaves the loop-side operands untyped (ext:303, 361): they arrive as views of the loop's
# buffers (view(g2_dev, :,:,:, rng_q), view(dev.imap_i, rng, ik)). Here they are any device array
# (AnyCuArray), so these methods are the ones dispatched for every device form the extension takes; the
# library reads them through plain pointers, so a non-contiguous one is refused with an ArgumentError.
function ElectronPhonon.eph_window_scatter!(g2_out::DenseCuArray{Float64}, ωq_out::DenseCuArray{Float64},
        g2vals::AnyCuArray{Float64,4}, imap_i_col::AnyCuArray{Int,1}, imap_f::AnyCuArray{Int,2}, ikqs,
        ωq::AnyCuArray{Float64,2}, nbandkq::Int, nbandk::Int, nm::Int, nq_batch::Int, ni_stride::Int, i0::Int)
    foreach(assert_dense, (g2vals, imap_i_col, imap_f, ωq))
    ikq_d = CuArray{Int64}(collect(ikqs))
    check(ccall((:epb_eph_window_scatter, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Int64}, CuPtr{Int64}, Int64,
                 CuPtr{Int64}, CuPtr{Float64}, Int64, Int64, Int64, Int64, Int64, Int64),
                ctx().h, g2_out, ωq_out, devptr(g2vals), devptr(imap_i_col), devptr(imap_f), colstride(imap_f), ikq_d,
                devptr(ωq), nbandkq, nbandk, nm, nq_batch, ni_stride, i0))
    nothing
end

function ElectronPhonon.bte_window_accumulate!(Sₒ_out::DenseCuArray{Float64}, Sᵢ_out, g2vals::AnyCuArray{Float64,4},
        ωqmat::AnyCuArray{Float64,2}, imap_i_at_k::AnyCuArray{Int,1}, imap_f::AnyCuArray{Int,2}, ikqs, e_i, e_f, wf,
        μs, Ts, ηs, method::Int, ω_cutoff, nbandkq::Int, nbandk::Int, nmodes::Int, nq_batch::Int, i0::Int)
    foreach(assert_dense, (g2vals, ωqmat, imap_i_at_k, imap_f))
    ikq_d = CuArray{Int64}(collect(ikqs))
    dev(x) = x isa DenseCuArray{Float64} ? x : CuArray{Float64}(collect(x))
    sin_ptr = Sᵢ_out === nothing ? NULLDEV : devptr(assert_dense(Sᵢ_out))
    ni_tile, n_f = Sᵢ_out === nothing ? (0, 0) : (size(Sᵢ_out, 1), size(Sᵢ_out, 2))
    check(ccall((:epb_bte_window_accumulate, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{Float64}, Int64, Int64, CuPtr{Float64}, CuPtr{Float64},
                 CuPtr{Int64}, CuPtr{Int64}, Int64, CuPtr{Int64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64},
                 CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, Int64, Cint, Float64, Int64, Int64, Int64, Int64,
                 Int64),
                ctx().h, Sₒ_out, size(Sₒ_out, 1), sin_ptr, ni_tile, n_f, devptr(g2vals), devptr(ωqmat),
                devptr(imap_i_at_k), devptr(imap_f), colstride(imap_f), ikq_d, dev(e_i), dev(e_f), dev(wf), dev(μs),
                dev(Ts), dev(ηs), length(μs), method, ω_cutoff, nbandkq, nbandk, nmodes, nq_batch, i0))
    nothing
end

# ---- EPW reader (model_new.jl:487-568): the epmatwp file straight into HBM -----------------------
function read_epmat_device(filename, nw, nmodes, nr_el, nr_ep, irvec_el, irvec_ep, ind_el, ind_ep, ndegen_el,
        ndegen_ep, epmat_outer_momentum; skip_ndegen_ep = false, ndegen_pre_divided = false)
    layout = epmat_outer_momentum == "ph" ? Cint(1) : Cint(0)
    nd = nw^2 * nmodes
    out = layout == 0 ? CuMatrix{ComplexF64}(undef, nd * nr_ep, nr_el) : CuMatrix{ComplexF64}(undef, nd * nr_el, nr_ep)
    nel = Int32.(ndegen_el); nep = Int32.(ndegen_ep)
    check(ccall((:epb_read_epmat, LIB[]), Cint,
                (Ptr{Cvoid}, Cstring, Int64, Int64, Int64, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Int32}, Int64,
                 Ptr{Int32}, Int64, Int64, Cint, Cint, Cint, CuPtr{ComplexF64}),
                ctx().h, filename, nw, nmodes, nr_el, nr_ep, Int64.(ind_el), Int64.(ind_ep), nel, size(nel, 1),
                nep, size(nep, 1), size(nep, 2), skip_ndegen_ep, ndegen_pre_divided, layout, out))
    layout == 0 ? ElectronPhonon.WannierObject(irvec_el, out; irvec_next = irvec_ep) :
                  ElectronPhonon.WannierObject(irvec_ep, out; irvec_next = irvec_el)
end


# ---- whole e-ph pass (run_eph_over_k_and_q.jl:251-330, run the batched way) ---------------------
"""
    PassModel(model; mixed = true)

Binds a model already moved to the device (`to_device`: `el_ham.op_r`, `ph_dyn.op_r` and `epmat.op_r`
in the "el" layout as `CuMatrix{ComplexF64}`, `epmat.irvec_next` the Rp list) for `eph_pass` and
`serta`. With `mixed`, also builds the split-BF16 operand planes of the tensor-core path (one-time
cost, like `to_device`). The device operators stay owned by `model` and are kept alive here.
"""
mutable struct PassModel
    h::Ptr{Cvoid}
    nw::Int
    nm::Int
    ops::Tuple
end
function PassModel(model; mixed::Bool = true)
    ham, dyn, ep = model.el_ham, model.ph_dyn, model.epmat
    mass = model.mass isa CuArray ? model.mass : CuArray{Float64}(collect(model.mass))
    nw = isqrt(size(ham.op_r, 1))
    nm = isqrt(size(dyn.op_r, 1))
    irel = collect(reinterpret(Int64, ham.irvec))
    irph = collect(reinterpret(Int64, dyn.irvec))
    irep = collect(reinterpret(Int64, ep.irvec_next))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:epb_model_create, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Ptr{Int64}, Int64, CuPtr{ComplexF64}, CuPtr{Float64}, Int64,
                 Ptr{Int64}, Int64, CuPtr{ComplexF64}, Ptr{Int64}, Int64, Cint, Ptr{Ptr{Cvoid}}),
                ctx().h, ham.op_r, nw, irel, length(ham.irvec), dyn.op_r, mass, nm, irph, length(dyn.irvec),
                ep.op_r, irep, length(ep.irvec_next), Cint(mixed ? 1 : 0), r))
    pm = PassModel(r[], nw, nm, (ham.op_r, dyn.op_r, mass, ep.op_r))
    finalizer(x -> ccall((:epb_model_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), pm)
    pm
end

"""
    eph_pass(pm, xks, xqs; prec = DRIVER_PREC[], k_batch = 0, sample_stride = 0)

All-band e-ph pass over the k list x the q list: electrons at k and k+q, phonons at q,
g2 = |u_kq' g u_ph|^2 / (2 omega). Returns device arrays `ek` (nw x nk), `omega` (nm x nq), `g2sum`
(nm x nk, summed over bands and q) and, for `sample_stride > 0`, the full g2 blocks of every
`sample_stride`-th q, (nw, nw, nm, nsamp, nk); `k_batch <= 0` lets the library time the batch sizes.
"""
function eph_pass(pm::PassModel, xks, xqs; prec::Integer = DRIVER_PREC[], k_batch::Integer = 0, sample_stride::Integer = 0)
    xk = xk_device(xks)
    xq = xk_device(xqs)
    nk, nq = size(xk, 2), size(xq, 2)
    ek = CuArray{Float64}(undef, pm.nw, nk)
    om = CuArray{Float64}(undef, pm.nm, nq)
    g2sum = CuArray{Float64}(undef, pm.nm, nk)  # zeroed by the library
    samp = sample_stride > 0 ? CuArray{Float64}(undef, pm.nw, pm.nw, pm.nm, cld(nq, sample_stride), nk) : nothing
    stats = zeros(Int64, 4)
    check(ccall((:epb_eph_pass, LIB[]), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{Float64}, Int64, Cint, Int64, Int64,
                 CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, Ptr{Int64}),
                ctx().h, pm.h, xk, nk, xq, nq, Cint(prec), k_batch, max(sample_stride, 1), ek, om, g2sum,
                samp === nothing ? CuPtr{Float64}(0) : samp, stats))
    (ek = ek, omega = om, g2sum = g2sum, g2_sample = samp, n_elements = stats[1], k_batch = stats[2],
     rotation = stats[3], kq_form = stats[4])
end

"Capture the pass as a CUDA graph on its second call with the same buffers and replay it afterwards."
set_graph_mode(on::Bool) = check(ccall((:epb_set_graph_mode, LIB[]), Cint, (Ptr{Cvoid}, Cint), ctx().h, Cint(on)))

# ---- SERTA consumer (run_eph_over_k_and_kq.jl:792-892, electron_lbte.jl:153-185) ----------------
struct BteParams  # epb_bte_params, field for field (isbits: the C struct's layout)
    ngrid::Int64
    wmin::Float64
    wmax::Float64
    mu::Float64
    temperature::Float64
    smearing::Float64
    omega_cutoff::Float64
    spin_degeneracy::Float64
    volume::Float64
    lattice::NTuple{9,Float64}
    method::Int32
    prec::Int32
    k_batch::Int64
    pair_chunk::Int64
    shard_rank::Int64
    shard_count::Int64
end

"""
    serta(pm, ngrid, wmin, wmax, mu, T, smearing; lattice, volume, spin = 2.0, method = 5,
          omega_cutoff = ElectronPhonon.omega_acoustic, prec = DRIVER_PREC[], k_batch = 0, shard = (0, 1),
          inv_tau = false)

SERTA conductivity (3 x 3, host, in the reference's units) over commensurate ngrid^3 k = q grids.
With `shard = (rank, count)` this call takes the rank's contiguous share of the kept k and returns
that share's partial sigma: add the shards' sigmas over the ranks (`MPI.Allreduce!`, the reference's
`mpi_comm_k` split). `inv_tau = true` also returns the out-scattering rates of the window states.
"""
function serta(pm::PassModel, ngrid::Integer, wmin, wmax, mu, T, smearing; lattice::AbstractMatrix, volume,
               spin = 2.0, method::Integer = 5, omega_cutoff = ElectronPhonon.omega_acoustic,
               prec::Integer = DRIVER_PREC[], k_batch::Integer = 0, shard = (0, 1), inv_tau::Bool = false)
    p = Ref(BteParams(ngrid, wmin, wmax, mu, T, smearing, omega_cutoff, spin, volume,
                      NTuple{9,Float64}(Float64.(vec(lattice))), Int32(method), Int32(prec), k_batch, 0,
                      shard[1], shard[2]))
    cap = inv_tau ? ngrid^3 * pm.nw : 0
    it = inv_tau ? CuArray{Float64}(undef, cap) : nothing
    sigma = zeros(Float64, 9)
    stats = zeros(Int64, 4)
    check(ccall((:epb_bte_serta, LIB[]), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ref{BteParams}, Ptr{Float64}, CuPtr{Float64}, Int64, Ptr{Int64}),
                ctx().h, pm.h, p, sigma, it === nothing ? CuPtr{Float64}(0) : it, cap, stats))
    sig = reshape(sigma, 3, 3)
    inv_tau ? (sig, stats, it[1:stats[2]]) : (sig, stats)
end


# ---- band energies and windows straight from H(R) (filter.jl:40-72, 109-133; electron_state.jl:118-150) --
"Binds H(R) (`ham.op_r` a device matrix) for band-energy and window queries."
mutable struct Bands
    h::Ptr{Cvoid}
    nw::Int
    op::Any
end
function Bands(ham)
    nw = isqrt(size(ham.op_r, 1))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:epb_bands_create, LIB[]), Cint, (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Ptr{Int64}, Int64,
                Ptr{Ptr{Cvoid}}), ctx().h, ham.op_r, nw, collect(reinterpret(Int64, ham.irvec)), length(ham.irvec), r))
    b = Bands(r[], nw, ham.op_r)
    finalizer(x -> ccall((:epb_bands_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), b)
    b
end

"Ascending band energies (nw x nk) at the k list (get_el_eigen_valueonly_batched)."
function band_eigvals(b::Bands, xks; prec::Integer = DRIVER_PREC[])
    xk = xk_device(xks)
    E = CuArray{Float64}(undef, b.nw, size(xk, 2))
    check(ccall((:epb_bands_eigvals, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{Float64},
                Cint), ctx().h, b.h, xk, size(xk, 2), E, Cint(prec)))
    E
end

"Energy of one band (1-based) at every point of the k list."
function band_energy(b::Bands, xks, band::Integer; prec::Integer = DRIVER_PREC[])
    xk = xk_device(xks)
    E = CuArray{Float64}(undef, size(xk, 2))
    check(ccall((:epb_bands_band_energy, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, Int64,
                CuPtr{Float64}, Cint), ctx().h, b.h, xk, size(xk, 2), band, E, Cint(prec)))
    E
end

const WindowStats = NTuple{9,Int64}  # epb_window_stats: tested, culled, evaluated, rechecked, kept, audited,
                                     # violations, fallback_chunks, screened

"""
    bands_window(b, xks, wmin, wmax; prec, guard = 1e-3)

`_filter_kpoints` from H(R) without downloading the energies: per point the 1-based band range
(0 / 0 when empty) and the 0-based ascending list of kept points.
"""
function bands_window(b::Bands, xks, wmin, wmax; prec::Integer = DRIVER_PREC[], guard = 1e-3)
    xk = xk_device(xks)
    nk = size(xk, 2)
    bmin = CuVector{Int32}(undef, nk)
    bmax = CuVector{Int32}(undef, nk)
    keep = CuVector{Int32}(undef, nk)
    n = Ref{Int64}(0)
    st = Ref{WindowStats}(ntuple(_ -> Int64(0), 8))
    check(ccall((:epb_bands_window, LIB[]), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, Float64, Float64, Cint, Float64, CuPtr{Int32},
                 CuPtr{Int32}, CuPtr{Int32}, Ref{Int64}, Ref{WindowStats}),
                ctx().h, b.h, xk, nk, wmin, wmax, Cint(prec), guard, bmin, bmax, keep, n, st))
    (keep = keep[1:n[]], band_min = bmin, band_max = bmax, stats = st[])
end

"""
    pair_window(b, xks, xqs, wmin, wmax; mlp = C_NULL, prec, guard = 1e-3, capacity)

Kept (k, q) pairs (pair index ik * nq + iq, 0-based) with their band ranges at k + q; `mlp`, a
calibrated surrogate handle, culls pairs before the plain evaluation.
"""
function pair_window(b::Bands, xks, xqs, wmin, wmax; mlp::Ptr{Cvoid} = C_NULL, prec::Integer = DRIVER_PREC[],
                     guard = 1e-3, capacity::Integer)
    xk = xk_device(xks)
    xq = xk_device(xqs)
    pairs = CuVector{Int64}(undef, capacity)
    bmin = CuVector{Int32}(undef, capacity)
    bmax = CuVector{Int32}(undef, capacity)
    n = Ref{Int64}(0)
    st = Ref{WindowStats}(ntuple(_ -> Int64(0), 8))
    check(ccall((:epb_pair_window, LIB[]), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{Float64}, Int64, Float64, Float64, Ptr{Cvoid},
                 Cint, Float64, CuPtr{Int64}, CuPtr{Int32}, CuPtr{Int32}, Int64, Ref{Int64}, Ref{WindowStats}),
                ctx().h, b.h, xk, size(xk, 2), xq, size(xq, 2), wmin, wmax, mlp, Cint(prec), guard, pairs, bmin, bmax,
                capacity, n, st))
    (pairs = pairs[1:n[]], band_min = bmin[1:n[]], band_max = bmax[1:n[]], stats = st[])
end

# ---- uneven eigensolve batches (eigen_batched over ragged inputs, ext:80-115) ---------------------
"Eigen-decompose matrices of different orders packed in `A` (in place; orders 1..96)."
function eigen_varlen!(A::DenseCuVector{ComplexF64}, a_offset::DenseCuVector{Int64}, n::DenseCuVector{Int32}, E::DenseCuVector{Float64},
                       e_offset::DenseCuVector{Int64}; jobz::Char = 'V', prec::Integer = PREC[])
    check(ccall((:epb_eigh_varlen, LIB[]), Cint, (Ptr{Cvoid}, CuPtr{ComplexF64}, CuPtr{Int64}, CuPtr{Int32}, Int64,
                CuPtr{Float64}, CuPtr{Int64}, Cchar, Cint), ctx().h, A, a_offset, n, length(n), E, e_offset,
                Cchar(jobz), Cint(prec)))
    A, E
end

# ---- q index of k+q on a commensurate grid (_fill_iqs!, run_eph_over_k_and_kq.jl:565-582) -----------
function fill_iqs!(iqs::DenseCuVector{Int64}, xkq_int::DenseCuMatrix{Int64}, xk_int::AbstractVector{<:Integer}, ngrid,
                   dense_hash_to_iq::DenseCuVector{Int64})
    check(ccall((:epb_fill_iqs, LIB[]), Cint, (Ptr{Cvoid}, CuPtr{Int64}, Int64, Ptr{Int64}, Int64, Int64, Int64,
                CuPtr{Int64}, CuPtr{Int64}), ctx().h, xkq_int, size(xkq_int, 2), Int64.(collect(xk_int)),
                ngrid[1], ngrid[2], ngrid[3], dense_hash_to_iq, iqs))
    iqs
end

# ---- window filter without library allocations (for callers whose memory pool owns the device) ----
"""
    window_filter_noalloc(E, wmin, wmax, band_min, band_max, keep, nkeep)

The window filter on caller-owned buffers (`nkeep` a one-element device vector), using the library's
fixed static scratch (nk <= 16,777,216); calls that overlap on one device race.
"""
function window_filter_noalloc(E::DenseCuMatrix{Float64}, wmin, wmax, band_min::DenseCuVector{Int32}, band_max::DenseCuVector{Int32},
                               keep::DenseCuVector{Int32}, nkeep::DenseCuVector{Int64})
    nw, nk = size(E)
    check(ccall((:epb_window_filter_noalloc, LIB[]), Cint, (Ptr{Cvoid}, CuPtr{Float64}, Int64, Int64, Float64,
                Float64, CuPtr{Int32}, CuPtr{Int32}, CuPtr{Int32}, CuPtr{Int64}, CuPtr{Float64}),
                CUDA.stream().handle, E, nw, nk, wmin, wmax, band_min, band_max, keep, nkeep, CuPtr{Float64}(0)))
    nkeep
end


# ---- TiledDeviceOutput (calculator/tiled_device_output.jl) ------------------------------------------
struct TiledInfo  # epb_tiled_info, field for field
    allocated::Int32
    block::Int32
    ni_cap::Int64
    tile_offset::Int64
    tile_length::Int64
    tile_stride::Int64
end

"""
    TiledOutput(dims, i_axis, narr, T, iks, nk, n_batch_max; force_block = -1, headroom = 1.2)

`narr` arrays of element type `T` (4, 8 or 16 bytes) and shape `dims`, axis `i_axis` (1-based) running
over the outer states whose 1-based k indices are `iks`; resident whole, or one outer-k tile at a time
when the full output does not fit (`force_block`: -1 decide from free memory, 0 whole, 1 tiled).
"""
mutable struct TiledOutput
    h::Ptr{Cvoid}
    T::DataType
end
function TiledOutput(dims, i_axis::Integer, narr::Integer, T::DataType, iks::AbstractVector{<:Integer}, nk::Integer,
                     n_batch_max::Integer; force_block::Integer = -1, headroom = 1.2)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    d = Int64.(collect(dims))
    check(ccall((:epb_tiled_create, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Int64}, Cint, Cint, Cint, Int64, Cint, Float64,
                Ptr{Int64}, Int64, Int64, Int64, Ptr{Ptr{Cvoid}}), ctx().h, d, Cint(length(d)), Cint(i_axis - 1),
                Cint(narr), Int64(sizeof(T)), Cint(force_block), headroom, Int64.(collect(iks)), length(iks), nk,
                n_batch_max, r))
    t = TiledOutput(r[], T)
    finalizer(x -> ccall((:epb_tiled_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), t)
    t
end
"tile_begin! for the 1-based k batch kstart:kend (allocates on first use; zeroes the tile in block mode)."
tile_begin!(t::TiledOutput, kstart::Integer, kend::Integer) =
    check(ccall((:epb_tiled_begin, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int64), ctx().h, t.h, kstart, kend))
function tile_info(t::TiledOutput)
    info = Ref{TiledInfo}(TiledInfo(0, 0, 0, 0, 0, 0))
    check(ccall((:epb_tiled_get_info, LIB[]), Cint, (Ptr{Cvoid}, Ref{TiledInfo}), t.h, info))
    info[]
end
"Device pointer of array k (1-based) for the scatter kernels (tile_offset / tile_stride apply)."
function device_pointer(t::TiledOutput, k::Integer)
    p = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:epb_tiled_device_array, LIB[]), Cint, (Ptr{Cvoid}, Cint, Ptr{Ptr{Cvoid}}), t.h, Cint(k - 1), p))
    CuPtr{t.T}(UInt(p[]))
end
"tile_download!: array k (1-based) of the current tile (block mode) or the whole array into `host`."
function tile_download!(host::Array, t::TiledOutput, k::Integer)
    check(ccall((:epb_tiled_download, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}), ctx().h, t.h,
                Cint(k - 1), host))
    host
end
tile_free!(t::TiledOutput) = check(ccall((:epb_tiled_free, LIB[]), Cint, (Ptr{Cvoid},), t.h))

"residency_use_block: would the full output (bytes, times headroom) not fit the free device memory?"
function residency_use_block(full_bytes::Integer, headroom = 1.2)
    b = Ref{Cint}(0)
    check(ccall((:epb_residency_use_block, LIB[]), Cint, (Ptr{Cvoid}, Int64, Float64, Ref{Cint}), ctx().h,
                full_bytes, headroom, b))
    b[] != 0
end
"ind_range_for_k_range: the 1-based (first, last) states of k range kstart:kend ((1, 0) when empty)."
function ind_range_for_k_range(iks::AbstractVector{<:Integer}, nk::Integer, kstart::Integer, kend::Integer)
    f = Ref{Int64}(0)
    l = Ref{Int64}(0)
    check(ccall((:epb_ind_range_for_k_range, LIB[]), Cint, (Ptr{Int64}, Int64, Int64, Int64, Int64, Ref{Int64},
                Ref{Int64}), Int64.(collect(iks)), length(iks), nk, kstart, kend, f, l))
    f[]:l[]
end


# ---- outer-q loop with EPDataKBatched calculators (run_eph_over_q_and_k.jl:428-613) -------------------
struct OuterQParams  # epb_outer_q_params
    wmin_k::Float64
    wmax_k::Float64
    wmin_kq::Float64
    wmax_kq::Float64
    k_batch::Int64
    q_chunk::Int64
    prec::Cint
    phonon_basis::Cint
end
struct KBatchPayload  # epb_kbatch_payload: device pointers valid during run_batch, ordered on `stream`
    iq::Int64
    k0::Int64
    nk::Int64
    nw::Int64
    nm::Int64
    eps::Ptr{ComplexF64}
    ek::Ptr{Float64}
    ekq::Ptr{Float64}
    uk::Ptr{ComplexF64}
    ukq::Ptr{ComplexF64}
    wtk::Ptr{Float64}
    xk::Ptr{Float64}
    ik::Ptr{Int32}
    omega::Ptr{Float64}
    stream::Ptr{Cvoid}
end
struct OuterQCalc  # epb_outer_q_calc
    begin_q::Ptr{Cvoid}
    run_batch::Ptr{Cvoid}
    end_q::Ptr{Cvoid}
    user::Ptr{Cvoid}
end

# The hooks a calculator (a mutable object) implements: the OuterIteration brackets and
# run_calculator!(::EPDataKBatched); the payload's device pointers become CuArrays with
# unsafe_wrap(CuArray, CuPtr{T}(UInt(ptr)), dims) for the duration of the call.
outer_q_begin!(calc, iq) = nothing
outer_q_end!(calc, iq) = nothing
function outer_q_run_batch! end

function _oq_begin(user::Ptr{Cvoid}, iq::Int64, stream::Ptr{Cvoid})::Cint
    try
        outer_q_begin!(unsafe_pointer_to_objref(user), iq + 1)
        return Cint(0)
    catch
        return Cint(1)
    end
end
function _oq_run(user::Ptr{Cvoid}, p::Ptr{KBatchPayload})::Cint
    try
        outer_q_run_batch!(unsafe_pointer_to_objref(user), unsafe_load(p))
        return Cint(0)
    catch
        return Cint(1)  # the library stops the loop and returns EPB_ERR_ARG
    end
end
function _oq_end(user::Ptr{Cvoid}, iq::Int64, stream::Ptr{Cvoid})::Cint
    try
        outer_q_end!(unsafe_pointer_to_objref(user), iq + 1)
        return Cint(0)
    catch
        return Cint(1)
    end
end

"""
    eph_outer_q(pm, xks, xqs, calcs; window_k, window_kq, wtk = nothing, prec = DRIVER_PREC[], k_batch = 0,
                q_chunk = 0, phonon_basis = 0)

The outer-q batched loop: per q, g(Re, q) and the phonon modes, then per batch of kept k the k+q states
and ep = ukq' g(k, q) uk, handed to each calculator's `outer_q_run_batch!`. Returns the gauge-invariant
record A[iq] = sum_k wtk sum |ep|^2 and the stats (kept k, k batch, q chunk, batches).
"""
function eph_outer_q(pm::PassModel, xks, xqs, calcs::AbstractVector; window_k, window_kq, wtk = nothing,
                     prec::Integer = DRIVER_PREC[], k_batch::Integer = 0, q_chunk::Integer = 0, phonon_basis::Integer = 0)
    xk = collect(reinterpret(reshape, Float64, collect(Vec3{Float64}, xks)))  # host 3 x nk
    xq = collect(reinterpret(reshape, Float64, collect(Vec3{Float64}, xqs)))
    nk, nq = size(xk, 2), size(xq, 2)
    w = wtk === nothing ? nothing : Float64.(collect(wtk))
    params = Ref(OuterQParams(window_k[1], window_k[2], window_kq[1], window_kq[2], k_batch, q_chunk, Cint(prec),
                              Cint(phonon_basis)))
    fb = @cfunction(_oq_begin, Cint, (Ptr{Cvoid}, Int64, Ptr{Cvoid}))
    fr = @cfunction(_oq_run, Cint, (Ptr{Cvoid}, Ptr{KBatchPayload}))
    fe = @cfunction(_oq_end, Cint, (Ptr{Cvoid}, Int64, Ptr{Cvoid}))
    A = zeros(Float64, nq)
    stats = zeros(Int64, 4)
    GC.@preserve calcs begin
        cs = [OuterQCalc(fb, fr, fe, pointer_from_objref(c)) for c in calcs]
        check(ccall((:epb_eph_outer_q, LIB[]), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ref{OuterQParams},
                     Ptr{OuterQCalc}, Cint, Ptr{Float64}, Ptr{Int64}),
                    ctx().h, pm.h, xk, w === nothing ? Ptr{Float64}(C_NULL) : w, nk, xq, nq, params, cs,
                    Cint(length(cs)), A, stats))
    end
    A, stats
end


# ---- learned band-energy surrogate for the pair window (no counterpart in the reference) ------------
struct MlpTrainOpts  # epb_mlp_train_opts
    epochs::Int64
    batch::Int64
    lr::Float64
    lr_final::Float64
    seed::UInt64
    use_graph::Int32
    reserved::Int32
end

"""
    Surrogate(fvecs, nout; hidden = 256, nhidden = 3, seed = 1)

MLP on the Fourier features [cos 2 pi f.k, sin 2 pi f.k] of the integer vectors `fvecs` (e.g. the H(R)
lattice vectors), predicting `nout` band energies. Train it with `train!`, calibrate its culling margins
on held-out points with `calibrate!`, then pass `s.h` as `mlp` to `pair_window`.
"""
mutable struct Surrogate
    h::Ptr{Cvoid}
    nout::Int
end
function Surrogate(fvecs::Vector{Vec3{Int}}, nout::Integer; hidden::Integer = 256, nhidden::Integer = 3,
                   seed::Integer = 1)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    f = Int32.(collect(reinterpret(Int64, fvecs)))
    check(ccall((:epb_mlp_create, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Int32}, Int64, Int64, Int64, Int64, UInt64,
                Ptr{Ptr{Cvoid}}), ctx().h, f, length(fvecs), hidden, nhidden, nout, UInt64(seed), r))
    m = Surrogate(r[], nout)
    finalizer(x -> ccall((:epb_mlp_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), m)
    m
end

"Adam training on points `xks` with band energies `E` (nout x n, device); returns the loss of each epoch."
function train!(m::Surrogate, xks, E::DenseCuMatrix{Float64}; epochs::Integer = 200, batch::Integer = 2048,
                lr = 2e-3, lr_final = 2e-5, seed::Integer = 1, use_graph::Bool = true)
    x = xk_device(xks)
    opts = Ref(MlpTrainOpts(epochs, batch, lr, lr_final, UInt64(seed), Int32(use_graph), Int32(0)))
    loss = zeros(Float64, epochs)
    check(ccall((:epb_mlp_train, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64,
                Ref{MlpTrainOpts}, Ptr{Float64}), ctx().h, m.h, x, E, size(x, 2), opts, loss))
    loss
end

"Culling margins from held-out points: safety x the largest prediction error of each band."
function calibrate!(m::Surrogate, xks, E::DenseCuMatrix{Float64}; safety = 1.5)
    x = xk_device(xks)
    margins = zeros(Float64, m.nout)
    check(ccall((:epb_mlp_calibrate, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64,
                Float64, Ptr{Float64}), ctx().h, m.h, x, E, size(x, 2), safety, margins))
    margins
end

"Predicted band energies (nout x n) at the points `xks`."
function predict(m::Surrogate, xks)
    x = xk_device(xks)
    E = CuArray{Float64}(undef, m.nout, size(x, 2))
    check(ccall((:epb_mlp_predict, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{Float64}),
                ctx().h, m.h, x, size(x, 2), E))
    E
end

end # module
