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
const PREC = Ref{Cint}(1)  # 0: plain FP64, 1: split-BF16 tensor cores + FP32/FP64 eigensolve

last_error() = unsafe_string(ccall((:epb_last_error, LIB[]), Cstring, ()))
check(st::Integer) = st == 0 || error("libepb200: status $st: $(last_error())")

# ---- context: one per task (the reference's batched loop is single-threaded) -----------------
mutable struct Ctx
    h::Ptr{Cvoid}
end
const CTX = Dict{Tuple{Int,UInt},Ctx}()
function ctx()
    dev = CUDA.deviceid(CUDA.device())
    s = CUDA.stream()
    key = (dev, UInt(pointer_from_objref(s)))
    get!(CTX, key) do
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:epb_create, LIB[]), Cint, (Ptr{Ptr{Cvoid}}, Cint, Ptr{Cvoid}), r, dev, s.handle))
        c = Ctx(r[])
        finalizer(x -> ccall((:epb_destroy, LIB[]), Cint, (Ptr{Cvoid},), x.h), c)
        c
    end
end

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

xk_device(xks) = CuArray(reinterpret(reshape, Float64, collect(Vec3{Float64}, xks)))  # 3 x nk

# ---- backend (ext:34-37) -----------------------------------------------------------------------
function ElectronPhonon.free_bytes(::ElectronPhonon.GPUBackend)
    f = Ref{UInt64}(0); t = Ref{UInt64}(0)
    check(ccall((:epb_free_bytes, LIB[]), Cint, (Ptr{Cvoid}, Ref{UInt64}, Ref{UInt64}), ctx().h, f, t))
    Int(f[])
end
ElectronPhonon.synchronize(::ElectronPhonon.GPUBackend) =
    check(ccall((:epb_synchronize, LIB[]), Cint, (Ptr{Cvoid},), ctx().h))

# ---- Fourier (batched_fourier_core.jl:24-30, 117-139) ----------------------------------------
function ElectronPhonon.fourier_phase!(phase::CuMatrix{ComplexF64}, irvec::Vector{Vec3{Int}}, xks)
    xk = xk_device(xks)
    check(ccall((:epb_fourier_phase, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{ComplexF64}),
                ctx().h, rset(irvec).h, xk, size(xk, 2), phase))
    phase
end

function ElectronPhonon.get_fourier_batched!(out::CuMatrix{ComplexF64},
        itp::ElectronPhonon.BatchedWannierInterpolator, xks)
    p = itp.parent
    xk = xk_device(xks)
    @assert size(out) == (p.ndata, size(xk, 2))
    check(ccall((:epb_fourier, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{ComplexF64}, Cint),
                ctx().h, p.op_r, size(p.op_r, 1), p.ndata, rset(p.irvec).h, xk, size(xk, 2), out, PREC[]))
    out
end

# ---- eigensolves (ext:80-115) -----------------------------------------------------------------
function ElectronPhonon.eigvals_batched(Hk::CuArray{ComplexF64,3})
    nw, _, nk = size(Hk)
    E = CuArray{Float64}(undef, nw, nk)
    check(ccall((:epb_eigh_batched, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, CuPtr{Float64}, Cchar, Cint),
                ctx().h, Hk, nw, nk, E, 'N', PREC[]))
    E
end

function ElectronPhonon.eigen_batched(Hk::CuArray{ComplexF64,3})
    nw, _, nk = size(Hk)
    E = CuArray{Float64}(undef, nw, nk)
    check(ccall((:epb_eigh_batched, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, CuPtr{Float64}, Cchar, Cint),
                ctx().h, Hk, nw, nk, E, 'V', PREC[]))
    E, Hk  # eigenvectors overwrite Hk (destroy-input contract)
end

# phonons: D(q) / sqrt(m_i m_j) -> eigen -> omega = sign sqrt, u ./= sqrt(m) (compute_states.jl:293-300)
function phonon_eigen_batched!(Dq::CuArray{ComplexF64,3}, mass::CuVector{Float64})
    nm, _, nq = size(Dq)
    ω = CuArray{Float64}(undef, nm, nq)
    check(ccall((:epb_ph_eigen_batched, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, CuPtr{Float64}, Int64, Int64, CuPtr{Float64}, Cint),
                ctx().h, Dq, mass, nm, nq, ω, PREC[]))
    ω, Dq
end

# ---- e-ph chain (wannier_to_bloch_batched.jl:178-273, 442-455) -------------------------------
function ElectronPhonon.get_eph_RR_to_kR_batched!(ep_ekpR_all::CuArray{ComplexF64,3},
        itp_epmat::ElectronPhonon.BatchedWannierInterpolator, ks, uks::CuArray{ComplexF64,3};
        additional_phase = nothing)
    epmat = itp_epmat.parent
    nr_ep = length(epmat.irvec_next)
    nw, nband, nk = size(uks)
    nmodes = div(epmat.ndata, nw^2 * nr_ep)
    xk = xk_device(ks)
    ph = additional_phase === nothing ? CU_NULL : pointer(additional_phase)
    check(ccall((:epb_eph_RR_to_kR, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Ptr{Cvoid}, CuPtr{Float64}, Int64,
                 CuPtr{ComplexF64}, Int64, CuPtr{ComplexF64}, CuPtr{ComplexF64}, Cint),
                ctx().h, epmat.op_r, nw, nmodes, nr_ep, rset(epmat.irvec).h, xk, nk, uks, nband, ph,
                ep_ekpR_all, PREC[]))
    ep_ekpR_all
end

function ElectronPhonon.get_eph_kR_to_kq_batched!(ep_kq_all::CuArray{ComplexF64,4}, ep_kR::CuMatrix{ComplexF64},
        phase::CuMatrix{ComplexF64}, u_phs, ukqs; ws = nothing, g2_out = nothing, ωq = nothing)
    nbandkq, nbandk, nmodes, nq = size(ep_kq_all)
    nw = size(ukqs, 1)
    check(ccall((:epb_eph_kR_to_kq, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Int64, Int64, CuPtr{ComplexF64}, Int64,
                 CuPtr{ComplexF64}, Int64, CuPtr{ComplexF64}, CuPtr{Float64}, CuPtr{ComplexF64}, CuPtr{Float64}, Cint),
                ctx().h, ep_kR, size(ep_kR, 1), nw, nbandk, nmodes, size(ep_kR, 2), phase, nq, ukqs, nbandkq,
                u_phs, ωq === nothing ? CU_NULL : ωq, ep_kq_all, g2_out === nothing ? CU_NULL : g2_out, PREC[]))
    ep_kq_all
end

function ElectronPhonon.eph_apply_rotations!(ep_kq_all::CuArray{ComplexF64,4}, g::CuArray{ComplexF64,4},
        ukqs::CuArray, u_phs::CuArray, tmp; g2_out = nothing, ωq = nothing)
    nbandkq, nbandk, nmodes, nq = size(ep_kq_all)
    nw = size(ukqs, 1)
    check(ccall((:epb_eph_apply_rotations, LIB[]), Cint,
                (Ptr{Cvoid}, CuPtr{ComplexF64}, Int64, Int64, Int64, Int64, Int64, CuPtr{ComplexF64}, Int64,
                 CuPtr{ComplexF64}, CuPtr{Float64}, CuPtr{ComplexF64}, CuPtr{Float64}),
                ctx().h, g, nw * nbandk * nmodes, nw, nbandk, nmodes, nq, ukqs, nbandkq, u_phs,
                ωq === nothing ? CU_NULL : ωq, ep_kq_all, g2_out === nothing ? CU_NULL : g2_out))
    ep_kq_all
end

# ---- energy window (filter.jl:19,40-72): band ranges and kept k without copying E to the host --
function window_filter(E::CuMatrix{Float64}, wmin::Real, wmax::Real)
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

end # module
