# DiffMoMB200.jl -- ccall layer a DiffMoM.jl maintainer adds to reach
# libdiffmom_b200.so (source only; Julia is not part of this build).
module DiffMoMB200
using ..DiffMoM: TriMesh, RWGData, PlaneWaveExcitation
const lib = get(ENV, "DIFFMOM_B200_LIB", "libdiffmom_b200")

struct GmresStats; niter::Int32; solved::Int32; residual::Float64
    true_residual::Float64; restarts::Int32; reserved::Int32; end

function check(ctx, st)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:dmb_last_error, lib), Cstring, (Ptr{Cvoid},), ctx))
    st in (1, 4) && throw(ArgumentError(msg))
    st == 2 && throw(OverflowError(msg))
    st == 3 && throw(DimensionMismatch(msg))
    error(msg)
end

mutable struct Device
    ptr::Ptr{Cvoid}
    function Device(mesh::TriMesh, rwg::RWGData; device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:dmb_ctx_create, lib), Cint, (Cint, Ref{Ptr{Cvoid}}), device, r)
        st == 0 || error("dmb_ctx_create failed ($st)")
        d = new(r[]); finalizer(x -> ccall((:dmb_ctx_destroy, lib), Cint, (Ptr{Cvoid},), x.ptr), d)
        GC.@preserve mesh begin
            check(d.ptr, ccall((:dmb_mesh_upload, lib), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}, Int64, Int64),
                d.ptr, mesh.xyz, mesh.tri, size(mesh.xyz, 2), size(mesh.tri, 2)))
        end
        GC.@preserve rwg begin
            check(d.ptr, ccall((:dmb_rwg_upload, lib), Cint,
                (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64},
                 Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                d.ptr, rwg.nedges, rwg.tplus, rwg.tminus, rwg.evert, rwg.vplus_opp,
                rwg.vminus_opp, rwg.len, rwg.area_plus, rwg.area_minus))
        end
        return d
    end
end

# assemble_Z_efie(mesh, rwg, k; ...) with the matrix computed on the GPU
function assemble_Z_efie_gpu(d::Device, N, k; quad_order=3, eta0=376.730313668,
                             precision=:fp64, copy_out=true)
    Z = copy_out ? Matrix{ComplexF64}(undef, N, N) : nothing
    check(d.ptr, ccall((:dmb_assemble_z, lib), Cint,
        (Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{ComplexF64}),
        d.ptr, k, eta0, quad_order, precision === :fp64 ? 0 : 1,
        copy_out ? Z : Ptr{ComplexF64}(C_NULL)))
    return Z
end

# build_nearfield_preconditioner(Z, mesh, rwg, cutoff; factorization=:lu|:diag)
nf_build!(d::Device, cutoff; factorization=:lu) = check(d.ptr, ccall((:dmb_nf_build, lib),
    Cint, (Ptr{Cvoid}, Cdouble, Cint, Ptr{Cdouble}), d.ptr, cutoff,
    factorization === :lu ? 1 : 2, C_NULL))

# solve_gmres(Z, rhs; preconditioner, precond_side, tol, maxiter) on the device
function solve_gmres_gpu(d::Device, rhs::Vector{ComplexF64}; tol=1e-8, maxiter=200,
                         preconditioner=:nf_lu, precond_side=:left,
                         check_gmres_convergence=true)
    x = similar(rhs); st = Ref{GmresStats}()
    kind = preconditioner === :none ? 0 : preconditioner === :nf_lu ? 1 : 2
    check(d.ptr, ccall((:dmb_gmres, lib), Cint,
        (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}, Int64, Cdouble, Cint, Cint, Cint, Cint,
         Ref{GmresStats}),
        d.ptr, rhs, x, 1, tol, maxiter, kind, precond_side === :left ? 0 : 1,
        check_gmres_convergence ? 1 : 0, st))
    return x, st[]
end
# build_aca_operator(mesh, rwg, k; ...) on the GPU; the device's operator is
# then the H-matrix (solve_gmres_gpu runs on it until the next assembly)
function build_aca_operator_gpu(d::Device, k; leaf_size=64, eta=1.5, aca_tol=1e-6, max_rank=50,
                                quad_order=3, eta0=376.730313668, max_block_tasks=2_000_000,
                                max_storage_bytes=2_000_000_000)
    info = zeros(UInt8, 80)   # dmb_aca_info: 6 x Int64 + 4 x Float64
    check(d.ptr, ccall((:dmb_aca_build, lib), Cint,
        (Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Cdouble, Cdouble, Cint, Int64, Int64, Ptr{UInt8}),
        d.ptr, k, eta0, quad_order, leaf_size, eta, aca_tol, max_rank, max_block_tasks,
        max_storage_bytes, info))
    return reinterpret(Int64, info[1:48]), reinterpret(Float64, info[49:80])
end

# matrixfree_efie_operator(mesh, rwg, k; ...) then mul!(y, A, x) on the device
# (entries recomputed on every product; nothing of size N^2 is stored)
prepare_operator!(d::Device, k; quad_order=3, eta0=376.730313668) = check(d.ptr,
    ccall((:dmb_prepare_operator, lib), Cint, (Ptr{Cvoid}, Cdouble, Cdouble, Cint), d.ptr, k, eta0, quad_order))
function matvec_free_gpu!(d::Device, y::Vector{ComplexF64}, x::Vector{ComplexF64})
    check(d.ptr, ccall((:dmb_matvec_free, lib), Cint, (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}),
                       d.ptr, x, y))
    return y
end
# The same product for callers that must not allocate device memory once set
# up (a CuArray pool that owns the device memory, a fixed budget): x and y are
# device vectors, e.g. pointer(x::CuVector{ComplexF64}); at most 32,768
# triangles; calls on one device must not overlap.
matvec_free_noalloc!(d::Device, y_dev::Ptr{ComplexF64}, x_dev::Ptr{ComplexF64}) = check(d.ptr,
    ccall((:dmb_matvec_free_noalloc, lib), Cint, (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}),
          d.ptr, x_dev, y_dev))

# build_nearfield_preconditioner(A_aca; factorization) from the H-matrix's dense blocks
aca_nf_build!(d::Device; factorization=:lu, precision=:fp64) = check(d.ptr,
    ccall((:dmb_aca_nf_build, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}),
          d.ptr, factorization === :lu ? 1 : 2, precision === :fp64 ? 0 : 1, C_NULL))
end # module
