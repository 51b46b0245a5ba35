# Julia-side shim: the reference's RK4 hot-path API on top of libmpsb200 (ccall).
#
# UNVERIFIED: Julia is not installed in the build image, so this file has never been run.
# It targets Julia >= 1.6 (the reference itself needs Julia 0.6.4, whose `ccall` syntax is
# the same).  Host tensors keep the reference layouts (Array{ComplexF64,3} sites,
# Array{ComplexF64,4} MPO sites), so `pointer(A[j])` is passed straight to the C ABI.
module MatrixProductStatesB200

const LIB = joinpath(@__DIR__, "..", "mpsb200", "libmpsb200.so")

struct MpsbError <: Exception
    status::Cint
    func::Symbol
    msg::String
end

function check(st, f)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:mpsb_last_error, LIB), Cstring, ()))
    st == -2 && throw(DimensionMismatch("$f: $msg"))
    throw(MpsbError(st, f, msg))
end

mutable struct Ctx
    h::Ptr{Cvoid}
end
function Ctx(device::Integer = 0)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mpsb_ctx_create, LIB), Cint, (Cint, Ptr{Ptr{Cvoid}}), device, r), :mpsb_ctx_create)
    c = Ctx(r[])
    finalizer(x -> ccall((:mpsb_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), c)
    return c
end

# Device MPS / MPO / env handles ("TA = GPU" of the reference's TN/TA type parameters)
mutable struct DMPS
    h::Ptr{Cvoid}
    dims::Vector{Int64}
    d::Int
end
mutable struct DMPO
    h::Ptr{Cvoid}
    w::Vector{Int64}
    d::Int
end
mutable struct DEnv
    h::Ptr{Cvoid}
end

function DMPS(ctx::Ctx, A::Vector{<:Array{ComplexF64,3}})
    dims = Int64[1; [size(a, 3) for a in A]]
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mpsb_mps_create, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Int64}, Ptr{Ptr{Cvoid}}),
                ctx.h, length(A), size(A[1], 2), dims, r), :mpsb_mps_create)
    m = DMPS(r[], dims, size(A[1], 2))
    for (j, a) in enumerate(A)
        check(ccall((:mpsb_mps_set_site, LIB), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), m.h, j, a),
              :mpsb_mps_set_site)
    end
    finalizer(x -> ccall((:mpsb_mps_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), m)
    return m
end

function collect_sites(m::DMPS)
    na = length(m.dims) - 1
    out = Vector{Array{ComplexF64,3}}(undef, na)
    for j in 1:na
        a = Array{ComplexF64,3}(undef, m.dims[j], m.d, m.dims[j+1])
        check(ccall((:mpsb_mps_get_site, LIB), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), m.h, j, a),
              :mpsb_mps_get_site)
        out[j] = a
    end
    return out
end

function DMPO(ctx::Ctx, O::Vector{<:Array{ComplexF64,4}})
    w = Int64[1; [size(o, 3) for o in O]]
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mpsb_mpo_create, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Int64}, Ptr{Ptr{Cvoid}}),
                ctx.h, length(O), size(O[1], 2), w, r), :mpsb_mpo_create)
    m = DMPO(r[], w, size(O[1], 2))
    for (j, o) in enumerate(O)
        check(ccall((:mpsb_mpo_set_site, LIB), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), m.h, j, o),
              :mpsb_mpo_set_site)
    end
    finalizer(x -> ccall((:mpsb_mpo_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), m)
    return m
end

# update_h!/update_L_spin_model! refresh one MPO site in place (same device buffer)
set_site!(m::DMPO, j::Integer, o::Array{ComplexF64,4}) =
    check(ccall((:mpsb_mpo_set_site, LIB), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), m.h, j, o), :mpsb_mpo_set_site)

# build_env(TN, TA, dims1, dims2[, mpo_dims])   src/constructors.jl:347-375
function build_env(ctx::Ctx, dims1::Vector{<:Integer}, dims2::Vector{<:Integer}, mpo_dims = nothing)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    wptr = mpo_dims === nothing ? Ptr{Int64}(C_NULL) : pointer(Int64.(mpo_dims))
    w = mpo_dims === nothing ? Int64[] : Int64.(mpo_dims)
    GC.@preserve w begin
        check(ccall((:mpsb_env_create, LIB), Cint,
                    (Ptr{Cvoid}, Cint, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Ptr{Cvoid}}),
                    ctx.h, length(dims1) - 1, Int64.(dims1), Int64.(dims2),
                    mpo_dims === nothing ? C_NULL : pointer(w), r), :mpsb_env_create)
    end
    e = DEnv(r[])
    finalizer(x -> ccall((:mpsb_env_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), e)
    return e
end

# RK4stp_apply_H_half!(dt, H, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop)
#   src/timeevolution.jl:188-196; the 10-argument in-place form passes psi twice.
function RK4stp_apply_H_half!(ctx::Ctx, dt::Real, H::Vector{DMPO}, psi0::DMPS, psi::DMPS, psi1::DMPS,
                              psi2::DMPS, psi3::DMPS, env1::DEnv, env2::DEnv, env3::DEnv, envop::DEnv)
    check(ccall((:mpsb_rk4stp_apply_H_half, LIB), Cint,
                (Ptr{Cvoid}, Cdouble, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid},
                 Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                ctx.h, dt, H[1].h, H[2].h, H[3].h, psi0.h, psi.h, psi1.h, psi2.h, psi3.h,
                env1.h, env2.h, env3.h, envop.h), :mpsb_rk4stp_apply_H_half)
end
RK4stp_apply_H_half!(ctx::Ctx, dt::Real, H::Vector{DMPO}, psi::DMPS, psi1::DMPS, psi2::DMPS, psi3::DMPS,
                     env1::DEnv, env2::DEnv, env3::DEnv, envop::DEnv) =
    RK4stp_apply_H_half!(ctx, dt, H, psi, psi, psi1, psi2, psi3, env1, env2, env3, envop)

# compress_var_apply_H!(A0, envop, Ain, A, H, maxsweeps)   src/compression.jl:217-258
compress_var_apply_H!(ctx::Ctx, A0::DMPS, envop::DEnv, Ain::DMPS, A::DMPS, H::DMPO, maxsweeps::Integer) =
    check(ccall((:mpsb_compress_var_apply_H, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint),
                ctx.h, A0.h, envop.h, Ain.h, A.h, H.h, maxsweeps), :mpsb_compress_var_apply_H)

# compress_sum_var_apply_H!(A0, envop, coef, A, H, maxsweeps)   src/compression.jl:805-887
function compress_sum_var_apply_H!(ctx::Ctx, A0::DMPS, envop::DEnv, coef::Vector{<:Number}, A::Vector{DMPS},
                                   H::DMPO, maxsweeps::Integer)
    c = ComplexF64.(coef)
    hs = [a.h for a in A]
    GC.@preserve c hs check(ccall((:mpsb_compress_sum_var_apply_H, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{ComplexF64}, Cint, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}, Cint),
        ctx.h, A0.h, envop.h, c, length(c), hs, H.h, maxsweeps), :mpsb_compress_sum_var_apply_H)
end

# compress_sum_var(Ain, coef, A, maxsweeps)   src/compression.jl:496-565 (A0 = the new MPS)
function compress_sum_var!(ctx::Ctx, A0::DMPS, Ain::DMPS, coef::Vector{<:Number}, A::Vector{DMPS},
                           maxsweeps::Integer)
    c = ComplexF64.(coef)
    hs = [a.h for a in A]
    GC.@preserve c hs check(ccall((:mpsb_compress_sum_var, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{ComplexF64}, Cint, Ptr{Ptr{Cvoid}}, Cint),
        ctx.h, A0.h, Ain.h, c, length(c), hs, maxsweeps), :mpsb_compress_sum_var)
end

# ground_state_search!(At, H, maxsweeps, converge_rat, eigs_tol)   src/groundstate.jl:67-147
function ground_state_search!(ctx::Ctx, At::DMPS, H::DMPO, maxsweeps::Integer, converge_rat::Real, eigs_tol::Real)
    ae = Ref{Cdouble}(0)
    check(ccall((:mpsb_ground_state_search, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cdouble, Cdouble, Ref{Cdouble}),
                ctx.h, At.h, H.h, maxsweeps, converge_rat, eigs_tol, ae), :mpsb_ground_state_search)
    return ae[]
end

# normalize_lo!(mps)   src/orthonormalisation.jl:97-103
# Contraction precision of the sweeps (no reference counterpart): 0 = FP64, 3..7 = int8 slices on
# the tensor cores for GEMMs of at least `min_tiles` output tiles.
set_precision!(ctx::Ctx, slices::Integer, min_tiles::Integer = 64) =
    check(ccall((:mpsb_ctx_set_precision, LIB), Cint, (Ptr{Cvoid}, Cint, Cint), ctx.h, slices, min_tiles),
          :mpsb_ctx_set_precision)
# batched calls: the sliced path from min_flops = 8 M N K of one copy's GEMM (the autotuned value)
set_batched_split_threshold!(ctx::Ctx, min_flops::Real) =
    check(ccall((:mpsb_ctx_set_batched_split_threshold, LIB), Cint, (Ptr{Cvoid}, Cdouble), ctx.h, min_flops),
          :mpsb_ctx_set_batched_split_threshold)

# B copies of the sites A (a batch handle: every engine call on it runs all copies per kernel)
function DMPS(ctx::Ctx, A::Vector{<:Array{ComplexF64,3}}, B::Integer)
    dims = Int64[1; [size(a, 3) for a in A]]
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mpsb_mps_create_batch, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Int64}, Cint, Ptr{Ptr{Cvoid}}),
                ctx.h, length(A), size(A[1], 2), dims, B, r), :mpsb_mps_create_batch)
    m = DMPS(r[], dims, size(A[1], 2))
    for b in 0:B-1, (j, a) in enumerate(A)
        check(ccall((:mpsb_mps_set_site_copy, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{ComplexF64}), m.h, b, j, a),
              :mpsb_mps_set_site_copy)
    end
    finalizer(x -> ccall((:mpsb_mps_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), m)
    return m
end

# normalize_lo! of every copy of a batch handle: the norms^2 before scaling
function normalize_lo_batch!(ctx::Ctx, A::DMPS, B::Integer)
    no = zeros(Float64, B)
    check(ccall((:mpsb_normalize_lo_batch, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}), ctx.h, A.h, no),
          :mpsb_normalize_lo_batch)
    return no
end

function normalize_lo!(ctx::Ctx, A::DMPS)
    no = Ref{Cdouble}(0)
    check(ccall((:mpsb_normalize_lo, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Cdouble}), ctx.h, A.h, no),
          :mpsb_normalize_lo)
    return no[]
end

# scal_prod_no_conj(mps1, mps2)   src/MatrixProductStates.jl:366-379
function scal_prod_no_conj(ctx::Ctx, A::DMPS, B::DMPS)
    out = zeros(Cdouble, 2)
    check(ccall((:mpsb_scal_prod_no_conj, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cdouble}),
                ctx.h, A.h, B.h, out), :mpsb_scal_prod_no_conj)
    return complex(out[1], out[2])
end

# Wrap a handle the library created (its dims read back through mpsb_mps_info)
function wrap_new_mps(h::Ptr{Cvoid})
    na, d = Ref{Cint}(0), Ref{Cint}(0)
    check(ccall((:mpsb_mps_info, LIB), Cint, (Ptr{Cvoid}, Ref{Cint}, Ref{Cint}, Ptr{Int64}), h, na, d, C_NULL),
          :mpsb_mps_info)
    dims = zeros(Int64, na[] + 1)
    check(ccall((:mpsb_mps_info, LIB), Cint, (Ptr{Cvoid}, Ref{Cint}, Ref{Cint}, Ptr{Int64}), h, na, d, dims),
          :mpsb_mps_info)
    m = DMPS(h, dims, Int(d[]))
    finalizer(x -> ccall((:mpsb_mps_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), m)
    return m
end

# compressionSVD!(mps, dmax, tol)   src/compression.jl:1280-1312
# Returns (new MPS with the truncated bond dims, err_glob, err_trim, ent_ent); the reference
# resizes `mps` in place, here the result is a new handle.
function compressionSVD!(ctx::Ctx, A::DMPS, dmax::Integer, tol::Real)
    na = length(A.dims) - 1
    out = Ref{Ptr{Cvoid}}(C_NULL)
    err_glob = Ref{Cdouble}(0)
    err_trim, ent = zeros(Cdouble, na), zeros(Cdouble, na)
    check(ccall((:mpsb_compression_svd, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cdouble, Ptr{Ptr{Cvoid}}, Ref{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                ctx.h, A.h, dmax, tol, out, err_glob, err_trim, ent), :mpsb_compression_svd)
    return wrap_new_mps(out[]), err_glob[], err_trim, ent
end

# compress_var_apply_H_two_site(Ain, A, H, maxsweeps, svd_tol, dims, dlim)   src/compression.jl:355-411
# Returns the compressed MPS (new handle; its `dims` are the reference's updated dims).
function compress_var_apply_H_two_site(ctx::Ctx, Ain::DMPS, A::DMPS, H::DMPO, maxsweeps::Integer,
                                       svd_tol::Real, dlim::Integer)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mpsb_compress_var_apply_H_two_site, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cdouble, Cint, Ptr{Ptr{Cvoid}}),
                ctx.h, Ain.h, A.h, H.h, maxsweeps, svd_tol, dlim, out), :mpsb_compress_var_apply_H_two_site)
    return wrap_new_mps(out[])
end

# compress_sum_var_apply_H_two_site(Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim)   src/compression.jl:1072-1157
# half = 1: the _left form (:1159-1215), half = 2: the _right form (:1218-1276); H = nothing:
# compress_sum_var_two_site (:574-648).  Returns the compressed MPS (new handle, updated dims).
function compress_sum_var_apply_H_two_site(ctx::Ctx, Ain::DMPS, coef::Vector{<:Number}, A::Vector{DMPS},
                                           H::Union{DMPO,Nothing}, maxsweeps::Integer, svd_tol::Real,
                                           dlim::Integer; half::Integer = 0)
    c = ComplexF64.(coef)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mpsb_compress_sum_var_apply_H_two_site, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{ComplexF64}, Cint, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}, Cint, Cdouble, Cint, Cint,
                 Ptr{Ptr{Cvoid}}),
                ctx.h, Ain.h, c, length(c), [a.h for a in A], H === nothing ? C_NULL : H.h, maxsweeps, svd_tol, dlim,
                half, out), :mpsb_compress_sum_var_apply_H_two_site)
    return wrap_new_mps(out[])
end
compress_sum_var_two_site(ctx::Ctx, Ain::DMPS, coef::Vector{<:Number}, A::Vector{DMPS}, maxsweeps::Integer,
                          svd_tol::Real, dlim::Integer) =
    compress_sum_var_apply_H_two_site(ctx, Ain, coef, A, nothing, maxsweeps, svd_tol, dlim)

# RK4stp_apply_H_half_full_two_site(dt, H, psi, svd_tol, dims, dlim)   src/timeevolution.jl:208-215
# Four two-site half sweeps with adapting bonds; returns the new psi (its `dims` field holds
# the reference's updated dims).
function RK4stp_apply_H_half_full_two_site(ctx::Ctx, dt::Real, H::Vector{DMPO}, psi::DMPS, svd_tol::Real,
                                           dlim::Integer)
    s(Ain, c, A, O, half) = compress_sum_var_apply_H_two_site(ctx, Ain, c, A, O, 1, svd_tol, dlim; half = half)
    psi1 = s(psi, [1.0], [psi], H[1], 1)
    psi2 = s(psi1, [1.0, dt / 2], [psi, psi1], H[2], 2)
    psi3 = s(psi2, [1.0, dt], [psi, psi2], H[2], 1)
    return s(psi3, [-1 / 3, 1 / 3, 2 / 3, 1 / 3], [psi, psi1, psi2, psi3], H[3], 2)
end

# Two-lane RK4 step on (1, default) or off (0); no reference counterpart (results are identical)
set_pipeline!(ctx::Ctx, enable::Bool) =
    check(ccall((:mpsb_ctx_set_pipeline, LIB), Cint, (Ptr{Cvoid}, Cint), ctx.h, enable ? 1 : 0),
          :mpsb_ctx_set_pipeline)

end # module
