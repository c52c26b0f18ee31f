# FrequencyMaxwellCUDA.jl -- Julia binding of libfmcuda (C ABI in include/fmcuda.h).
#
# Source only: Julia is not available where this repository is built and tested, so this file is
# not executed here.  It shows the ccall layer a FrequencyMaxwell.jl maintainer adds so that
# `ConvergentBornSolver(...; device = :fmcuda)` routes `solve(solver, sources, medium)` to the GPU.
module FrequencyMaxwellCUDA

using FrequencyMaxwell
using KernelAbstractions
using LinearAlgebra
using LinearSolve

const libfmcuda = get(ENV, "FMCUDA_LIB", joinpath(@__DIR__, "..", "fmcuda", "libfmcuda.so"))

# Marker backend stored in solver.backend (convergent_born.jl:99); the device plugin point is
# GPU_BACKENDS / register_gpu_backend! (FrequencyMaxwell.jl:127-140).
struct FMCUDABackend <: KernelAbstractions.Backend end

const FM_OK = Cint(0)
const FM_NOT_CONVERGED = Cint(3)
const FM_PREC_F64 = Cint(0)
const FM_PREC_F32 = Cint(1)
const FM_PREC_F32_MATH64 = Cint(2)
const FM_METHOD_GMRES = Cint(0)
const FM_METHOD_BICGSTAB = Cint(1)
const FM_ORTHO_MGS = Cint(0)
const FM_ORTHO_CGS = Cint(1)
const FM_ORTHO_CGS2 = Cint(2)
const FM_ORTHO_BLOCK = Cint(3)
const FM_BLOCK_FP64 = Cint(0)
const FM_BLOCK_STORAGE = Cint(1)
const FM_BLOCK_FP64_ORTHO = Cint(2)
const FM_TUNE_Y_TMA = Cint(0)
const FM_TUNE_Z_TMA = Cint(1)
const FM_TUNE_TMA_CTAS_PER_SM = Cint(2)
const FM_TUNE_ROW_THREADS = Cint(3)
const FM_TUNE_WAVE_RHS = Cint(4)
const FM_TUNE_BLOCK_DOT = Cint(5)

struct FMPlanDesc
    grid::NTuple{3,Cint}
    pad::NTuple{3,Cint}
    resolution::NTuple{3,Cdouble}
    absorbing::NTuple{3,Cint}
    precision::Cint
    max_rhs::Cint
    device::Cint
end

struct FMSolveOpts
    method::Cint
    ortho::Cint
    restart::Cint
    maxiters::Cint
    reltol::Cdouble
    abstol::Cdouble
    timeout_s::Cdouble
    block::Cint
    block_store::Cint
end

struct FMSolveInfo
    iterations::Cint
    solved::Cint
    residual::Cdouble
    residual0::Cdouble
end

struct FMPotentialInfo
    eps_imag::Cdouble
    k_bg::Cdouble
    bornmax::Cint
end

struct FMPlaneWave
    wavelength::Cdouble
    polarization::NTuple{6,Cdouble}
    k_vector::NTuple{3,Cdouble}
    amplitude::Cdouble
    phase::Cdouble
end

# fm_shape: one region of a phantom painted on the device (fm_phantom_fill)
const FM_SHAPE_SPHERE, FM_SHAPE_PLATE, FM_SHAPE_CYLINDER = Cint(0), Cint(1), Cint(2)
struct FMShape
    kind::Cint
    axis::Cint
    center::NTuple{3,Cdouble}
    radius::Cdouble
    extent::Cdouble
    value::NTuple{2,Cdouble}
end

# phantom_bead's spheres (phantoms.jl:84-100): beads stacked along z about the grid centre (N+1)/2
function bead_shapes(grid_size::NTuple{3,Int}, permittivity_profile, pixel_radius::Real;
                     bead_distance::Real = 2 * pixel_radius)
    n = length(permittivity_profile)
    c = ntuple(i -> (grid_size[i] + 1) / 2, 3)
    shapes = FMShape[]
    for b in 1:n
        zc = c[3] + (b - (n + 1) / 2) * bead_distance
        (zc < 1 || zc > grid_size[3]) && continue
        v = ComplexF64(permittivity_profile[(b - 1) % n + 1])
        push!(shapes, FMShape(FM_SHAPE_SPHERE, Cint(3), (c[1], c[2], zc), pixel_radius, 0.0, (real(v), imag(v))))
    end
    return shapes
end

# paint `shapes` (in order) over permittivity_bg into the plan's device permittivity; the next
# build_potential_device! builds the potential from it without a host array
function phantom_fill!(plan, permittivity_bg::Real, shapes::Vector{FMShape})
    check(ccall((:fm_phantom_fill, libfmcuda), Cint, (Ptr{Cvoid}, Cdouble, Cint, Ptr{FMShape}, Ptr{ComplexF64}),
                plan, permittivity_bg, length(shapes), shapes, C_NULL))
end

function build_potential_device!(plan, solver, permittivity_bg::Real, wavelength)
    fx, fy, fz = (attenuation_filter(solver, d) for d in 1:3)
    pinfo = Ref{FMPotentialInfo}()
    check(ccall((:fm_build_potential, libfmcuda), Cint,
                (Ptr{Cvoid}, Ptr{ComplexF64}, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Cint,
                 Ref{FMPotentialInfo}),
                plan, C_NULL, permittivity_bg, wavelength, fx, fy, fz, solver.iterations_max, pinfo))
    return Int(pinfo[].bornmax)
end

function check(status)
    status == FM_OK && return status
    msg = unsafe_string(ccall((:fm_last_error, libfmcuda), Cstring, ()))
    status == Cint(1) && throw(ArgumentError(msg))
    status == FM_NOT_CONVERGED && return status
    error("libfmcuda: " * msg)
end

function plan_desc(solver::ConvergentBornSolver{T}; max_rhs::Integer = 1) where {T}
    bcs = solver.boundary_conditions
    pad = ntuple(i -> FrequencyMaxwell.padding_pixels(bcs[i], solver.resolution[i]), 3)
    prec = T === Float64 ? FM_PREC_F64 : FM_PREC_F32_MATH64
    FMPlanDesc(Cint.(solver.grid_size), Cint.(pad), Cdouble.(solver.resolution),
               ntuple(i -> Cint(FrequencyMaxwell.requires_averaging(bcs[i])), 3), prec, Cint(max_rhs), Cint(0))
end

plane_wave(s) = FMPlaneWave(s.wavelength,
                            (real(s.polarization[1]), imag(s.polarization[1]), real(s.polarization[2]),
                             imag(s.polarization[2]), real(s.polarization[3]), imag(s.polarization[3])),
                            Tuple(Float64.(s.k_vector)), s.amplitude, s.phase)

# device potential of `medium` on `plan`; returns Bornmax
function build_potential!(plan, solver, medium, wavelength)
    eps = ComplexF64.(FrequencyMaxwell.permittivity(medium))
    fx, fy, fz = (attenuation_filter(solver, d) for d in 1:3)
    pinfo = Ref{FMPotentialInfo}()
    check(ccall((:fm_build_potential, libfmcuda), Cint,
                (Ptr{Cvoid}, Ptr{ComplexF64}, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Cint,
                 Ref{FMPotentialInfo}),
                plan, eps, FrequencyMaxwell.permittivity_bg(medium), wavelength, fx, fy, fz,
                solver.iterations_max, pinfo))
    bornmax = Int(pinfo[].bornmax)
    bornmax >= 1 || throw(ArgumentError("Bornmax < 1"))
    return bornmax
end

# the per-axis filters of _apply_attenuation_to_potential! (convergent_born.jl:893-944)
function attenuation_filter(solver, dim)
    bc = solver.boundary_conditions[dim]
    pad = FrequencyMaxwell.padding_pixels(bc, solver.resolution[dim])
    n = solver.grid_size[dim] + 2pad
    (FrequencyMaxwell.requires_padding(bc) && pad > 0) || return ones(Float64, n)
    L = min(pad, round(Int, bc.attenuation_thickness / (solver.resolution[dim] * 2)))
    w = FrequencyMaxwell._create_attenuation_window(bc.profile, L, Float64) .* bc.sharpness .+ (1 - bc.sharpness)
    return vcat(w, ones(Float64, solver.grid_size[dim] + 2 * (pad - L)), reverse(w))
end

"""
    solve_fmcuda(solver, sources, medium) -> ElectromagneticField

`solve(solver, sources, medium)` (convergent_born.jl:565-600) on libfmcuda.  A maintainer adds, as the
first line of that method,

    solver.backend isa FrequencyMaxwellCUDA.FMCUDABackend &&
        return FrequencyMaxwellCUDA.solve_fmcuda(solver, sources, medium)
"""
function solve_fmcuda(solver::ConvergentBornSolver{T}, sources, medium) where {T}
    FrequencyMaxwell.grid_size(medium) == solver.grid_size ||
        throw(ArgumentError("medium grid_size must match solver grid_size"))
    srcs = sources isa AbstractVector ? sources : [sources]
    wavelength = FrequencyMaxwell.source_wavelength(sources)
    desc = Ref(plan_desc(solver))
    plan = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fm_plan_create, libfmcuda), Cint, (Ref{FMPlanDesc}, Ref{Ptr{Cvoid}}), desc, plan))
    try
        eps = ComplexF64.(FrequencyMaxwell.permittivity(medium))
        fx, fy, fz = (attenuation_filter(solver, d) for d in 1:3)
        pinfo = Ref{FMPotentialInfo}()
        check(ccall((:fm_build_potential, libfmcuda), Cint,
                    (Ptr{Cvoid}, Ptr{ComplexF64}, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Cint,
                     Ref{FMPotentialInfo}),
                    plan[], eps, FrequencyMaxwell.permittivity_bg(medium), wavelength, fx, fy, fz,
                    solver.iterations_max, pinfo))
        bornmax = Int(pinfo[].bornmax)
        bornmax >= 1 || throw(ArgumentError("Bornmax < 1"))
        waves = [FMPlaneWave(s.wavelength,
                             (real(s.polarization[1]), imag(s.polarization[1]), real(s.polarization[2]),
                              imag(s.polarization[2]), real(s.polarization[3]), imag(s.polarization[3])),
                             Tuple(Float64.(s.k_vector)), s.amplitude, s.phase) for s in srcs]
        first = Cint[0, length(waves)]
        method = solver.linear_solver isa LinearSolve.KrylovJL && occursin("bicgstab", lowercase(string(solver.linear_solver.KrylovAlg))) ? Cint(1) : Cint(0)
        opts = Ref(FMSolveOpts(method, T === Float64 ? Cint(0) : Cint(1), Cint(0), Cint(max(2bornmax, 100)),
                               solver.tolerance, solver.tolerance * 1e-2, 0.0, Cint(0), Cint(0)))
        E = Array{ComplexF64}(undef, solver.grid_size..., 3)
        H = similar(E)
        info = Ref{FMSolveInfo}()
        st = check(ccall((:fm_solve_plane_waves, libfmcuda), Cint,
                         (Ptr{Cvoid}, Cint, Ptr{Cint}, Ptr{FMPlaneWave}, Cdouble, Ref{FMSolveOpts}, Ptr{ComplexF64},
                          Ptr{ComplexF64}, Ref{FMSolveInfo}),
                         plan[], Cint(1), first, waves, FrequencyMaxwell.permittivity_bg(medium), opts, E, H, info))
        st == FM_NOT_CONVERGED && @warn "LinearSolve.jl did not converge."
        solver.Bornmax = bornmax
        solver.iteration_count = info[].iterations
        push!(solver.residual_history, T(info[].residual))
        return ElectromagneticField(Complex{T}.(E), Complex{T}.(H), solver.resolution, wavelength)
    finally
        ccall((:fm_plan_destroy, libfmcuda), Cvoid, (Ptr{Cvoid},), plan[])
    end
end

"""
    solve_fmcuda_batch(solver, sources_list, medium; block = 8) -> Vector{ElectromagneticField}

Many illuminations of one medium (each element of `sources_list` a source or a vector of sources, coherently
superposed) as the right-hand sides of one batched solve.  The batch uses s-step block GMRES with FP64 block
vectors stored orthonormalised (`block` vectors per block), which takes the iterates of full GMRES.  It needs
restart = 0 and at most 128 basis vectors: max(2 Bornmax, 100) + block + 1.
"""
function solve_fmcuda_batch(solver::ConvergentBornSolver{T}, sources_list, medium; block::Integer = 8) where {T}
    FrequencyMaxwell.grid_size(medium) == solver.grid_size ||
        throw(ArgumentError("medium grid_size must match solver grid_size"))
    lists = [s isa AbstractVector ? s : [s] for s in sources_list]
    isempty(lists) && throw(ArgumentError("sources_list cannot be empty"))
    wavelength = FrequencyMaxwell.source_wavelength(lists[1])
    n = length(lists)
    desc = Ref(plan_desc(solver; max_rhs = n))
    plan = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fm_plan_create, libfmcuda), Cint, (Ref{FMPlanDesc}, Ref{Ptr{Cvoid}}), desc, plan))
    try
        bornmax = build_potential!(plan[], solver, medium, wavelength)
        waves = [plane_wave(s) for l in lists for s in l]
        first = Cint.(cumsum([0; length.(lists)]))
        opts = Ref(FMSolveOpts(FM_METHOD_GMRES, FM_ORTHO_BLOCK, Cint(0), Cint(max(2bornmax, 100)),
                               solver.tolerance, solver.tolerance * 1e-2, 0.0, Cint(block), FM_BLOCK_FP64_ORTHO))
        E = Array{ComplexF64}(undef, solver.grid_size..., 3, n)
        H = similar(E)
        info = Vector{FMSolveInfo}(undef, n)
        st = check(ccall((:fm_solve_plane_waves, libfmcuda), Cint,
                         (Ptr{Cvoid}, Cint, Ptr{Cint}, Ptr{FMPlaneWave}, Cdouble, Ref{FMSolveOpts}, Ptr{ComplexF64},
                          Ptr{ComplexF64}, Ptr{FMSolveInfo}),
                         plan[], Cint(n), first, waves, FrequencyMaxwell.permittivity_bg(medium), opts, E, H, info))
        st == FM_NOT_CONVERGED && @warn "LinearSolve.jl did not converge."
        solver.Bornmax = bornmax
        solver.iteration_count = info[end].iterations
        push!(solver.residual_history, T(info[end].residual))
        return [ElectromagneticField(Complex{T}.(E[:, :, :, :, b]), Complex{T}.(H[:, :, :, :, b]), solver.resolution,
                                     wavelength) for b in 1:n]
    finally
        ccall((:fm_plan_destroy, libfmcuda), Cvoid, (Ptr{Cvoid},), plan[])
    end
end

# ---- the operator and preconditioner for any LinearSolve.jl algorithm ---------------------------------
# The device CBS operator (I - G_avg V) and left preconditioner (i/eps) V behind the reference's own
# interfaces, so LinearSolve.jl algorithms other than the two that libfmcuda runs itself (e.g. IDRs,
# BiCGStabL; docs/src/api.md:129-136) iterate on the device matvec:
#
#     A, Pl = fmcuda_operators(solver, medium, wavelength)
#     sol = LinearSolve.solve(LinearProblem(A, b), IDRs(); Pl = Pl, reltol = 1e-6)
#
# Vectors are flattened (Nx', Ny', Nz', 3) fields on the padded grid, ComplexF64 on the host.

"""Device plan with its potential, shared by the operator and the preconditioner below."""
mutable struct FMCUDAPlan
    ptr::Ptr{Cvoid}
    n::Int               # 3 * padded voxels
    bornmax::Int
    function FMCUDAPlan(solver::ConvergentBornSolver, medium, wavelength)
        desc = Ref(plan_desc(solver))
        plan = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:fm_plan_create, libfmcuda), Cint, (Ref{FMPlanDesc}, Ref{Ptr{Cvoid}}), desc, plan))
        p = new(plan[], 0, 0)
        finalizer(q -> q.ptr == C_NULL || ccall((:fm_plan_destroy, libfmcuda), Cvoid, (Ptr{Cvoid},), q.ptr), p)
        p.bornmax = build_potential!(p.ptr, solver, medium, wavelength)
        d = desc[]
        p.n = 3 * prod(Int(d.grid[i]) + 2 * Int(d.pad[i]) for i in 1:3)
        return p
    end
end

"""`CBSLinearOperator` (convergent_born.jl:452-518) on libfmcuda: y = beta*y + alpha*(x - G_avg(V.*x))."""
struct FMCUDALinearOperator{T <: AbstractFloat}
    plan::FMCUDAPlan
end

"""`CBSPreconditioner` (convergent_born.jl:379-431) on libfmcuda: y = (i/eps_imag) V.*x."""
struct FMCUDAPreconditioner{T <: AbstractFloat}
    plan::FMCUDAPlan
end

function fmcuda_operators(solver::ConvergentBornSolver{T}, medium, wavelength) where {T}
    p = FMCUDAPlan(solver, medium, wavelength)
    return FMCUDALinearOperator{T}(p), FMCUDAPreconditioner{T}(p)
end

function LinearAlgebra.mul!(y::AbstractVector, A::FMCUDALinearOperator, x::AbstractVector, α, β)
    length(x) == A.plan.n == length(y) || throw(DimensionMismatch("operator is $(A.plan.n) x $(A.plan.n)"))
    xc = Vector{ComplexF64}(x)
    yc = Vector{ComplexF64}(y)
    a, b = ComplexF64(α), ComplexF64(β)
    check(ccall((:fm_apply_operator, libfmcuda), Cint,
                (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}, Cdouble, Cdouble, Cdouble, Cdouble),
                A.plan.ptr, Cint(1), xc, yc, real(a), imag(a), real(b), imag(b)))
    y .= yc
    return y
end
LinearAlgebra.mul!(y::AbstractVector, A::FMCUDALinearOperator, x::AbstractVector) = mul!(y, A, x, true, false)
Base.:*(A::FMCUDALinearOperator{T}, x::AbstractVector) where {T} = mul!(similar(x, Complex{T}), A, x)
Base.size(A::FMCUDALinearOperator) = (A.plan.n, A.plan.n)
Base.size(A::FMCUDALinearOperator, dim::Integer) = size(A)[dim]
Base.eltype(::FMCUDALinearOperator{T}) where {T} = Complex{T}
Base.ndims(::FMCUDALinearOperator) = 2

function LinearAlgebra.ldiv!(y::AbstractVector, P::FMCUDAPreconditioner, x::AbstractVector)
    length(x) == P.plan.n == length(y) || throw(DimensionMismatch("preconditioner is $(P.plan.n) x $(P.plan.n)"))
    xc = Vector{ComplexF64}(x)
    yc = similar(xc)
    check(ccall((:fm_apply_preconditioner, libfmcuda), Cint,
                (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}), P.plan.ptr, Cint(1), xc, yc))
    y .= yc
    return y
end
LinearAlgebra.ldiv!(P::FMCUDAPreconditioner, x::AbstractVector) = ldiv!(x, P, copy(x))

function __init__()
    FrequencyMaxwell.register_gpu_backend!(:fmcuda, () -> FMCUDABackend())
end

end # module
