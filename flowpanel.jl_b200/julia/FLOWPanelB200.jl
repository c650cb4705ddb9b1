# Julia face of libflowpanel_b200.so: the GPU solver type for FLOWPanel.jl's
# `solve(body, Uinfs, Das, Dbs; solver=B200Solver(...))`, its `Uind!` and
# `phi!` device paths, the grad(mu) surface velocity and surface loads of
# `calcfield_Ugradmu` / `Cp` / `F` / `LDS`, and the ChainRulesCore pullback of
# the solve. Every function is one
# `ccall` into include/flowpanel_b200.h; array layouts are FLOWPanel's own
# (3 x N Float64 column-major, passed without copies).
#
# Include it from FLOWPanel.jl's module (next to src/FLOWPanel.jl:64-73) after
# setting `libfp` to the library path. Julia is not available where this file
# was written: it follows the header and mirrors the tested Python twin
# (flowpanel.jl_b200/_capi.py, bodies.py, adjoint.py) call for call.

const FP_OK = Cint(0)
const FP_ELEMENT_SOURCE = Cint(0)
const FP_ELEMENT_VORTEXRING = Cint(1)
const FP_ELEMENT_SOURCE_DOUBLET = Cint(2)
const FP_PREC_FP64 = Cint(0)
const FP_PREC_MIXED = Cint(1)
const FP_PREC_MIXED_GEPP = Cint(2)
const FP_SOLVER_LU = Cint(0)
const FP_SOLVER_GMRES = Cint(1)
const FP_UGRADMU_COMBINED = Cint(0)
const FP_UGRADMU_CELL = Cint(1)
const FP_UGRADMU_NODE = Cint(2)

struct FPSolveOpts
    solver::Cint
    precision::Cint
    ir_tol::Cdouble
    ir_maxiter::Cint
    gmres_memory::Cint
    gmres_atol::Cdouble
    gmres_rtol::Cdouble
    gmres_itmax::Cint
    gmres_restart::Cint   # 0: Krylov.jl's gmres without restart (the reference's call); 1: GMRES(memory)
end

struct FPStats
    ms_assemble::Cdouble
    ms_factor::Cdouble
    ms_solve::Cdouble
    ir_iters::Cint
    gmres_iters::Cint
    used_gmres::Cint
    gepp_certified::Cint
    max_abs_L::Cdouble
    rel_residual::Cdouble
end

"""
    B200Solver(; method=:ludiv, precision=:fp64, device=0, ir_tol=1e-12)

GPU drop-in for the `solver` keyword of `solve`: owns a device context that
assembles, factors and solves on a B200. `method` is `:ludiv`, `:backslash`
(both LU) or `:gmres`; `precision` is `:fp64` (plain), `:mixed` (FP32
tensor-core factors with a static row order and FP64 refinement) or
`:mixed_gepp` (the same factors pivoted as the FP64 form).
"""
mutable struct B200Solver
    ctx::Ptr{Cvoid}
    opts::FPSolveOpts
    stats::Union{Nothing, FPStats}
    offsets::Vector{Int32}            # CSR connectivity of the loaded body, 0-based
    pnodes::Vector{Int32}
    shedding::Matrix{Int32}           # 6 x nsh, 0-based, pj == -1 kept
    function B200Solver(; method=:ludiv, precision=:fp64, device=0, ir_tol=1e-12, ir_maxiter=10,
                        gmres_memory=50, atol=-1.0, rtol=-1.0, itmax=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:fp_ctx_create, libfp), Cint, (Cint, Ref{Ptr{Cvoid}}), device, r)
        rc == FP_OK || error("fp_ctx_create failed on device $device (status $rc)")
        opts = FPSolveOpts(method == :gmres ? FP_SOLVER_GMRES : FP_SOLVER_LU,
                           precision == :mixed ? FP_PREC_MIXED :
                           precision == :mixed_gepp ? FP_PREC_MIXED_GEPP : FP_PREC_FP64, ir_tol, ir_maxiter,
                           gmres_memory, atol, rtol, itmax, Cint(0))
        s = new(r[], opts, nothing, Int32[], Int32[], zeros(Int32, 6, 0))
        finalizer(x -> ccall((:fp_ctx_destroy, libfp), Cint, (Ptr{Cvoid},), x.ctx), s)
        return s
    end
end

fp_check(s::B200Solver, rc) =
    rc == FP_OK || error(unsafe_string(ccall((:fp_last_error, libfp), Cstring, (Ptr{Cvoid},), s.ctx)))

"""CSR connectivity (0-based Int32) of a body's grid, built once per mesh: the
node indices of each cell as the reference's assembly loops read them
(gt.get_cell_t! with the body's work arrays, src/FLOWPanel_liftingbody.jl:476-503)."""
function fp_connectivity(body)
    offsets = Int32[0]
    pnodes = Int32[]
    tri_out, tricoor, quadcoor, quad_out, lin, ndivscells, cin = gt.generate_getcellt_args!(body.grid)
    for i in 1:body.ncells
        panel = gt.get_cell_t!(tri_out, tricoor, quadcoor, quad_out, body.grid, i, lin, ndivscells, cin)
        append!(pnodes, Int32.(panel .- 1))
        push!(offsets, length(pnodes))
    end
    return offsets, pnodes
end

function fp_set_arrays!(s::B200Solver, nodes, CPs, normals, Das, Dbs)
    GC.@preserve nodes CPs normals begin
        fp_check(s, ccall((:fp_set_geometry, libfp), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Int32}, Ptr{Int32}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
            s.ctx, nodes, size(nodes, 2), s.offsets, s.pnodes, length(s.offsets) - 1, CPs, normals, C_NULL))
    end
    sh = s.shedding
    GC.@preserve sh Das Dbs fp_check(s, ccall((:fp_set_wake, libfp), Cint,
        (Ptr{Cvoid}, Ptr{Int32}, Int64, Ptr{Float64}, Ptr{Float64}), s.ctx, sh, size(sh, 2), Das, Dbs))
end

function fp_load!(s::B200Solver, body)
    s.offsets, s.pnodes = fp_connectivity(body)
    sh = Int32.(body.shedding)
    for e in 1:size(sh, 2)
        sh[1, e] -= 1                          # upper panel, 0-based
        sh[4, e] = sh[4, e] == -1 ? -1 : sh[4, e] - 1   # lower panel, -1 kept
        for r in (2, 3, 5, 6); sh[r, e] -= 1; end       # panel-local node indices
    end
    s.shedding = sh
end

"Gamma for the given geometry arrays (the differentiable core of solve_b200)."
function gamma_b200(s::B200Solver, nodes, CPs, normals, Uinfs, Das, Dbs; kerneloffset=1e-8, kernelcutoff=1e-14)
    fp_set_arrays!(s, Matrix{Float64}(nodes), Matrix{Float64}(CPs), Matrix{Float64}(normals),
                   Matrix{Float64}(Das), Matrix{Float64}(Dbs))
    Gamma = zeros(length(s.offsets) - 1)
    st = Ref{FPStats}()
    U = Matrix{Float64}(Uinfs)
    GC.@preserve U Gamma fp_check(s, ccall((:fp_solve_body, libfp), Cint,
        (Ptr{Cvoid}, Cint, Cdouble, Cdouble, Ptr{Float64}, Int64, Ref{FPSolveOpts}, Ptr{Float64}, Ref{FPStats}),
        s.ctx, FP_ELEMENT_VORTEXRING, kerneloffset, kernelcutoff, U, 1, s.opts, Gamma, st))
    s.stats = st[]
    return Gamma
end

"""
    solve(body, Uinfs, Das, Dbs, solver::B200Solver)

The GPU path of src/FLOWPanel_liftingbody.jl:172-216 / src/FLOWPanel_multibody.jl:312-364:
same argument checks, then assembly + RHS + factorisation + solve on the
device, then the strengths and fields stored as the reference stores them.
"""
function solve_b200(self, Uinfs::AbstractMatrix, Das, Dbs, solver::B200Solver)
    size(Uinfs) == (3, self.ncells) || error("Invalid Uinfs; expected size (3, $(self.ncells)), got $(size(Uinfs))")
    normals = _calc_normals(self)
    CPs = _calc_controlpoints(self, normals)
    fp_load!(solver, self)
    Gamma = gamma_b200(solver, self.grid._nodes, CPs, normals, Uinfs, Das, Dbs;
                       kerneloffset=self.kerneloffset, kernelcutoff=self.kernelcutoff)
    _set_strength(self, Gamma)
    add_field(self, "Uinf", "vector", collect(eachcol(Uinfs)), "cell")
    add_field(self, "Da", "vector", collect(eachcol(Das)), "system")
    add_field(self, "Db", "vector", collect(eachcol(Dbs)), "system")
    add_field(self, "Gamma", "scalar", view(self.strength, :, 1), "cell")
    return nothing
end

"Device path of Uind! (src/FLOWPanel_liftingbody.jl:576-661): adds into out (3 x M)."
function Uind_b200!(self, targets::Matrix{Float64}, out::Matrix{Float64}, solver::B200Solver)
    s = Vector{Float64}(self.strength[:, 1])
    GC.@preserve s targets out fp_check(solver, ccall((:fp_uind, libfp), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Cint, Cdouble, Cdouble),
        solver.ctx, FP_ELEMENT_VORTEXRING, s, targets, size(targets, 2), out, FP_PREC_FP64,
        self.kerneloffset, self.kernelcutoff))
    return out
end

"""Device path of phi! (src/FLOWPanel_abstractbody.jl:118-127): adds into out (M). `element`
is FP_ELEMENT_VORTEXRING for a RigidWakeBody{VortexRing} (wake doublets included, as
src/FLOWPanel_liftingbody.jl:664-742) or a NonLiftingBody{ConstantDoublet}, FP_ELEMENT_SOURCE
for NonLiftingBody{ConstantSource}, FP_ELEMENT_SOURCE_DOUBLET for the source+doublet body
(self.strength N x 2, column-major as Julia holds it)."""
function phi_b200!(self, targets::Matrix{Float64}, out::Vector{Float64}, solver::B200Solver, element::Cint)
    s = element == FP_ELEMENT_SOURCE_DOUBLET ? Matrix{Float64}(self.strength[:, 1:2]) :
                                               Vector{Float64}(self.strength[:, 1])
    GC.@preserve s targets out fp_check(solver, ccall((:fp_phi, libfp), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Cdouble),
        solver.ctx, element, s, targets, size(targets, 2), out, self.kerneloffset))
    return out
end

"""Device path of calcfield_Ugradmu! / _cell! / _node! (src/FLOWPanel_postprocess.jl:139-941) for a
solved body with triangular panels: `scheme` FP_UGRADMU_COMBINED (out_cell and out_node
receive the two schemes' fields), FP_UGRADMU_CELL (adds into out, maxgrad) or FP_UGRADMU_NODE
(overwrites out). `cpoffset` holds every panel's CPoffset (each member's own in a MultiBody).
`sharpTE` (node and combined schemes) and `smoothPass` / `smoothRows` (cell scheme, the rows
placed on the loft's cell grid `ndivscells` = (n1, n2), column-major) as in the reference."""
function Ugradmu_b200!(self, out::Matrix{Float64}, solver::B200Solver, cpoffset::Vector{Float64};
                       scheme=FP_UGRADMU_COMBINED, out_cell=nothing, out_node=nothing,
                       anglecrit=30.0, force_cellTE=true, maxgrad=Inf, Gammai=1, sharpTE=false,
                       smoothPass=0, smoothRows=(0,), ndivscells=(0, 0))
    s = Vector{Float64}(self.strength[:, Gammai])
    oc = out_cell === nothing ? C_NULL : out_cell
    on = out_node === nothing ? C_NULL : out_node
    cells = smoothPass == 0 || smoothRows[1] == 0 ? Int32[] :
            Int32[(i - 1) + ndivscells[1] * (j - 1) for i in smoothRows for j in 1:ndivscells[2]]
    GC.@preserve s cpoffset out out_cell out_node cells fp_check(solver, ccall((:fp_ugradmu_ex, libfp), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Cdouble, Cint, Cdouble, Cint, Ptr{Int32}, Int64, Cint,
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        solver.ctx, scheme, s, cpoffset, anglecrit, Cint(force_cellTE), maxgrad, Cint(sharpTE),
        isempty(cells) ? C_NULL : cells, length(cells), Cint(smoothPass), out, oc, on))
    return out
end

"""Device path of the examples' post-processing (calcfield_U + calcfield_Ugradmu + addfields +
calcfield_Cp + calcfield_F + calcfield_LDS, examples/sweptwing_solverbenchmark.jl:14-66):
returns (U 3 x N, Cp N, F 3 x N, LDS 3 x 3)."""
function surface_loads_b200(self, solver::B200Solver, cpoffset::Vector{Float64}, magVinf, rho,
                            Lhat, Dhat, Shat; element=FP_ELEMENT_VORTEXRING, ugradmu=true,
                            correct_kuttacondition=true)
    N = self.ncells
    s = Vector{Float64}(self.strength[:, 1])
    Uinfs = hcat(get_field(self, "Uinf")["field_data"]...)
    U, Cp, F, LDS = zeros(3, N), zeros(N), zeros(3, N), zeros(3, 3)
    L, D, S = Vector{Float64}(Lhat), Vector{Float64}(Dhat), Vector{Float64}(Shat)
    GC.@preserve s Uinfs cpoffset L D S U Cp F LDS fp_check(solver, ccall((:fp_surface_loads, libfp), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Cdouble, Cdouble, Cint, Cdouble, Cdouble,
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        solver.ctx, element, s, Uinfs, cpoffset, self.kerneloffset, self.kernelcutoff, Cint(ugradmu),
        magVinf, rho, L, D, S, Cint(correct_kuttacondition), U, Cp, F, LDS))
    return U, Cp, F, LDS
end

# ChainRulesCore pullback of Gamma = A(nodes, CPs, normals, Das, Dbs) \ b(Uinfs, normals):
# lambda = A^-T dGamma on the saved factors, then the reverse-mode assembly.
function ChainRulesCore.rrule(::typeof(gamma_b200), solver::B200Solver, nodes, CPs, normals, Uinfs, Das, Dbs)
    Gamma = gamma_b200(solver, nodes, CPs, normals, Uinfs, Das, Dbs)
    function pullback(dGamma)
        ybar = Vector{Float64}(ChainRulesCore.unthunk(dGamma))
        lam = similar(ybar)
        GC.@preserve ybar lam fp_check(solver, ccall((:fp_adjoint_solve, libfp), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}), solver.ctx, ybar, 1, lam))
        dn, dc, dnr, dU = zeros(size(nodes)), zeros(size(CPs)), zeros(size(normals)), zeros(size(Uinfs))
        dDa, dDb = zeros(size(Das)), zeros(size(Dbs))
        U = Matrix{Float64}(Uinfs)
        GC.@preserve U dn dc dnr dU dDa dDb fp_check(solver, ccall((:fp_assembly_vjp, libfp), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
             Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
            solver.ctx, C_NULL, C_NULL, U, dn, dc, dnr, dU, dDa, dDb))
        return (ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), dn, dc, dnr, dU, dDa, dDb)
    end
    return Gamma, pullback
end
