"""The tcgen05 3xTF32 trailing update of the mixed-precision LU, on the GPU.

C0 - A B for seeded random FP32 operands in [-1, 1], against an FP64
evaluation. Tolerance: error / k <= 1e-6 (FP32-level; a single TF32 product
would sit near 1e-4), and no worse than 4x the SIMT FP32 kernel's error.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (300, 200, 64), (257, 130, 40), (1000, 777, 256),
                                   (129, 1500, 224)])
def test_tc_update_matches_fp64(fp, m, n, k):
    err_tc, err_simt, ms = fp._capi.tc_selftest(m, n, k)
    assert err_tc < 1e-6, (err_tc, err_simt)
    assert err_tc <= 4 * err_simt + 1e-7, (err_tc, err_simt)


@pytest.mark.parametrize("nc,ns", [(8, 4), (12, 8), (20, 24), (40, 48), (60, 80)])
@pytest.mark.parametrize("precision", ["mixed", "mixed_gepp"])
def test_mixed_lu_refines_in_few_steps(fp, O, ctx, nc, ns, precision):
    """With the tensor-core update the FP32 factors stay FP32-accurate: the
    FP64 refinement converges to 1e-12 in a handful of steps, without GMRES,
    for the static row order (mixed) and the pivoted factors (mixed_gepp);
    sizes from one partial panel (32, 96 panels) to many panels with a partial
    last one (480, 1920, 4800)."""
    w = fp.meshes.swept_wing("0012", nc, ns)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(4.2)
    V = np.array([np.cos(a), 0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", precision))
    assert st.used_gmres == 0 and st.ir_iters <= 5, st.asdict()
    assert st.max_abs_L < 10.0   # multipliers of order one (0 when there are no rows below a diagonal block)
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10


@pytest.mark.parametrize("nc,ns", [(8, 4), (12, 8), (20, 24), (40, 48), (60, 80), (50, 30)])
@pytest.mark.parametrize("knob,value", [("FP_TUNE_TC_SPLIT", 1), ("FP_TUNE_TC_SPLIT", 2), ("FP_TUNE_TC_SPLIT", 3),
                                        ("FP_TUNE_TC_RED", 0), ("FP_TUNE_TC_TILES", 2), ("FP_TUNE_TC_TILES", 4),
                                        ("FP_TUNE_ASM32", 1), ("FP_TUNE_TC_NARROW", 0), ("FP_TUNE_TRS2", 1),
                                        ("FP_TUNE_PANEL_GEMM", 0), ("FP_TUNE_PANEL_GEMM", 1), ("FP_TUNE_PANEL_GEMM", 2),
                                        ("FP_TUNE_TC_PREFETCH", 1), ("FP_TUNE_PDL", 1), ("FP_TUNE_LU_SPLIT", 0),
                                        ("FP_TUNE_LU_FUSE", 1), ("FP_TUNE_REST_SPLIT", 1),
                                        ("FP_TUNE_REST_SPLIT", 2)])
def test_static_lu_update_variants(fp, O, nc, ns, knob, value):
    """The static-order LU's tensor-core update variants: FP_TUNE_TC_SPLIT
    1..3 reads unsplit FP32 operands and splits them into TF32 hi / lo in
    shared memory; FP_TUNE_TC_RED 0 adds the product to C by a TMA
    reduce-add instead of red.global; FP_TUNE_TC_TILES runs the multi-tile
    kernel (double-buffered accumulator, red.global epilogue); FP_TUNE_ASM32
    assembles the FP32 AIC in panel-local FP32 coordinates and the FP64 AIC
    on a background stream; FP_TUNE_TRS2 1 runs the FP32 sweeps' chain two
    blocks a step; FP_TUNE_PANEL_GEMM 0 forms L21 and U12 by block
    substitution, 1 as products with the full panel inverses, 2 forms L21 by
    substitution and inv(L) on a third stream, U12 as a product;
    FP_TUNE_TC_PREFETCH 1 prefetches each CTA's C tile into L2; FP_TUNE_PDL 1
    launches the kernels with programmatic dependent launch; FP_TUNE_LU_SPLIT 0
    keeps the rows below the next panel on the panel stream; FP_TUNE_LU_FUSE 1
    updates the next diagonal tile inside the U12 kernel; FP_TUNE_REST_SPLIT 1
    runs the trailing update as the next panel's rows, then the rows below
    (2: the first range on the fourth stream). The factors are as accurate as the default's (refinement
    in a handful of steps, the oracle's solution to 1e-10), for one partial
    panel up to many panels with a partial last one (1,500 panels: a last K
    block of 92)."""
    w = fp.meshes.swept_wing("0012", nc, ns)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(4.2)
    V = np.array([np.cos(a), 0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    c = fp._capi.Context(0)
    try:
        # the TF32-pair update, whose variants these are (the BF16-pair default
        # has its own test below)
        c.set_tuning(fp._capi.FP_TUNE_TC_BF16X3, 0)
        c.set_tuning(getattr(fp._capi, knob), value)
        c.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
        c.set_wake(w.shedding, D, D)
        x, st = c.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "mixed"))
    finally:
        c.close()
    assert st.used_gmres == 0 and st.ir_iters <= 5, st.asdict()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10


@pytest.mark.parametrize("nc,ns", [(12, 8), (20, 24), (60, 80), (50, 30)])
@pytest.mark.parametrize("panel,prefetch,pdl,split,fuse,wide,l21a,u12a,rsplit",
                         [(1, 0, 0, 0, 0, 0, 0, 0, 0), (2, 0, 0, 0, 0, 0, 0, 0, 0), (2, 1, 0, 0, 0, 0, 0, 0, 0),
                          (2, 1, 1, 0, 0, 0, 0, 0, 0), (2, 1, 1, 1, 0, 0, 0, 0, 0), (2, 1, 1, 1, 1, 0, 0, 0, 0),
                          (2, 1, 1, 1, 0, 1, 0, 0, 0), (2, 1, 1, 1, 0, 0, 1, 0, 0), (2, 1, 1, 1, 0, 0, 1, 1, 0),
                          (2, 1, 1, 1, 1, 1, 1, 1, 0), (2, 1, 1, 1, 0, 0, 1, 0, 1), (2, 1, 1, 1, 1, 0, 1, 0, 1),
                          (2, 1, 1, 0, 0, 0, 1, 0, 1), (1, 1, 1, 1, 0, 0, 1, 0, 1), (2, 1, 1, 1, 0, 0, 1, 0, 2),
                          (2, 1, 1, 1, 1, 0, 1, 0, 2)])
def test_bf16_pair_update_reaches_fp64_solution(fp, O, nc, ns, panel, prefetch, pdl, split, fuse, wide, l21a, u12a,
                                                rsplit):
    """FP_TUNE_TC_BF16X3 1: the mixed form's trailing update multiplies BF16
    pairs (hi + lo, three MMAs) instead of TF32 pairs; the factors carry 16-bit
    operand splits, and the FP64 refinement (GMRES-IR behind it) still reaches
    the oracle's solution to 1e-10, from one partial panel to many panels with
    a partial last one."""
    w = fp.meshes.swept_wing("0012", nc, ns)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(4.2)
    V = np.array([np.cos(a), 0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    c = fp._capi.Context(0)
    try:
        c.set_tuning(fp._capi.FP_TUNE_PANEL_GEMM, panel)
        c.set_tuning(fp._capi.FP_TUNE_TC_BF16X3, 1)
        c.set_tuning(fp._capi.FP_TUNE_TC_PREFETCH, prefetch)
        c.set_tuning(fp._capi.FP_TUNE_PDL, pdl)
        c.set_tuning(fp._capi.FP_TUNE_LU_SPLIT, split)
        c.set_tuning(fp._capi.FP_TUNE_LU_FUSE, fuse)
        c.set_tuning(fp._capi.FP_TUNE_U12_WIDE, wide)
        c.set_tuning(fp._capi.FP_TUNE_L21_ASYNC, l21a)
        c.set_tuning(fp._capi.FP_TUNE_U12_ASYNC, u12a)
        c.set_tuning(fp._capi.FP_TUNE_REST_SPLIT, rsplit)
        c.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
        c.set_wake(w.shedding, D, D)
        x, st = c.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "mixed"))
    finally:
        c.close()
    assert st.rel_residual < 1e-11, st.asdict()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10


@pytest.mark.parametrize("nc,ns", [(12, 8), (20, 24), (60, 80), (50, 30)])
@pytest.mark.parametrize("split,fuse,rsplit,x3", [(1, 0, 0, 1), (1, 1, 0, 1), (1, 0, 2, 1), (0, 0, 0, 1), (1, 0, 0, 0)])
def test_pdiag_full_inverse(fp, O, nc, ns, split, fuse, rsplit, x3):
    """FP_TUNE_PDIAG_LINV 1: the diagonal-block kernel forms the full inv(L)
    (no separate inverse launch) and L21 of the next panel's rows runs on the
    third stream; the mixed solve still reaches the oracle's solution to
    1e-10 with the split chain on or off, the fused U12 kernel, the trailing
    update in two row ranges, and either operand form."""
    w = fp.meshes.swept_wing("0012", nc, ns)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(4.2)
    V = np.array([np.cos(a), 0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    c = fp._capi.Context(0)
    try:
        c.set_tuning(fp._capi.FP_TUNE_PDIAG_LINV, 1)
        c.set_tuning(fp._capi.FP_TUNE_TC_BF16X3, x3)
        c.set_tuning(fp._capi.FP_TUNE_LU_SPLIT, split)
        c.set_tuning(fp._capi.FP_TUNE_LU_FUSE, fuse)
        c.set_tuning(fp._capi.FP_TUNE_REST_SPLIT, rsplit)
        c.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
        c.set_wake(w.shedding, D, D)
        x, st = c.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "mixed"))
    finally:
        c.close()
    assert st.used_gmres == 0 and st.ir_iters <= 5 and st.rel_residual < 1e-11, st.asdict()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10


@pytest.mark.parametrize("nc,ns", [(20, 24), (60, 80)])
def test_bf16_form_reaches_fp64_solution(fp, O, ctx, nc, ns):
    """FP_PREC_BF16: the factorisation starts from the BF16-rounded AIC and its
    trailing update multiplies BF16 operands with FP32 accumulation; plain
    refinement stalls on such factors and GMRES-IR with FP64 residuals takes
    over, reaching the FP64 solution to 1e-10 (ir_tol 1e-12)."""
    w = fp.meshes.swept_wing("0012", nc, ns)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(4.2)
    V = np.array([np.cos(a), 0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "bf16"))
    assert st.rel_residual < 1e-11, st.asdict()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_autotune_keeps_results(fp, O, precision):
    """fp_autotune through B200Solver(autotune=True): the knobs chosen for the
    size are cached (a second solve does not tune again) and the solution is
    the oracle's to 1e-10."""
    w = fp.meshes.swept_wing("0012", 40, 48)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(4.2)
    V = np.array([np.cos(a), 0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    solver = fp.B200Solver(method="ludiv", precision=precision, autotune=True)
    try:
        fp.solve(body, U, D, D, solver=solver)
        key = (w.npanels, precision)
        assert key in solver.tuned and len(solver.tuned[key]) == 10
        knobs = list(solver.tuned[key])
        fp.solve(body, U, D, D, solver=solver)
        assert solver.tuned[key] == knobs
        again = solver.ctx.autotune(fp._capi.FP_PREC_MIXED if precision == "mixed" else fp._capi.FP_PREC_FP64)
        assert again == knobs   # cached per size: applied, not re-timed
    finally:
        solver.close()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(body.strength - xr) / np.linalg.norm(xr) < 1e-10
