"""GPU parity: the CUDA path through the C ABI against the oracle.

Tolerances: AIC entries 1e-12 of the largest entry (same formulas; FMA and
reciprocal rewrites move the last bits); FP64 strengths 1e-10 relative (the
bar of the plain form); mixed-precision strengths 1e-10 relative after FP64
refinement; FP32 off-body velocity 1e-4 relative.
"""
import numpy as np
import pytest

from conftest import freestream

pytestmark = pytest.mark.gpu


def _wing_setup(fp, nc=20, ns=24, tri=False, aoa=4.2):
    w = fp.meshes.swept_wing("0012", nc, ns)
    if tri:
        w = fp.meshes.triangulate(w)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    V = freestream(aoa)
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    return w, body, normals, cps, D, U


@pytest.mark.parametrize("tri", [False, True])
def test_ring_aic_matches_oracle(fp, O, ctx, tri):
    w, body, normals, cps, D, U = _wing_setup(fp, tri=tri)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    ctx.assemble(fp._capi.FP_ELEMENT_VORTEXRING)
    G = ctx.get_aic()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    assert np.abs(G - Gr).max() <= 1e-12 * np.abs(Gr).max()
    big = np.abs(Gr) > 1e-3 * np.abs(Gr).max()
    assert np.max(np.abs(G[big] - Gr[big]) / np.abs(Gr[big])) < 1e-11


def test_ring_aic_shared_wake_columns(fp, O, ctx):
    """Two shedding edges on one panel column take the serial wake path."""
    w, body, normals, cps, D, U = _wing_setup(fp, 12, 8)
    sh = np.concatenate([w.shedding, w.shedding[:1]])
    D2 = np.concatenate([D, D[:1]])
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(sh, D2, D2)
    ctx.assemble(fp._capi.FP_ELEMENT_VORTEXRING)
    G = ctx.get_aic()
    w2 = fp.meshes.Mesh(w.nodes, w.panel_offsets, w.panel_nodes, sh, w.bodies)
    Gr = O.assemble_vortexring(w2, cps, normals, D2, D2)
    assert np.abs(G - Gr).max() <= 1e-12 * np.abs(Gr).max()


def test_source_aic_matches_oracle(fp, O, ctx):
    s = fp.meshes.sphere(1.0, 10, 20)
    body = fp.NonLiftingBody(s)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    ctx.set_geometry(s.nodes, s.panel_offsets, s.panel_nodes, cps, normals)
    ctx.assemble(fp._capi.FP_ELEMENT_SOURCE)
    G = ctx.get_aic()
    Gr = O.assemble_source(s, cps, normals)
    assert np.abs(G - Gr).max() <= 1e-12 * np.abs(Gr).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_gepp"])
def test_wing_solve_matches_oracle(fp, O, ctx, precision):
    w, body, normals, cps, D, U = _wing_setup(fp, 40, 48)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", precision))
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10
    assert st.rel_residual < 1e-11
    if precision == "fp64":
        assert st.max_abs_L > 0


@pytest.mark.parametrize("nc,ns", [(40, 48), (60, 90)])
@pytest.mark.parametrize("mode", [1, 2, 3, 4, 5, 6])
def test_fp64_lu_dmma_update_matches_oracle(fp, O, nc, ns, mode):
    """FP_TUNE_FP64_DMMA = 1..6: the FP64 LU's trailing update on the FP64
    tensor path (mma.sync .f64; 128 x 128 tiles with 8, 16 or 32 warps a CTA,
    128 x 64 tiles two CTAs an SM; 16- or 32-deep K slices) gives the oracle's
    strengths to 1e-10, and the SIMT update's to 1e-12 (1,920 and 5,400
    panels: several 256-column panels with partial tiles at the edges)."""
    w, body, normals, cps, D, U = _wing_setup(fp, nc, ns)
    xs = []
    for dmma in (mode, 0):
        c = fp._capi.Context(0)
        try:
            c.set_tuning(fp._capi.FP_TUNE_FP64_DMMA, dmma)
            c.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
            c.set_wake(w.shedding, D, D)
            x, st = c.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "fp64"))
            xs.append(x)
        finally:
            c.close()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(xs[0] - xr) / np.linalg.norm(xr) < 1e-10
    assert np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(xs[1]) < 1e-12


def test_multi_rhs_sweep(fp, O, ctx):
    """Angle-of-attack sweep as many right-hand sides on one factorisation (fixed wake)."""
    w, body, normals, cps, D, U = _wing_setup(fp, 20, 24)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    aoas = np.arange(-10, 11, 4.0)
    Us = np.stack([np.tile(freestream(a), (w.npanels, 1)) for a in aoas])
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    lu = O.lu_factor(Gr)
    for prec in ("fp64", "mixed", "mixed_gepp"):
        X, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, Us, opts=fp._capi.make_opts("ludiv", prec))
        for q in range(len(aoas)):
            xr = O.lu_solve(lu, O.rhs_noflowthrough(Us[q], normals))
            assert np.linalg.norm(X[q] - xr) / np.linalg.norm(xr) < 1e-10


def test_gmres_matches_oracle(fp, O, ctx):
    w, body, normals, cps, D, U = _wing_setup(fp, 20, 24)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    opts = fp._capi.make_opts("gmres", "fp64", gmres_atol=1e-13, gmres_rtol=1e-13)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=opts)
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    b = O.rhs_noflowthrough(U, normals)
    xr = O.solve_ludiv(Gr, b)
    assert st.used_gmres == 1 and st.gmres_iters > 0
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-9
    # the oracle's GMRES (Krylov.jl's unrestarted process) takes the same steps
    xg, it, conv = O.gmres(Gr, b, atol=1e-13, rtol=1e-13)
    assert conv and abs(it - st.gmres_iters) <= 2
    # GMRES(50) through the restart option converges too
    opts = fp._capi.make_opts("gmres", "fp64", gmres_atol=1e-13, gmres_rtol=1e-13, gmres_restart=True)
    x2, st2 = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=opts)
    assert np.linalg.norm(x2 - xr) / np.linalg.norm(xr) < 1e-9
    xg2, it2, conv2 = O.gmres(Gr, b, atol=1e-13, rtol=1e-13, restart=True)
    assert conv2 and abs(it2 - st2.gmres_iters) <= max(5, 0.2 * it2)


def test_uind_matches_oracle(fp, O, ctx):
    w, body, normals, cps, D, U = _wing_setup(fp, 20, 24)
    rng = np.random.default_rng(3)
    gamma = rng.standard_normal(w.npanels)
    probes = np.concatenate([cps + 0.05 * normals, rng.uniform(-3, 3, (500, 3))])
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    ref = O.uind_vortexring(w, gamma, D, D, probes)
    base = rng.standard_normal(probes.shape)
    got = ctx.uind(fp._capi.FP_ELEMENT_VORTEXRING, gamma, probes, base.copy())
    scale = np.abs(ref).max()
    assert np.abs(got - base - ref).max() <= 1e-12 * scale
    got32 = ctx.uind(fp._capi.FP_ELEMENT_VORTEXRING, gamma, probes, None, fp._capi.FP_PREC_MIXED)
    assert np.abs(got32 - ref).max() <= 1e-4 * scale


def test_uind_source_matches_oracle(fp, O, ctx):
    s = fp.meshes.sphere(1.0, 10, 20)
    body = fp.NonLiftingBody(s)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    rng = np.random.default_rng(5)
    sig = rng.standard_normal(s.npanels)
    probes = np.concatenate([cps, rng.uniform(-2, 2, (300, 3))])
    ctx.set_geometry(s.nodes, s.panel_offsets, s.panel_nodes, cps, normals)
    got = ctx.uind(fp._capi.FP_ELEMENT_SOURCE, sig, probes)
    ref = O.uind_source(s, sig, probes)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_sphere_host_api_analytic_cp(fp):
    """solve + calcfield_U + calcfield_Cp through the host mirror; Cp against
    1 - 9/4 sin^2(theta) (examples/sphere.jl:86-87)."""
    s = fp.meshes.sphere(1.0, 30, 60)
    body = fp.NonLiftingBody(s)
    U = np.tile([1.0, 0, 0], (s.npanels, 1))
    solver = fp.B200Solver("backslash", "fp64")
    fp.solve(body, U, solver=solver)
    Us = fp.calcfield_U(body, body, solver=solver)
    Cp = fp.calcfield_Cp(body, 1.0)
    cps = fp.calc_controlpoints(body)
    th = np.arccos(np.clip(cps[:, 0] / np.linalg.norm(cps, axis=1), -1, 1))
    err = Cp - (1 - 9 / 4 * np.sin(th) ** 2)
    assert np.sqrt(np.mean(err ** 2)) < 0.02 and np.abs(err).max() < 0.05
    # the same loads in one device pass (source body: no grad(mu) term)
    Dhat = np.array([1.0, 0.0, 0.0])
    Lhat = np.array([0.0, 0.0, 1.0])
    LDS = fp.surface_loads(body, 1.0, 1.225, Lhat, Dhat, solver=solver)
    Cp1 = body.get_field("Cp")["field_data"]
    F1 = body.get_field("F")["field_data"]
    assert np.abs(Cp1 - Cp).max() < 1e-12
    F = fp.calcfield_F(body, 1.0, 1.225, solver=solver)
    assert np.abs(F1 - F).max() < 1e-12
    # a closed body in potential flow: no net force (d'Alembert), to the mesh's accuracy
    assert np.abs(LDS).max() < 0.05 * 0.5 * 1.225 * np.pi
    solver.close()


def test_errors_mirror_reference(fp, ctx):
    cap = fp._capi
    w = fp.meshes.swept_wing("0012", 8, 4)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes)
    bad = np.tile([1.0, 0.0, 0.1], (w.nsheddings, 1))
    with pytest.raises(cap.FlowPanelError) as e:
        ctx.set_wake(w.shedding, bad, bad)
    assert e.value.code == cap.FP_EINVAL and "non-unitary" in str(e.value)
    offs = np.array([0, 5], np.int32)
    with pytest.raises(cap.FlowPanelError) as e:
        ctx.set_geometry(w.nodes, offs, np.arange(5, dtype=np.int32))
    assert e.value.code == cap.FP_EINVAL
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes)
    with pytest.raises(cap.FlowPanelError) as e:
        ctx.factor()
    assert e.value.code == cap.FP_ESTATE


def test_factor_trace(fp, ctx):
    """fp_trace: every launch of a factorisation on both streams, in order
    on each stream, inside the factorisation's span; no trace when off."""
    w, body, normals, cps, D, U = _wing_setup(fp, nc=24, ns=30)   # 720 panels: three outer panels
    cap = fp._capi
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    ctx.assemble(cap.FP_ELEMENT_VORTEXRING, precision=cap.FP_PREC_MIXED)
    ctx.trace(True)
    ctx.factor(cap.FP_PREC_MIXED)
    ctx.trace(False)
    tags, streams, t0, t1 = ctx.trace_read()
    assert len(tags) > 10
    assert set(np.unique(tags)) <= set(range(9)) and {0, 1, 2, 3, 8} <= set(np.unique(tags))   # 8: the panel inverses
    assert {0, 1} <= set(np.unique(streams)) <= {0, 1, 2, 3}
    assert np.all(t1 >= t0) and np.all(t0 >= 0)
    for s in (0, 1):
        o = np.argsort(t0[streams == s])
        a, b = t0[streams == s][o], t1[streams == s][o]
        assert np.all(a[1:] >= b[:-1] - 1e-3)   # launches on one stream do not overlap
    ctx.factor(cap.FP_PREC_MIXED)
    assert len(ctx.trace_read()[0]) == 0


# ------------------------------------------------------------------ pinned to the reference's records
@pytest.fixture(scope="module")
def vtu_wing(fp, O):
    from test_oracle_ugradmu import vtu_wing_oracle
    w = vtu_wing_oracle(fp, O)
    w["G"] = O.assemble_vortexring(w["mesh"], w["cps"], w["normals"], w["D"], w["D"])
    w["b"] = O.rhs_noflowthrough(w["Uinfs"], w["normals"])
    return w


@pytest.mark.parametrize("tol,niter", [(1e-8, 286), (1e-2, 88), (1e-1, 25)])
def test_gmres_published_iterations_vtu_wing(fp, O, ctx, vtu_wing, tol, niter):
    """solve_gmres! on the reference's swept-wing mesh takes the iteration
    counts the reference records (docs/resources/data/sweptwing000-gmres{8,2,1}.md:
    286, 88, 25; examples/sweptwing_solverbenchmark.jl:100-155). The device
    orthogonalises by classical Gram-Schmidt twice instead of modified
    Gram-Schmidt, which can move the step where the estimate crosses the
    tolerance by one. Strengths: relative to the oracle's GMRES iterate,
    max(1e-6, 1e-2 tol): an iterate stopped at a loose tolerance carries more
    of the orthogonalisation's rounding than a converged one (3e-5 at 1e-2)."""
    w = vtu_wing
    m = w["mesh"]
    ctx.set_geometry(m.nodes, m.panel_offsets, m.panel_nodes, w["cps"], w["normals"])
    ctx.set_wake(m.shedding, w["D"], w["D"])
    opts = fp._capi.make_opts("gmres", "fp64", gmres_atol=tol, gmres_rtol=tol)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, w["Uinfs"], opts=opts)
    assert st.used_gmres == 1
    assert abs(st.gmres_iters - niter) <= 1, st.gmres_iters
    xo, ito, conv = O.gmres(w["G"], w["b"], atol=tol, rtol=tol)
    assert conv and ito == niter
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < max(1e-6, 1e-2 * tol)


def test_mixed_gmres_ir_fallback(fp, O, ctx):
    """With one refinement step allowed the mixed solve hands over to GMRES-IR
    (right-preconditioned by the FP32 factors) and still reaches the FP64
    solution to 1e-10."""
    w, body, normals, cps, D, U = _wing_setup(fp, 40, 48)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    opts = fp._capi.make_opts("ludiv", "mixed", ir_maxiter=1)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=opts)
    assert st.ir_iters == 1 and st.used_gmres == 1 and st.gmres_iters > 0, st.asdict()
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10
    assert st.rel_residual < 1e-11


@pytest.mark.parametrize("tri", [False, True])
def test_sphere_strengths_match_oracle(fp, O, ctx, tri):
    """Config-1 sphere (30 x 60 cells: 1,800 source panels with 3-node pole
    rows, or 3,600 triangles): sigma = G \\ lambda against the oracle's
    assembly and LAPACK solve (src/FLOWPanel_nonliftingbody.jl:93-130) to
    1e-10 relative."""
    s = fp.meshes.sphere(1.0, 30, 60)
    if tri:
        s = fp.meshes.triangulate(s)
    body = fp.NonLiftingBody(s)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    U = np.tile([1.0, 0.0, 0.0], (s.npanels, 1))
    ctx.set_geometry(s.nodes, s.panel_offsets, s.panel_nodes, cps, normals)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_SOURCE, U, opts=fp._capi.make_opts("ludiv", "fp64"))
    Gr = O.assemble_source(s, cps, normals)
    xr = O.solve_ludiv(Gr, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10
    assert st.gepp_certified == 1


def _shuffled_wing(fp, nc, ns, seed):
    """The wing with its panels listed in a seeded random order (as an
    unstructured mesher may list them); shedding rows follow their panels."""
    w = fp.meshes.swept_wing("0012", nc, ns)
    perm = np.random.default_rng(seed).permutation(w.npanels)   # new panel i = old panel perm[i]
    inv = np.empty_like(perm)
    inv[perm] = np.arange(w.npanels)
    counts = np.diff(w.panel_offsets)[perm]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    pn = np.concatenate([w.panel(p) for p in perm]).astype(np.int32)
    sh = w.shedding.copy()
    sh[:, 0] = inv[sh[:, 0]]
    sh[:, 3] = np.where(sh[:, 3] >= 0, inv[np.maximum(sh[:, 3], 0)], -1)
    return fp.meshes.Mesh(w.nodes, offs, pn, sh, w.bodies)


def test_uncertified_pivots_are_refined(fp, O, ctx):
    """Panels in a shuffled order put column maxima outside the 64-row
    diagonal blocks, so the block-local pivots are not LAPACK's (max|L| > 1).
    The FP64 solve then refines against the FP64 AIC and still matches
    LAPACK's solution to 1e-10, as does the adjoint (transposed) solve; the
    allocation-free solve refuses those factors."""
    import ctypes
    w = _shuffled_wing(fp, 20, 24, seed=0)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    V = freestream(4.2)
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "fp64"))
    assert st.gepp_certified == 0 and st.max_abs_L > 1.0, st.asdict()
    assert st.ir_iters >= 1
    Gr = O.assemble_vortexring(w, cps, normals, D, D)
    lu = O.lu_factor(Gr)
    xr = O.lu_solve(lu, O.rhs_noflowthrough(U, normals))
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10
    ybar = np.random.default_rng(1).standard_normal(w.npanels)
    lam = ctx.adjoint_solve(ybar)
    lr = np.linalg.solve(Gr.T, ybar)
    assert np.linalg.norm(lam.ravel() - lr) / np.linalg.norm(lr) < 1e-10
    fake = ctypes.c_void_p(1 << 40)   # never dereferenced: the call is refused first
    assert fp._capi.lib().fp_lu_solve_noalloc(ctx.h, fake, w.npanels, 1) == fp._capi.FP_ESTATE
    # the mixed form's static row order on the same shuffled panels still refines to the FP64 solution
    xm, stm = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=fp._capi.make_opts("ludiv", "mixed"))
    assert np.linalg.norm(xm - xr) / np.linalg.norm(xr) < 1e-10, stm.asdict()
