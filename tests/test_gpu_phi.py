"""GPU parity of the potential field phi! and of the doublet and
source+doublet non-lifting bodies, through the C ABI, against the oracle
(src/FLOWPanel_abstractbody.jl:118-127, src/FLOWPanel_nonliftingbody.jl:221-815,
src/FLOWPanel_liftingbody.jl:664-742).

Tolerances: potentials 1e-12 of the largest |phi| (same formulas in FP64;
FMA and the order of the per-panel scaling move the last bits); solved doublet
strengths 1e-10 relative (the plain form's bar); grad(phi) = U by central
differences to 1e-6 relative (h = 1e-5)."""
import numpy as np
import pytest

from conftest import freestream

pytestmark = pytest.mark.gpu


def _targets(rng, m, lo, hi):
    return lo + (hi - lo) * rng.random((m, 3))


def _close(a, b, tol=1e-12):
    assert np.abs(a - b).max() <= tol * np.abs(b).max()


@pytest.fixture(scope="module")
def sphere(fp):
    return fp.meshes.sphere(1.0, 8, 12)


@pytest.fixture(scope="module")
def wing(fp):
    return fp.meshes.swept_wing("0012", 16, 20)


def _load(ctx, fp, mesh):
    body = fp.NonLiftingBody(mesh)
    normals = fp.calc_normals(body)
    ctx.set_geometry(mesh.nodes, mesh.panel_offsets, mesh.panel_nodes, fp.calc_controlpoints(body, normals),
                     normals)


@pytest.mark.parametrize("kind", ["source", "doublet", "source+doublet"])
def test_phi_nonlifting_matches_oracle(fp, O, ctx, sphere, kind):
    rng = np.random.default_rng(3)
    _load(ctx, fp, sphere)
    N = sphere.npanels
    s = rng.standard_normal((N, 2) if kind == "source+doublet" else N)
    X = np.vstack([_targets(rng, 150, -2.0, 2.0), 1.01 * sphere.nodes[rng.integers(0, sphere.nnodes, 50)]])
    el = {"source": fp._capi.FP_ELEMENT_SOURCE, "doublet": fp._capi.FP_ELEMENT_VORTEXRING,
          "source+doublet": fp._capi.FP_ELEMENT_SOURCE_DOUBLET}[kind]
    out0 = rng.standard_normal(len(X))
    got = ctx.phi(el, s, X, out0.copy())
    ref = out0 + O.phi_body(sphere, kind, s, X)
    _close(got, ref)


@pytest.mark.parametrize("split", [False, True])
def test_phi_lifting_body_with_wake(fp, O, ctx, wing, split):
    """Vortex rings + the wake's semi-infinite doublets; with split, db is
    tilted from da so that the (da, db) triangle term is exercised."""
    rng = np.random.default_rng(4)
    _load(ctx, fp, wing)
    V = freestream(4.2)
    Da = np.tile(V, (wing.nsheddings, 1))
    Db = Da.copy()
    if split:
        W = freestream(9.0)
        Db = np.tile(W, (wing.nsheddings, 1))
    ctx.set_wake(wing.shedding, Da, Db)
    s = rng.standard_normal(wing.npanels)
    X = _targets(rng, 200, np.array([-1.0, -3.0, -1.0]), np.array([4.0, 3.0, 1.0]))
    got = ctx.phi(fp._capi.FP_ELEMENT_VORTEXRING, s, X)
    ref = O.phi_body(wing, "vortexring", s, X, Da, Db)
    _close(got, ref)


def test_phi_gradient_is_velocity(fp, ctx, wing):
    """grad(phi) = Uind off the body (the reference's element tests check
    grad(phi) = u per element, test/runtests_elements.jl:37-315; here for a
    whole solved wing with its wake)."""
    body = fp.RigidWakeBody(wing)
    V = freestream(4.2)
    U = np.tile(V, (wing.npanels, 1))
    D = np.tile(V, (wing.nsheddings, 1))
    solver = fp.B200Solver()
    fp.solve(body, U, D, D, solver=solver)
    rng = np.random.default_rng(5)
    X = _targets(rng, 40, np.array([-1.0, -3.0, 0.3]), np.array([3.0, 3.0, 1.5]))
    h = 1e-5
    g = np.zeros_like(X)
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        g[:, d] = (fp.phi(body, X + e, np.zeros(len(X)), solver) - fp.phi(body, X - e, np.zeros(len(X)), solver)) / (2 * h)
    u = fp.Uind(body, X, np.zeros((len(X), 3)), solver)
    assert np.abs(g - u).max() <= 1e-6 * np.abs(u).max()
    solver.close()


def test_doublet_body_solve_matches_oracle(fp, O, wing):
    """NonLiftingBody{ConstantDoublet}: G of the doublet panels (vortex rings,
    no wake), mu = G \\ (-Uinf . n) (src/FLOWPanel_nonliftingbody.jl:258-352)."""
    body = fp.NonLiftingBody(wing, element="ConstantDoublet")
    V = freestream(2.0)
    U = np.tile(V, (wing.npanels, 1))
    solver = fp.B200Solver()
    fp.solve(body, U, solver=solver)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    G = O.assemble_vortexring(_nowake(wing), cps, normals, np.zeros((0, 3)), np.zeros((0, 3)))
    mu = O.solve_ludiv(G, -np.einsum("ij,ij->i", U, normals))
    assert np.abs(body.strength - mu).max() <= 1e-10 * np.abs(mu).max()
    assert body.check_field("mu") and body.solved
    X = np.array([[0.5, 0.3, 0.8], [2.0, -1.0, 0.4]])
    _close(fp.phi(body, X, np.zeros(2), solver), O.phi_body(wing, "doublet", body.strength, X))
    solver.close()


def test_source_doublet_body_solve_matches_oracle(fp, O, sphere):
    """NonLiftingBody{Union{ConstantSource, ConstantDoublet}}: sigma = -Uinf . n,
    mu = the potential of the sources -sigma at the control points; like the
    reference, solve returns mu (src/FLOWPanel_nonliftingbody.jl:425-600)."""
    body = fp.NonLiftingBody(sphere, element="ConstantSource+ConstantDoublet")
    V = freestream(0.0)
    U = np.tile(V, (sphere.npanels, 1))
    mu = fp.solve(body, U)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    sigma = -np.einsum("ij,ij->i", normals, U)
    ref = O.phi_body(sphere, "source", -sigma, cps)
    _close(mu, ref)
    assert not body.solved


def test_phi_rejects_opposite_wake(fp, ctx, wing):
    _load(ctx, fp, wing)
    V = freestream(4.2)
    Da = np.tile(V, (wing.nsheddings, 1))
    ctx.set_wake(wing.shedding, Da, -Da)
    with pytest.raises(fp._capi.FlowPanelError, match="opposite or orthogonal"):
        ctx.phi(fp._capi.FP_ELEMENT_VORTEXRING, np.ones(wing.npanels), np.zeros((1, 3)))


def _nowake(mesh):
    import copy
    m = copy.copy(mesh)
    m.shedding = np.zeros((0, 6), np.int64)
    return m
