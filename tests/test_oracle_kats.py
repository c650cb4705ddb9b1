"""Pin the oracle against the reference's own known-answer tests (CPU).

test/runtests_elements.jl:37-315 and test/runtests_semiinfiniteelements.jl:28-241
check properties of the element kernels: grad(phi) == u (ForwardDiff vs the
analytic velocity, tolerance 1e-8 %), div(u) == 0 (1e-14), phi(inf) == 0 and
the jump conditions across the panel. The same checks run here on the
restatement, with a forward dual number in place of ForwardDiff and seeded
random points in place of the reference's unseeded rand(3).

The reference's GeometricTools.rotation_matrix is unvendored; a fixed rotation
(30, 10, 40 degrees about x, y, z) stands in for it: the properties checked are
invariant under any rotation.
"""
import numpy as np
import pytest


def _rot(a, b, c):
    a, b, c = np.deg2rad([a, b, c])
    Rx = np.array([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]])
    Ry = np.array([[np.cos(b), 0, np.sin(b)], [0, 1, 0], [-np.sin(b), 0, np.cos(b)]])
    Rz = np.array([[np.cos(c), -np.sin(c), 0], [np.sin(c), np.cos(c), 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


# planar pentagon of test/runtests_elements.jl:41-52, rotated and moved to O = (1,1,1)
PENTAGON = np.array([[0, 0, 0], [0, 1, 0], [0.4, 1.2, 0], [1, 0.8, 0], [0.8, 0, 0]], float)
R = _rot(30, 10, 40)
NODES = (R.T @ PENTAGON.T).T + 1.0
PANEL = np.arange(5)
# semi-infinite panel of test/runtests_semiinfiniteelements.jl:31-51
SI = np.array([[-2, -1, 0], [0, 1, 0], [9999, 1, 0], [9999, -1, 0]], float)
SI_NODES = (R.T @ SI.T).T + 1.0
SI_D = R.T @ np.array([1.0, 0, 0])


@pytest.mark.parametrize("seed", range(6))
def test_grad_phi_equals_u_source(O, seed):
    X = np.random.default_rng(seed).random(3)
    g = O.grad_phi("source", NODES, PANEL, 1.0, X, offset=0.0)
    U = O.U_constant_source(NODES, PANEL, 1.0, X[None], offset=0.0)[0]
    assert np.all(np.abs(g - U) / np.abs(U) * 100 <= 1e-8)


@pytest.mark.parametrize("seed", range(6))
def test_grad_phi_equals_u_doublet(O, seed):
    X = np.random.default_rng(100 + seed).random(3)
    g = O.grad_phi("doublet", NODES, PANEL, 1.0, X)
    U = O.U_vortexring(NODES, PANEL, 1.0, X[None], cutoff=0.0, offset=0.0)[0]
    assert np.all(np.abs(g - U) / np.abs(U) * 100 <= 1e-8)


@pytest.mark.parametrize("seed", range(6))
def test_grad_phi_equals_u_semiinfinite(O, seed):
    X = np.random.default_rng(200 + seed).random(3)
    g = O.grad_phi("semiinfinite", SI_NODES, np.array([0, 1]), 1.0, X, d=SI_D)
    U, _ = O.jac_U("horseshoe", SI_NODES, np.array([0, 1]), 1.0, X, d=SI_D, cutoff=0.0, offset=0.0)
    assert np.all(np.abs(g - U) / np.abs(U) * 100 <= 1e-8)


@pytest.mark.parametrize("kind", ["source", "ring"])
@pytest.mark.parametrize("seed", range(4))
def test_divergence_free(O, kind, seed):
    X = np.random.default_rng(300 + seed).random(3)
    _, J = O.jac_U(kind, NODES, PANEL, 1.0, X)
    assert abs(np.trace(J)) < 1e-14


@pytest.mark.parametrize("seed", range(4))
def test_divergence_free_semiinfinite(O, seed):
    X = np.random.default_rng(400 + seed).random(3)
    _, J = O.jac_U("horseshoe", SI_NODES, np.array([0, 1]), 1.0, X, d=SI_D, cutoff=0.0, offset=0.0)
    assert abs(np.trace(J)) < 1e-14


@pytest.mark.parametrize("seed", range(4))
def test_source_and_doublet_properties(O, seed):
    """test/runtests_elements.jl:220-315: square panel in z = 0."""
    rng = np.random.default_rng(500 + seed)
    nodes = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], float)
    panel = np.arange(4)
    hinf = rng.choice([-1, 1]) * 1e10
    h = rng.choice([-1, 1]) * 1e-8
    off = np.append((np.round(rng.random(2), 3) - 0.5) * 1.99, 0)
    n = np.array([0, 0, 1.0])
    T = np.stack([off, hinf * n + off, h * n + off])
    phis = O.phi_constant_source(nodes, panel, 1.0, T, offset=0.0)
    assert abs(phis[1]) < 1e-5
    assert abs((phis[2] - phis[0]) / h - np.sign(h) * 0.5) < 1e-6
    phid = O.phi_constant_doublet(nodes, panel, 1.0, T)
    assert abs(phid[1]) < 1e-7
    assert abs(phid[2] - np.sign(-h) * 0.5) < 1e-6


@pytest.mark.parametrize("seed", range(4))
def test_semiinfinite_doublet_properties(O, seed):
    """test/runtests_semiinfiniteelements.jl:175-241."""
    rng = np.random.default_rng(600 + seed)
    hinf = rng.choice([-1, 1]) * 1e14
    h = rng.choice([-1, 1]) * 1e-8
    n = np.array([0, 0, 1.0])
    T = np.stack([np.zeros(3), hinf * n, h * n])
    phis = O.phi_semiinfinite_doublet(SI, np.array([0, 1]), np.array([1.0, 0, 0]), 1.0, T)
    assert abs(phis[1]) < 1e-8
    assert abs(phis[2] - (-np.sign(-h) * 0.5)) < 1e-8


def test_nonunit_direction_rejected(O):
    with pytest.raises(ValueError, match="non-unitary"):
        O.U_semiinfinite_horseshoe(SI_NODES, (0, 1), [1.0, 0, 0.1], [1.0, 0, 0], 1.0, np.ones((1, 3)))


def test_opcounts_pinned(O):
    """Per-interaction operation counts of the reference formulas (sqrt, log,
    atan2, abs and division as one operation), used by the roofline."""
    assert O.opcount("filament") == 62
    assert O.opcount("ring", 4) == 248
    assert O.opcount("ring", 3) == 186
    assert O.opcount("semiinfinite") == 114
    assert O.opcount("horseshoe") == 290
    assert O.opcount("source", 4) == 534


def test_horseshoe_is_three_filaments(O):
    """U_semiinfinite_horseshoe == semi-infinite(-G) + bound + semi-infinite(+G)
    (src/FLOWPanel_elements.jl:692-730), checked against a long closed ring."""
    p = np.array([[0, 0, 0], [0, 1, 0]], float)
    d = np.array([1.0, 0, 0])
    X = np.array([[0.3, 0.4, 0.5], [-1.0, 0.2, 0.3]])
    hs = O.U_semiinfinite_horseshoe(p, (0, 1), d, d, 1.0, X, cutoff=0, offset=0)
    L = 1e7
    ring_nodes = np.array([[L, 0, 0], [0, 0, 0], [0, 1, 0], [L, 1, 0]], float)
    ring = O.U_vortexring(ring_nodes, np.arange(4), 1.0, X, cutoff=0, offset=0)
    assert np.allclose(hs, ring, rtol=1e-6, atol=1e-12)
