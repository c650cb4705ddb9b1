"""Gradients of CL, CD and the induced-drag metric of a swept wing with
respect to every vertex coordinate, 13 section twists and the angle of
attack, by the adjoint (autograd through the GPU solve and field Functions),
checked two ways on a 20 x 24 panel coarsening of the 12k-panel wing:

* against forward mode through the CPU path: Dual-number assembly and field
  kernels of the oracle, LAPACK solve, torch forward mode for the O(N)
  geometry and post-processing (the stand-in for ForwardDiff through the
  reference); relative 1e-8 of the derivative's scale;
* against central finite differences of the GPU primal (FP64, h = 1e-6) on
  random unit directions; relative 2e-6 (FD truncation and rounding).
"""
import numpy as np
import pytest
import scipy.linalg as sla

pytestmark = pytest.mark.gpu

NC, NS, SPAN, AR, SWEEP, CHORD = 20, 24, 5.0, 5.0, 45.0, 1.0
AOA = np.deg2rad(4.2)


@pytest.fixture(scope="module")
def setup(fp):
    import torch
    A = fp.adjoint
    w = fp.meshes.swept_wing("0012", NC, NS, CHORD, SPAN, SWEEP, 1.0)
    g = A._Geom(w)
    phi, xqc, zqc = A.twist_basis(w.nodes, 13)
    solver = fp.B200Solver("ludiv", "fp64")
    yield dict(torch=torch, A=A, w=w, g=g, phi=phi, xqc=xqc, zqc=zqc, solver=solver)
    solver.close()


def _objectives(S, nodes0, tau, aoa):
    A = S["A"]
    nodes = A.apply_twist(nodes0, tau, S["phi"], S["xqc"], S["zqc"])
    CL, CD = A.wing_coefficients(S["solver"], S["g"], nodes, aoa, SPAN, CHORD)
    return CL, CD, A.induced_drag_metric(CL, CD, AR)


def _gradients(S, which):
    torch = S["torch"]
    nodes0 = torch.tensor(S["w"].nodes, dtype=torch.float64, requires_grad=True)
    tau = torch.zeros(13, dtype=torch.float64, requires_grad=True)
    aoa = torch.tensor(AOA, dtype=torch.float64, requires_grad=True)
    out = _objectives(S, nodes0, tau, aoa)[which]
    out.backward()
    return float(out.detach()), nodes0.grad.numpy(), tau.grad.numpy(), float(aoa.grad)


def _primal(S, dnodes, dtau, daoa, h, which):
    torch = S["torch"]
    with torch.no_grad():
        nodes0 = torch.tensor(S["w"].nodes + h * dnodes, dtype=torch.float64)
        tau = torch.tensor(h * dtau, dtype=torch.float64)
        aoa = torch.tensor(AOA + h * daoa, dtype=torch.float64)
        return float(_objectives(S, nodes0, tau, aoa)[which])


def _forward_mode_oracle(fp, O, S, vn, vt, va, which):
    """d(objective) along (vn, vt, va) through the CPU path in forward mode."""
    torch = S["torch"]
    from torch.func import jvp
    A, g, w = S["A"], S["g"], S["w"]
    nodes0 = torch.tensor(w.nodes, dtype=torch.float64)

    def geom(n0, tau, aoa):
        nodes = A.apply_twist(n0, tau, S["phi"], S["xqc"], S["zqc"])
        n, cps, cen, area = A.geometry(g, nodes)
        V = torch.stack([torch.cos(aoa), torch.zeros_like(aoa), torch.sin(aoa)])
        return nodes, n, cps, area, V, cen + 0.02 * CHORD * n

    prim = (nodes0, torch.zeros(13, dtype=torch.float64), torch.tensor(AOA, dtype=torch.float64))
    tang = (torch.tensor(vn), torch.tensor(vt), torch.tensor(va, dtype=torch.float64))
    (nodes, n, cps, area, V, probes), (dnodes, dn, dcps, _darea, dV, dprobes) = jvp(geom, prim, tang)
    np_ = lambda t: t.detach().numpy()
    m = fp.meshes.Mesh(np_(nodes), w.panel_offsets, w.panel_nodes, w.shedding, w.bodies)
    N, nsh = w.npanels, w.nsheddings
    Vn, dVn = np_(V), np_(dV)
    U, D = np.tile(Vn, (N, 1)), np.tile(Vn, (nsh, 1))
    dU, dD = np.tile(dVn, (N, 1)), np.tile(dVn, (nsh, 1))
    G = O.assemble_vortexring(m, np_(cps), np_(n), D, D)
    lu = sla.lu_factor(G)
    gam = sla.lu_solve(lu, O.rhs_noflowthrough(U, np_(n)))
    _, dr = O.residual_jvp(m, np_(cps), np_(n), D, D, U, None, gam, dnodes=np_(dnodes), dcps=np_(dcps),
                           dnormals=np_(dn), dDas=dD, dDbs=dD, dUinfs=dU, vector=True)
    dgam = sla.lu_solve(lu, dr)
    Ui, dUi = O.uind_jvp(m, gam, D, D, np_(probes), None, dnodes=np_(dnodes), dtargets=np_(dprobes),
                         dstrengths=dgam, dDas=dD, dDbs=dD, vector=True)

    def post(Up, n_, area_, V_):
        Cp = A.kutta_average(g, 1.0 - (Up * Up).sum(1))
        q = 0.5 * 1.225
        Ftot = ((-q * Cp * area_)[:, None] * n_).sum(0)
        Dhat = V_ / torch.linalg.norm(V_)
        Lhat = torch.cross(Dhat, torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64), dim=0)
        CL = torch.dot(Ftot, Lhat) / (q * SPAN * CHORD)
        CD = torch.dot(Ftot, Dhat) / (q * SPAN * CHORD)
        return (CL, CD, A.induced_drag_metric(CL, CD, AR))[which]

    Up = torch.tensor(U + Ui)
    _, d = jvp(post, (Up, n, area, V), (torch.tensor(dU + dUi), dn, _darea, dV))
    return float(d)


@pytest.mark.parametrize("which", [0, 1, 2])
def test_gradient_matches_forward_mode_oracle(fp, O, setup, which):
    S = setup
    _, gn, gt, ga = _gradients(S, which)
    rng = np.random.default_rng(40 + which)
    for _ in range(3):
        vn = rng.standard_normal(S["w"].nodes.shape)
        vt = rng.standard_normal(13)
        va = float(rng.standard_normal())
        adj = float(np.sum(gn * vn) + np.dot(gt, vt) + ga * va)
        fwd = _forward_mode_oracle(fp, O, S, vn, vt, va, which)
        scale = float(np.sum(np.abs(gn * vn)) + np.sum(np.abs(gt * vt)) + abs(ga * va))
        assert abs(adj - fwd) <= 1e-8 * scale, (which, adj, fwd, scale)


def test_gradient_matches_central_differences(fp, setup):
    S = setup
    CL0, gn, gt, ga = _gradients(S, 0)
    rng = np.random.default_rng(4)
    h = 1e-6
    for _ in range(10):
        vn = rng.standard_normal(S["w"].nodes.shape)
        vn /= np.linalg.norm(vn)
        fd = (_primal(S, vn, np.zeros(13), 0.0, h, 0) - _primal(S, -vn, np.zeros(13), 0.0, h, 0)) / (2 * h)
        adj = float(np.sum(gn * vn))
        assert abs(adj - fd) <= 2e-6 * max(abs(fd), np.abs(gn).max()), (adj, fd)
    for k in (0, 6, 12):
        e = np.zeros(13)
        e[k] = 1.0
        fd = (_primal(S, 0 * S["w"].nodes, e, 0.0, h, 0) - _primal(S, 0 * S["w"].nodes, -e, 0.0, h, 0)) / (2 * h)
        assert abs(gt[k] - fd) <= 2e-6 * max(abs(fd), 1.0), (k, gt[k], fd)
    fd = (_primal(S, 0 * S["w"].nodes, np.zeros(13), 1.0, h, 0) -
          _primal(S, 0 * S["w"].nodes, np.zeros(13), -1.0, h, 0)) / (2 * h)
    assert abs(ga - fd) <= 2e-6 * max(abs(fd), 1.0), (ga, fd)
    # a lifting wing: dCL/dAoA is positive and of thin-wing magnitude
    assert 1.0 < ga < 2 * np.pi


@pytest.fixture(scope="module")
def setup12k(fp):
    import torch
    A = fp.adjoint
    w = fp.meshes.swept_wing("0012", 100, 120, CHORD, SPAN, SWEEP, 1.0)   # the 12,000-panel wing
    g = A._Geom(w)
    phi, xqc, zqc = A.twist_basis(w.nodes, 13)
    solver = fp.B200Solver("ludiv", "fp64")
    yield dict(torch=torch, A=A, w=w, g=g, phi=phi, xqc=xqc, zqc=zqc, solver=solver)
    solver.close()


def test_gradient_matches_central_differences_12k(fp, setup12k):
    """The gradient at full size: dCL with respect to every vertex coordinate
    of the 12,000-panel wing by the adjoint, against central finite
    differences of the GPU primal (FP64, h = 1e-6) on 50 random unit
    directions."""
    S = setup12k
    assert S["w"].npanels == 12000
    CL0, gn, gt, ga = _gradients(S, 0)
    assert np.all(np.isfinite(gn)) and 0.1 < CL0 < 0.5
    rng = np.random.default_rng(12)
    h = 1e-6
    scale = np.abs(gn).max()
    errs = []
    for _ in range(50):
        vn = rng.standard_normal(S["w"].nodes.shape)
        vn /= np.linalg.norm(vn)
        fd = (_primal(S, vn, np.zeros(13), 0.0, h, 0) - _primal(S, -vn, np.zeros(13), 0.0, h, 0)) / (2 * h)
        adj = float(np.sum(gn * vn))
        errs.append(abs(adj - fd) / max(abs(fd), scale))
    assert max(errs) <= 2e-6, max(errs)
