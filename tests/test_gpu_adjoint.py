"""GPU adjoint: the transposed solve on the saved factors and the reverse-mode
assembly / induced-velocity kernels, through the C ABI, against the oracle.

* A^T lambda = ybar: against LAPACK on the oracle's AIC, 1e-10 relative (FP64
  factors; FP32 factors after FP64 refinement to a 1e-12 residual).
* Reverse mode: for random directions v of every input, <grad, v> from the
  CUDA reverse pass equals the forward-mode (Dual number) derivative of the
  oracle to 1e-9 of sum |grad_k v_k| (the two differ only in summation order
  and in the algebraic form of the derivative).
"""
import numpy as np
import pytest
import scipy.linalg as sla

from conftest import freestream

pytestmark = pytest.mark.gpu


def _wing(fp, nc=10, ns=8, tri=False):
    w = fp.meshes.swept_wing("0012", nc, ns)
    if tri:
        w = fp.meshes.triangulate(w)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    V = freestream(4.2)
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    return w, normals, cps, D, U


def _setup(fp, ctx, w, normals, cps, D, prec):
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    ctx.assemble(fp._capi.FP_ELEMENT_VORTEXRING, precision=prec)
    ctx.factor(prec)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_adjoint_solve_matches_lapack(fp, O, ctx, prec):
    P = fp._capi.FP_PREC_FP64 if prec == "fp64" else fp._capi.FP_PREC_MIXED
    w, normals, cps, D, U = _wing(fp, 20, 24)
    _setup(fp, ctx, w, normals, cps, D, P)
    G = O.assemble_vortexring(w, cps, normals, D, D)
    rng = np.random.default_rng(1)
    ybar = rng.standard_normal((3, w.npanels))
    lam = ctx.adjoint_solve(ybar)
    ref = sla.solve(G.T, ybar.T).T
    err = np.abs(lam - ref).max() / np.abs(ref).max()
    assert err < 1e-10, err


@pytest.mark.parametrize("tri", [False, True])
def test_assembly_vjp_matches_dual_oracle(fp, O, ctx, tri):
    w, normals, cps, D, U = _wing(fp, 10, 8, tri)
    _setup(fp, ctx, w, normals, cps, D, fp._capi.FP_PREC_FP64)
    n, nsh = w.npanels, w.nsheddings
    rng = np.random.default_rng(2)
    lam = rng.standard_normal(n)
    gam = rng.standard_normal(n)
    g = ctx.assembly_vjp(U, w.nodes.shape[0], lam=lam, gamma=gam)
    dirs = {"dnodes": rng.standard_normal(w.nodes.shape), "dcps": rng.standard_normal((n, 3)),
            "dnormals": rng.standard_normal((n, 3)), "dUinfs": rng.standard_normal((n, 3)),
            "dDas": rng.standard_normal((nsh, 3)), "dDbs": rng.standard_normal((nsh, 3))}
    for key, v in dirs.items():
        _, dF = O.residual_jvp(w, cps, normals, D, D, U, lam, gam, **{key: v})
        got = float(np.sum(g[key] * v))
        scale = float(np.sum(np.abs(g[key] * v)))
        assert abs(got - dF) <= 1e-9 * scale, (key, got, dF, scale)


def test_uind_vjp_matches_dual_oracle(fp, O, ctx):
    w, normals, cps, D, U = _wing(fp, 10, 8)
    _setup(fp, ctx, w, normals, cps, D, fp._capi.FP_PREC_FP64)
    n, nsh = w.npanels, w.nsheddings
    rng = np.random.default_rng(3)
    s = rng.standard_normal(n)
    X = rng.uniform([-1, -3, -1], [3, 3, 1], size=(200, 3))
    X = np.concatenate([X, cps + 0.02 * normals])   # near-surface probes as CL uses
    m = X.shape[0]
    wbar = rng.standard_normal((m, 3))
    g = ctx.uind_vjp(s, X, wbar, w.nodes.shape[0])
    dirs = {"dnodes": rng.standard_normal(w.nodes.shape), "dtargets": rng.standard_normal((m, 3)),
            "dstrengths": rng.standard_normal(n), "dDas": rng.standard_normal((nsh, 3)),
            "dDbs": rng.standard_normal((nsh, 3))}
    for key, v in dirs.items():
        _, dF = O.uind_jvp(w, s, D, D, X, wbar, **{key: v})
        got = float(np.sum(g[key] * v))
        scale = float(np.sum(np.abs(g[key] * v)))
        assert abs(got - dF) <= 1e-9 * scale, (key, got, dF, scale)


def test_assembly_vjp_device_resident_inputs(fp, ctx):
    """lambda / gamma taken from the device results of fp_adjoint_solve /
    fp_solve equal the same values passed from the host."""
    w, normals, cps, D, U = _wing(fp, 10, 8)
    _setup(fp, ctx, w, normals, cps, D, fp._capi.FP_PREC_FP64)
    ctx.set_rhs(U)
    x, _ = ctx.solve(1, fp._capi.make_opts())
    ybar = np.random.default_rng(4).standard_normal(w.npanels)
    lam = ctx.adjoint_solve(ybar)[0]
    g_dev = ctx.assembly_vjp(U, w.nodes.shape[0])
    g_host = ctx.assembly_vjp(U, w.nodes.shape[0], lam=lam, gamma=x)
    for k in g_dev:
        np.testing.assert_allclose(g_dev[k], g_host[k], rtol=1e-12, atol=1e-14 * np.abs(g_host[k]).max())
