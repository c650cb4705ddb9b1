"""GPU parity of the least-squares solve of watertight vortex-ring bodies
(RigidWakeBody{VortexRing, 2} / MultiBody{VortexRing, 2},
src/FLOWPanel_liftingbody.jl:236-447, src/FLOWPanel_multibody.jl:373-617)
through the C ABI, against the oracle's restatement with LAPACK's LU.

Tolerance: the normal equations square the condition number, and the Gram
products are summed in a different order here and in BLAS, so the strengths
agree to eps * cond(Gls) relative (times a safety factor of 100), and in
every case to 1e-6."""
import numpy as np
import pytest

from conftest import freestream

pytestmark = pytest.mark.gpu


def _check(fp, O, body, U, D, pres, got):
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    G = O.assemble_vortexring(body.mesh, cps, normals, D, D) if body.nsheddings else \
        O.assemble_vortexring(body.mesh, cps, normals, np.zeros((0, 3)), np.zeros((0, 3)))
    rhs = -np.einsum("ij,ij->i", U, normals)
    ref, Gls = O.solve_leastsquares(G, rhs, pres)
    tol = min(1e-6, 100 * np.finfo(float).eps * np.linalg.cond(Gls))
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    for i, v in pres:
        assert got[i] == v


def test_watertight_ellipsoid(fp, O):
    """A closed vortex-ring body (its direct system is singular), no wake, the
    default prescription: first panel at 0."""
    m = fp.meshes.prolate_ellipsoid(4.0, 0.5, 24, 16, tail=1.0)
    body = fp.RigidWakeBody(m, watertight=True)
    U = np.tile(freestream(5.0), (m.npanels, 1))
    fp.solve(body, U, np.zeros((0, 3)), np.zeros((0, 3)))
    assert body.solved and body.check_field("Gamma")
    _check(fp, O, body, U, np.zeros((0, 3)), [(0, 0.0)], body.strength)


def test_prescribed_values_and_wake(fp, O):
    """A wing with its wake, two prescribed strengths (one nonzero), given out
    of order (they are sorted as the reference sorts them)."""
    w = fp.meshes.swept_wing("0012", 12, 16)
    body = fp.RigidWakeBody(w)
    V = freestream(4.2)
    U = np.tile(V, (w.npanels, 1))
    D = np.tile(V, (w.nsheddings, 1))
    pres = [(77, 0.3), (5, 0.0)]
    fp.solve(body, U, D, D, elprescribe=pres)
    _check(fp, O, body, U, D, pres, body.strength)


def test_multibody_automatic_prescription(fp, O):
    """MultiBody of a watertight fuselage and a wing: only the watertight
    member gets a prescribed panel (its first)."""
    fuse = fp.RigidWakeBody(fp.meshes.prolate_ellipsoid(6.0, 0.4, 20, 12, tail=1.0), watertight=True)
    wing = fp.RigidWakeBody(fp.meshes.swept_wing("0012", 10, 12))
    mb = fp.MultiBody([fuse, wing])
    assert fp.bodies.calc_elprescribe(mb) == [(0, 0.0)]
    V = freestream(3.0)
    U = np.tile(V, (mb.ncells, 1))
    D = np.tile(V, (mb.nsheddings, 1))
    fp.solve(mb, U, D, D)
    _check(fp, O, mb, U, D, [(0, 0.0)], mb.strength)


def test_bad_prescription(fp, ctx):
    w = fp.meshes.swept_wing("0012", 8, 8)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, fp.calc_controlpoints(body, normals), normals)
    U = np.tile(freestream(0.0), (w.npanels, 1))
    for pres in ([(3, 0.0), (3, 1.0)], [(w.npanels, 0.0)]):
        with pytest.raises(fp._capi.FlowPanelError, match="distinct and in"):
            ctx.solve_ls(U, pres)
