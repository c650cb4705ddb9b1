"""The RAE 101 swept wing of the reference's solver test
(test/runtests_solvers.jl:25-177) on CPU: the simplewing loft pinned against
the reference's own lofted mesh, then the test's lift within 3 % of the
experimental CL = 0.238 through the oracle.

The wing: span b = 98 in, aspect ratio 5, no taper, twist or dihedral, 45 deg
sweep, RAE 101 section re-discretised with rfl_NDIVS = (0.25, 8, 10),
(0.50, 8, 1, central), (0.25, 8, 0.1); 8 span cells per side at expansion 10
lofted from each tip to the root; CPoffset = +-5e-9 with characteristic
length b/ar; vortex rings with a rigid wake; AoA 4.2 deg at 30 m/s. The
velocity is probed 0.02 b/ar off the surface (calcfield_U with offset), Cp
and F carry the Kutta correction, CL = sign(L.Lhat) |L| / (rho V^2 b^2 / (2 ar)).

The re-discretised section is the one of the reference's lofted mesh
(examples/data/sweptwing-{left,right}000.vtu, the same airfoil file and
rfl_NDIVS with 15 span cells), read from the committed fixture: the loft
reproduces that mesh exactly, nodes, triangles and shedding rows.
"""
import numpy as np
import pytest

from test_meshio import GOLDEN, SPANDIR, fixture_mesh, te_line

B = 98 * 0.0254
AR = 5.0
CL_EXP = 0.238


def rae101_section():
    """The RAE 101 section of the reference's lofted swept wing: 48 points on a
    unit chord from the trailing edge along the lower surface."""
    z = np.load(f"{GOLDEN}/sweptwing_vtu.npz")
    X = z["nodes_L"].reshape(16, 48, 3)
    c = B / AR
    return np.stack([(X[0, :, 0] - abs(X[0, 0, 1])) / c, X[0, :, 2] / c], axis=1)


def rae101_halves(fp, span_n, cpoffset):
    sec = rae101_section()
    L = fp.meshes.simplewing(sec, B, AR, 1.0, 45.0, 0.0, [(1.0, span_n, 10.0, False)], -1.0, 0.0, name="L",
                             CPoffset=cpoffset)
    R = fp.meshes.simplewing(sec, B, AR, 1.0, 45.0, 0.0, [(1.0, span_n, 10.0, False)], 1.0, 0.0, name="R",
                             CPoffset=-cpoffset)
    return L, R


def test_discretize_ndivs(fp):
    """Linear growth of the cell lengths by the expansion factor; central
    sections mirror it; sections split the length by their fractions."""
    M = fp.meshes
    x = M.discretize_ndivs([(1.0, 15, 10.0, False)])
    d = np.diff(x)
    assert len(x) == 16 and abs(x[-1] - 1.0) < 1e-15
    assert abs(d[-1] / d[0] - 10.0) < 1e-12 and np.allclose(np.diff(d), np.diff(d)[0])
    x = M.discretize_ndivs([(0.25, 8, 10.0, False), (0.5, 8, 1.0, True), (0.25, 8, 0.1, False)], 2.0)
    assert len(x) == 25 and abs(x[8] - 0.5) < 1e-14 and abs(x[16] - 1.5) < 1e-14
    assert np.allclose(np.diff(x[8:17]), 0.125)
    x = M.discretize_ndivs([(1.0, 6, 4.0, True)])
    d = np.diff(x)
    assert np.allclose(d, d[::-1]) and abs(d[2] / d[0] - 4.0) < 1e-12


def test_simplewing_loft_reproduces_reference_mesh(fp):
    """15 span cells per side: the loft gives the reference's lofted mesh
    (.vtu fixture) to round-off, the same triangles, and the shedding rows
    of generate_loft_liftbody equal the ones found from the trailing-edge
    line (meshio.calc_shedding)."""
    sec = rae101_section()
    for side, (lo, up) in (("L", (-1.0, 0.0)), ("R", (1.0, 0.0))):
        m = fp.meshes.simplewing(sec, B, AR, 1.0, 45.0, 0.0, [(1.0, 15, 10.0, False)], lo, up)
        ref = fixture_mesh(fp, side)
        assert np.abs(m.nodes - ref.nodes).max() < 1e-14
        assert np.array_equal(m.panel_offsets, ref.panel_offsets)
        assert np.array_equal(m.panel_nodes, ref.panel_nodes)
        line = te_line(fp, side)
        span = np.ptp(line @ np.asarray(SPANDIR[side], float))
        assert np.array_equal(m.shedding, fp.meshio.calc_shedding(ref, line, tolerance=0.001 * span))


def oracle_rae101(fp, O, span_n=8, cpoffset=5e-9):
    L, R = rae101_halves(fp, span_n, cpoffset)
    mesh = fp.meshes.concat([L, R])
    aoa, mag, rho = 4.2, 30.0, 1.225
    Vinf = mag * np.array([np.cos(np.deg2rad(aoa)), 0.0, np.sin(np.deg2rad(aoa))])
    cpoff = mesh.cpoffset()
    lch = np.full(mesh.npanels, B / AR)
    normals, cps, areas = O.geometry(mesh, off=cpoff, l=lch)
    D = np.tile(Vinf / mag, (mesh.nsheddings, 1))
    G = O.assemble_vortexring(mesh, cps, normals, D, D)
    Uinfs = np.tile(Vinf, (mesh.npanels, 1))
    gam = O.solve_ludiv(G, O.rhs_noflowthrough(Uinfs, normals))
    sgn = np.where(cpoff < 0, -1.0, 1.0)
    _, cps_off, _ = O.geometry(mesh, off=0.02 * sgn, l=lch)
    U = Uinfs + O.uind_vortexring(mesh, gam, D, D, cps_off)
    Cp = O.calcfield_Cp(U, mag, mesh.shedding)
    F = O.calcfield_F(Cp, areas, normals * sgn[:, None], mag, rho, mesh.shedding)
    Dhat = Vinf / mag
    Shat = np.array([0.0, 1.0, 0.0])
    Lhat = np.cross(Dhat, Shat)
    LDS = O.calcfield_LDS(F, Lhat, Dhat, Shat)
    nd = 0.5 * rho * mag ** 2 * B ** 2 / AR
    CL = np.sign(LDS[:, 0] @ Lhat) * np.linalg.norm(LDS[:, 0]) / nd
    CD = np.sign(LDS[:, 1] @ Dhat) * np.linalg.norm(LDS[:, 1]) / nd
    return dict(mesh=mesh, L=L, R=R, Vinf=Vinf, mag=mag, rho=rho, gam=gam, CL=CL, CD=CD, Lhat=Lhat, Dhat=Dhat,
                Shat=Shat, D=D, Uinfs=Uinfs)


def test_rae101_wing_lift_within_3pct_of_experiment(fp, O):
    """test/runtests_solvers.jl:135-176: |CL - 0.238| / 0.238 <= 0.03 (LU; the
    reference's backslash is the same LU here)."""
    r = oracle_rae101(fp, O)
    assert r["mesh"].npanels == 2 * 48 * 8 * 2
    err = abs(r["CL"] - CL_EXP) / CL_EXP
    assert err <= 0.03, (r["CL"], err)
    assert 0.0 < r["CD"] < 0.02
