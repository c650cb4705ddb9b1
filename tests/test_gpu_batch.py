"""Batched solves of bodies with uneven panel counts (fp_batch_solve): every
strength vector equals the one the same body gets from a solve of its own
(the same kernels run; 1e-12 relative for the refinement's stopping point),
and the FP64 batch matches the oracle's LAPACK solve to 1e-10 relative."""
import numpy as np
import pytest

from conftest import freestream

pytestmark = pytest.mark.gpu


def _wings(fp):
    sizes = [(12, 8, 45.0), (20, 24, 30.0), (16, 10, 10.0), (10, 6, 0.0), (24, 30, 20.0), (14, 16, 40.0)]
    out = []
    for nc, ns, sweep in sizes:
        w = fp.meshes.swept_wing("0012", nc, ns, 1.0, 5.0, sweep, 0.7)
        out.append(fp.RigidWakeBody(w))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_solves(fp, precision):
    bodies = _wings(fp)
    V = freestream(4.2)
    Us = [np.tile(V, (b.ncells, 1)) for b in bodies]
    Ds = [np.tile(V, (b.nsheddings, 1)) for b in bodies]
    stats = fp.solve_batch(bodies, Us, Ds, Ds, precision=precision, nslots=3)
    assert len(stats) == len(bodies)
    opts = fp._capi.make_opts("ludiv", precision)
    ctx = fp._capi.Context(0)
    try:
        for b, U, D in zip(bodies, Us, Ds):
            normals = fp.calc_normals(b)
            cps = fp.calc_controlpoints(b, normals)
            ctx.set_geometry(b.mesh.nodes, b.mesh.panel_offsets, b.mesh.panel_nodes, cps, normals)
            ctx.set_wake(b.mesh.shedding, D, D)
            x, _ = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, U, opts=opts)
            np.testing.assert_allclose(b.strength, x, rtol=1e-12, atol=1e-12 * np.abs(x).max())
    finally:
        ctx.close()


def test_batch_fp64_matches_oracle(fp, O):
    bodies = _wings(fp)[:3]
    V = freestream(4.2)
    Us = [np.tile(V, (b.ncells, 1)) for b in bodies]
    Ds = [np.tile(V, (b.nsheddings, 1)) for b in bodies]
    fp.solve_batch(bodies, Us, Ds, Ds, precision="fp64", nslots=2)
    for b, U, D in zip(bodies, Us, Ds):
        normals = fp.calc_normals(b)
        cps = fp.calc_controlpoints(b, normals)
        G = O.assemble_vortexring(b.mesh, cps, normals, D, D)
        ref = O.solve_ludiv(G, O.rhs_noflowthrough(U, normals))
        assert np.abs(b.strength - ref).max() <= 1e-10 * np.abs(ref).max()


def test_batch_reports_the_failing_body(fp):
    bodies = _wings(fp)[:3]
    V = freestream(4.2)
    Us = [np.tile(V, (b.ncells, 1)) for b in bodies]
    Ds = [np.tile(V, (b.nsheddings, 1)) for b in bodies]
    Ds[1] = 2.0 * Ds[1]   # non-unit wake direction: rejected like src/FLOWPanel_elements.jl:495-498
    with pytest.raises(fp._capi.FlowPanelError) as e:
        fp.solve_batch(bodies, Us, Ds, Ds, precision="fp64", nslots=2)
    assert "body 1" in str(e.value)
