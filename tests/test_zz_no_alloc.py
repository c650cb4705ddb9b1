"""fp_lu_solve_noalloc: the FP64 solve on caller-owned device memory whose
triangular-solve flags live in a static device array (no device allocation
by the library). Two calls in a row are compared with the solution of the
existing entry point fp_solve (LU, FP64) on the same factors.

This file is collected last, so it runs both after the other GPU tests (which
leave their own contexts and allocations behind) and alone.

Tolerance: 1e-12 relative to the largest strength. Both paths run the same
pivoting and triangular-solve kernels; the right-hand side here is formed on
the host (-U.n) instead of by the RHS kernel, which moves the last bits.
"""
import ctypes

import numpy as np
import pytest

from conftest import freestream

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _factored_wing(fp, ctx, nc, ns):
    w = fp.meshes.swept_wing("0012", nc, ns)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    V = freestream(4.2)
    D = np.tile(V, (w.nsheddings, 1))
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    ctx.assemble(fp._capi.FP_ELEMENT_VORTEXRING)
    ctx.factor(fp._capi.FP_PREC_FP64)
    return w, normals, V


def _rhs(normals, Vs):
    return np.stack([-(normals @ V) for V in Vs])   # k x N


@pytest.mark.parametrize("nc,ns,k", [(20, 24, 1), (24, 40, 3)])
def test_noalloc_matches_fp_solve_twice(fp, nc, ns, k):
    import torch

    ctx = fp._capi.Context(0)
    try:
        w, normals, V = _factored_wing(fp, ctx, nc, ns)
        n = w.npanels
        Vs = [freestream(4.2 + 1.5 * q, 1.0 + 0.1 * q) for q in range(k)]
        ctx.set_rhs(np.concatenate([np.tile(Vq, (n, 1))[None] for Vq in Vs]))
        x_ref, _ = ctx.solve(k, fp._capi.make_opts(solver="ludiv", precision="fp64"))
        x_ref = np.atleast_2d(x_ref)
        b = _rhs(normals, Vs)
        ldb = n + 5   # a leading dimension larger than N
        scale = np.abs(x_ref).max()
        Bs = []
        for call in range(2):
            B = torch.zeros((k, ldb), dtype=torch.float64, device="cuda:0")
            B[:, :n] = torch.from_numpy(b)
            Bs.append(B)
        torch.cuda.synchronize()   # the library's stream does not wait for torch's
        for call, B in enumerate(Bs):
            free0 = torch.cuda.mem_get_info(0)[0]
            ctx.lu_solve_noalloc(B.data_ptr(), ldb, k)
            free1 = torch.cuda.mem_get_info(0)[0]
            if call == 1:   # the first call may load device code; after it nothing is allocated
                assert free1 == free0, f"device free memory moved by {free0 - free1} bytes"
            x = B[:, :n].cpu().numpy()
            err = np.abs(x - x_ref).max() / scale
            assert err <= TOL, f"call {call}: max relative difference {err:.3e}"
            # rows beyond N in each column are left as they were
            assert torch.count_nonzero(B[:, n:]).item() == 0
    finally:
        ctx.close()


def test_noalloc_argument_and_state_errors(fp):
    L = fp._capi.lib()
    ctx = fp._capi.Context(0)
    try:
        w, normals, V = _factored_wing(fp, ctx, 12, 8)
        n = w.npanels
        fake = ctypes.c_void_p(1 << 40)   # never dereferenced: every call below is rejected first
        assert L.fp_lu_solve_noalloc(ctx.h, None, n, 1) == fp._capi.FP_EINVAL
        assert L.fp_lu_solve_noalloc(ctx.h, fake, n - 1, 1) == fp._capi.FP_EINVAL
        assert L.fp_lu_solve_noalloc(ctx.h, fake, n, 0) == fp._capi.FP_EINVAL
        # FP32 factors only: there are no FP64 factors to solve with
        ctx.assemble(fp._capi.FP_ELEMENT_VORTEXRING, precision=fp._capi.FP_PREC_MIXED)
        ctx.factor(fp._capi.FP_PREC_MIXED)
        assert L.fp_lu_solve_noalloc(ctx.h, fake, n, 1) == fp._capi.FP_ESTATE
    finally:
        ctx.close()
