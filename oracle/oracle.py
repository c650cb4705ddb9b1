"""ORACLE — test infrastructure only.

Python face of the CPU restatement of FLOWPanel.jl's panel-method hot path
(``fp_oracle.hpp``). Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module, and only as the
checker: the product path is the CUDA library and never routes through here.

* element kernels, geometry, assembly and induced velocity: the C++ restatement
  (``_build/libfporacle.so``), bit-faithful to the reference's operation order;
* LU / ``ldiv!``: LAPACK ``dgetrf``/``dgetrs`` through scipy, the routine family
  Julia's ``LinearAlgebra.lu!`` calls (src/FLOWPanel_linearsolver.jl:57-78,173-234);
* GMRES: a restatement of Krylov.jl's restarted GMRES with the reference's
  defaults (memory=50, atol=rtol=sqrt(eps)) (src/FLOWPanel_linearsolver.jl:136-147);
* post-processing Cp / F / LDS: src/FLOWPanel_postprocess.jl:1059-1689.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfporacle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build():
    """Compile the restatement with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.fpo_opcount.restype = C.c_longlong
        for name in ("fpo_U_semiinfinite_vortex", "fpo_U_semiinfinite_horseshoe",
                     "fpo_phi_semiinfinite_doublet", "fpo_phi_semiinfinite_doublet2",
                     "fpo_assemble_vortexring", "fpo_uind_vortexring"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _pts(a):
    """(n,3) float64 C-contiguous == 3 x n column-major."""
    a = _f64(a)
    assert a.ndim == 2 and a.shape[1] == 3
    return a


# ----------------------------------------------------------------- elements
def U_constant_source(nodes, panel, strength, targets, dot_with=None, offset=1e-8):
    nodes, targets = _pts(nodes), _pts(targets)
    panel = _i32(panel)
    nt = targets.shape[0]
    out = np.zeros(nt if dot_with is not None else (nt, 3))
    dw = _pts(dot_with) if dot_with is not None else None
    lib().fpo_U_constant_source(_d(nodes), _i(panel), len(panel), C.c_double(strength), _d(targets),
                                C.c_longlong(nt), _d(out), _d(dw) if dw is not None else None,
                                C.c_double(offset))
    return out


def phi_constant_source(nodes, panel, strength, targets, offset=1e-8):
    nodes, targets = _pts(nodes), _pts(targets)
    panel = _i32(panel)
    out = np.zeros(targets.shape[0])
    lib().fpo_phi_constant_source(_d(nodes), _i(panel), len(panel), C.c_double(strength), _d(targets),
                                  C.c_longlong(len(out)), _d(out), C.c_double(offset))
    return out


def U_vortexring(nodes, panel, strength, targets, dot_with=None, cutoff=1e-14, offset=1e-8):
    nodes, targets = _pts(nodes), _pts(targets)
    panel = _i32(panel)
    nt = targets.shape[0]
    out = np.zeros(nt if dot_with is not None else (nt, 3))
    dw = _pts(dot_with) if dot_with is not None else None
    lib().fpo_U_vortexring(_d(nodes), _i(panel), len(panel), C.c_double(strength), _d(targets),
                           C.c_longlong(nt), _d(out), _d(dw) if dw is not None else None,
                           C.c_double(cutoff), C.c_double(offset))
    return out


def phi_constant_doublet(nodes, panel, strength, targets):
    nodes, targets = _pts(nodes), _pts(targets)
    panel = _i32(panel)
    out = np.zeros(targets.shape[0])
    lib().fpo_phi_constant_doublet(_d(nodes), _i(panel), len(panel), C.c_double(strength), _d(targets),
                                   C.c_longlong(len(out)), _d(out))
    return out


def U_semiinfinite_horseshoe(nodes, TE, da, db, strength, targets, dot_with=None,
                             cutoff=1e-14, offset=1e-8):
    nodes, targets = _pts(nodes), _pts(targets)
    nt = targets.shape[0]
    out = np.zeros(nt if dot_with is not None else (nt, 3))
    dw = _pts(dot_with) if dot_with is not None else None
    rc = lib().fpo_U_semiinfinite_horseshoe(_d(nodes), int(TE[0]), int(TE[1]), _d(_f64(da)), _d(_f64(db)),
                                            C.c_double(strength), _d(targets), C.c_longlong(nt), _d(out),
                                            _d(dw) if dw is not None else None, C.c_double(cutoff),
                                            C.c_double(offset))
    if rc:
        raise ValueError("Found non-unitary semi-infinite direction")
    return out


def phi_semiinfinite_doublet(nodes, TE, d, strength, targets, db=None, infinitelength=1e12):
    nodes, targets = _pts(nodes), _pts(targets)
    out = np.zeros(targets.shape[0])
    if db is None:
        rc = lib().fpo_phi_semiinfinite_doublet(_d(nodes), int(TE[0]), int(TE[1]), _d(_f64(d)),
                                                C.c_double(strength), _d(targets),
                                                C.c_longlong(len(out)), _d(out))
    else:
        rc = lib().fpo_phi_semiinfinite_doublet2(_d(nodes), int(TE[0]), int(TE[1]), _d(_f64(d)),
                                                 _d(_f64(db)), C.c_double(strength), _d(targets),
                                                 C.c_longlong(len(out)), _d(out),
                                                 C.c_double(infinitelength))
    if rc:
        raise ValueError("Invalid semi-infinite direction(s)")
    return out


def phi_body(mesh, kind, strengths, targets, Das=None, Dbs=None, offset=1e-8):
    """phi! of a body at targets (M, 3) -> (M,), by the reference's loops over
    panels and then shedding edges: constant sources
    (src/FLOWPanel_nonliftingbody.jl:221-250), constant doublets (:388-420),
    both with strengths (N, 2) (:763-815), or vortex rings plus the wake's
    semi-infinite doublets, (da, db) on the upper panel's TE nodes with its
    strength and (db, da) on the lower's (src/FLOWPanel_liftingbody.jl:664-742).
    kind: 'source' | 'doublet' | 'source+doublet' | 'vortexring'."""
    targets = _pts(targets)
    out = np.zeros(targets.shape[0])
    s = np.asarray(strengths, float)
    for i in range(mesh.npanels):
        pan = mesh.panel(i)
        if kind == "source":
            out += phi_constant_source(mesh.nodes, pan, s[i], targets, offset)
        elif kind == "source+doublet":
            out += phi_constant_source(mesh.nodes, pan, s[i, 0], targets, offset)
            out += phi_constant_doublet(mesh.nodes, pan, s[i, 1], targets)
        else:
            out += phi_constant_doublet(mesh.nodes, pan, s[i], targets)
    if kind == "vortexring":
        for e, (pi, nia, nib, pj, nja, njb) in enumerate(np.asarray(mesh.shedding).reshape(-1, 6)):
            P = mesh.panel(pi)
            out += phi_semiinfinite_doublet(mesh.nodes, (P[nia], P[nib]), Das[e], s[pi], targets, db=Dbs[e])
            if pj != -1:
                Q = mesh.panel(pj)
                out += phi_semiinfinite_doublet(mesh.nodes, (Q[nja], Q[njb]), Dbs[e], s[pj], targets, db=Das[e])
    return out


def grad_phi(kind, nodes, panel, strength, X, d=(1.0, 0.0, 0.0), offset=0.0):
    """grad(phi) at X by forward-mode duals. kind: 'source' | 'doublet' | 'semiinfinite'."""
    k = {"source": 0, "doublet": 1, "semiinfinite": 2}[kind]
    nodes = _pts(nodes)
    panel = _i32(panel)
    g = np.zeros(3)
    lib().fpo_grad_phi(k, _d(nodes), nodes.shape[0], _i(panel), len(panel), _d(_f64(d)),
                       C.c_double(strength), _d(_f64(X)), C.c_double(offset), _d(g))
    return g


def jac_U(kind, nodes, panel, strength, X, d=(1.0, 0.0, 0.0), cutoff=0.0, offset=0.0):
    """(U, dU_i/dX_j) at X by forward-mode duals. kind: 'source' | 'ring' | 'horseshoe'."""
    k = {"source": 0, "ring": 1, "horseshoe": 2}[kind]
    nodes = _pts(nodes)
    panel = _i32(panel)
    U = np.zeros(3)
    J = np.zeros(9)
    lib().fpo_jac_U(k, _d(nodes), nodes.shape[0], _i(panel), len(panel), _d(_f64(d)),
                    C.c_double(strength), _d(_f64(X)), C.c_double(cutoff), C.c_double(offset),
                    _d(U), _d(J))
    return U, J.reshape(3, 3)


def opcount(which, nn=4):
    """Operations per interaction as written in the reference (see fpo_opcount)."""
    k = {"filament": 0, "ring": 1, "semiinfinite": 2, "horseshoe": 3, "source": 4}[which]
    return int(lib().fpo_opcount(k, nn))


# ----------------------------------------------------------------- geometry
def geometry(mesh, off=None, l=None):
    """Normals, control points and areas of every panel.

    ``off``/``l`` per panel (CPoffset with the MultiBody sign rule already applied,
    and the characteristic length)."""
    npan = mesh.npanels
    nodes = _pts(mesh.nodes)
    offs, pn = _i32(mesh.panel_offsets), _i32(mesh.panel_nodes)
    off = _f64(np.broadcast_to(0.0 if off is None else off, (npan,)))
    l = _f64(np.broadcast_to(1.0 if l is None else l, (npan,)))
    normals = np.zeros((npan, 3))
    cps = np.zeros((npan, 3))
    areas = np.zeros(npan)
    lib().fpo_geometry(_d(nodes), _i(offs), _i(pn), C.c_longlong(npan), _d(off), _d(l),
                       _d(normals), _d(cps), _d(areas))
    return normals, cps, areas


# ----------------------------------------------------------------- assembly
def assemble_vortexring(mesh, cps, normals, Das, Dbs, offset=1e-8, cutoff=1e-14, nthreads=0):
    """Dense vortex-ring AIC with Kutta wake columns; returns G (ncp x npanels, Fortran order)."""
    cps, normals = _pts(cps), _pts(normals)
    ncp = cps.shape[0]
    G = np.zeros((ncp, mesh.npanels), order="F")
    sh = _i32(mesh.shedding.reshape(-1, 6)) if mesh.nsheddings else np.zeros((0, 6), np.int32)
    Das, Dbs = _pts(np.reshape(Das, (-1, 3))), _pts(np.reshape(Dbs, (-1, 3)))
    rc = lib().fpo_assemble_vortexring(_d(_pts(mesh.nodes)), _i(_i32(mesh.panel_offsets)),
                                       _i(_i32(mesh.panel_nodes)), C.c_longlong(mesh.npanels),
                                       _d(cps), _d(normals), C.c_longlong(ncp), _i(sh),
                                       C.c_longlong(len(sh)), _d(Das), _d(Dbs),
                                       C.c_double(offset), C.c_double(cutoff),
                                       G.ctypes.data_as(_dp), nthreads)
    if rc:
        raise ValueError("Found non-unitary semi-infinite direction")
    return G


def assemble_source(mesh, cps, normals, offset=1e-8, nthreads=0):
    cps, normals = _pts(cps), _pts(normals)
    ncp = cps.shape[0]
    G = np.zeros((ncp, mesh.npanels), order="F")
    lib().fpo_assemble_source(_d(_pts(mesh.nodes)), _i(_i32(mesh.panel_offsets)),
                              _i(_i32(mesh.panel_nodes)), C.c_longlong(mesh.npanels), _d(cps),
                              _d(normals), C.c_longlong(ncp), C.c_double(offset),
                              G.ctypes.data_as(_dp), nthreads)
    return G


def rhs_noflowthrough(Uinfs, normals):
    """calc_bc_noflowthrough!: RHS_i = -U_i . n_i (src/FLOWPanel_linearsolver.jl:297-312)."""
    Uinfs, normals = _pts(Uinfs), _pts(normals)
    return -(Uinfs[:, 0] * normals[:, 0] + Uinfs[:, 1] * normals[:, 1] + Uinfs[:, 2] * normals[:, 2])


def uind_vortexring(mesh, strength, Das, Dbs, targets, offset=1e-8, cutoff=1e-14, nthreads=0):
    targets = _pts(targets)
    out = np.zeros((targets.shape[0], 3))
    sh = _i32(mesh.shedding.reshape(-1, 6)) if mesh.nsheddings else np.zeros((0, 6), np.int32)
    rc = lib().fpo_uind_vortexring(_d(_pts(mesh.nodes)), _i(_i32(mesh.panel_offsets)),
                                   _i(_i32(mesh.panel_nodes)), C.c_longlong(mesh.npanels),
                                   _d(_f64(strength)), _i(sh), C.c_longlong(len(sh)),
                                   _d(_pts(np.reshape(Das, (-1, 3)))), _d(_pts(np.reshape(Dbs, (-1, 3)))),
                                   C.c_double(offset), C.c_double(cutoff), _d(targets),
                                   C.c_longlong(targets.shape[0]), _d(out), nthreads)
    if rc:
        raise ValueError("Found non-unitary semi-infinite direction")
    return out


def uind_source(mesh, strength, targets, offset=1e-8, nthreads=0):
    targets = _pts(targets)
    out = np.zeros((targets.shape[0], 3))
    lib().fpo_uind_source(_d(_pts(mesh.nodes)), _i(_i32(mesh.panel_offsets)),
                          _i(_i32(mesh.panel_nodes)), C.c_longlong(mesh.npanels),
                          _d(_f64(strength)), C.c_double(offset), _d(targets),
                          C.c_longlong(targets.shape[0]), _d(out), nthreads)
    return out


# ----------------------------------------------------------------- forward-mode derivatives
def _opt(a, shape):
    return None if a is None else _d(_f64(np.reshape(a, shape)))


def residual_jvp(mesh, cps, normals, Das, Dbs, Uinfs, lam, gamma, dnodes=None, dcps=None,
                 dnormals=None, dDas=None, dDbs=None, dUinfs=None, offset=1e-8, cutoff=1e-14,
                 nthreads=0, vector=False):
    """F = lam . (b - A gamma) (vortex-ring AIC with Kutta wake columns,
    b = -Uinf . n) and dF along the given directions, by Dual numbers (the
    oracle of the reverse-mode assembly). Returns (F, dF), or with
    ``vector=True`` the residual r = b - A gamma and its derivative dr."""
    n = mesh.npanels
    r = np.zeros(n) if vector else None
    dr = np.zeros(n) if vector else None
    sh = _i32(mesh.shedding.reshape(-1, 6)) if mesh.nsheddings else np.zeros((0, 6), np.int32)
    nsh = len(sh)
    F, dF = C.c_double(), C.c_double()
    lib().fpo_residual_jvp(_d(_pts(mesh.nodes)), _opt(dnodes, (-1, 3)), C.c_longlong(mesh.nodes.shape[0]),
                           _i(_i32(mesh.panel_offsets)), _i(_i32(mesh.panel_nodes)), C.c_longlong(n),
                           _d(_pts(cps)), _opt(dcps, (n, 3)), _d(_pts(normals)), _opt(dnormals, (n, 3)),
                           _i(sh), C.c_longlong(nsh), _d(_pts(np.reshape(Das, (-1, 3)))), _opt(dDas, (nsh, 3)),
                           _d(_pts(np.reshape(Dbs, (-1, 3)))), _opt(dDbs, (nsh, 3)),
                           _d(_pts(np.reshape(Uinfs, (n, 3)))), _opt(dUinfs, (n, 3)),
                           None if lam is None else _d(_f64(lam)), _d(_f64(gamma)), C.c_double(offset),
                           C.c_double(cutoff), C.byref(F), C.byref(dF), None if r is None else _d(r),
                           None if dr is None else _d(dr), nthreads)
    return (r, dr) if vector else (F.value, dF.value)


def uind_jvp(mesh, strengths, Das, Dbs, targets, wbar, dnodes=None, dtargets=None, dstrengths=None,
             dDas=None, dDbs=None, offset=1e-8, cutoff=1e-14, nthreads=0, vector=False):
    """F = sum_i wbar_i . Uind(targets_i) and dF along the given directions
    (Dual numbers). Returns (F, dF), or with ``vector=True`` the velocities
    U (m, 3) and their derivatives dU."""
    n = mesh.npanels
    targets = _pts(targets)
    m = targets.shape[0]
    U = np.zeros((m, 3)) if vector else None
    dU = np.zeros((m, 3)) if vector else None
    sh = _i32(mesh.shedding.reshape(-1, 6)) if mesh.nsheddings else np.zeros((0, 6), np.int32)
    nsh = len(sh)
    F, dF = C.c_double(), C.c_double()
    lib().fpo_uind_jvp(_d(_pts(mesh.nodes)), _opt(dnodes, (-1, 3)), C.c_longlong(mesh.nodes.shape[0]),
                       _i(_i32(mesh.panel_offsets)), _i(_i32(mesh.panel_nodes)), C.c_longlong(n),
                       _d(_f64(strengths)), _opt(dstrengths, (n,)), _i(sh), C.c_longlong(nsh),
                       _d(_pts(np.reshape(Das, (-1, 3)))), _opt(dDas, (nsh, 3)),
                       _d(_pts(np.reshape(Dbs, (-1, 3)))), _opt(dDbs, (nsh, 3)), _d(targets),
                       _opt(dtargets, (m, 3)), C.c_longlong(m),
                       None if wbar is None else _d(_pts(np.reshape(wbar, (m, 3)))),
                       C.c_double(offset), C.c_double(cutoff), C.byref(F), C.byref(dF),
                       None if U is None else _d(U), None if dU is None else _d(dU), nthreads)
    return (U, dU) if vector else (F.value, dF.value)


# ----------------------------------------------------------------- linear solvers
def lu_factor(G):
    """LAPACK dgetrf (partial pivoting), as Julia's LA.lu! (src/FLOWPanel_linearsolver.jl:173-185)."""
    import scipy.linalg as sla
    return sla.lu_factor(np.asfortranarray(G), check_finite=False)


def lu_solve(lu, b):
    import scipy.linalg as sla
    return sla.lu_solve(lu, b, check_finite=False)


def solve_ludiv(G, b):
    """solve_ludiv!: src/FLOWPanel_linearsolver.jl:57-78."""
    return lu_solve(lu_factor(G), b)


def solve_leastsquares(G, rhs, elprescribe):
    """The least-squares solve of a watertight vortex-ring body with the AIC G
    and RHS = -Uinf . n: prescribed strengths moved to the right-hand side,
    their columns dropped, normal equations Gred^T Gred Gamma = Gred^T r
    solved by LU (solve_ludiv!), the prescribed values put back
    (_G_U_RHS_leastsquares! and set_solution, src/FLOWPanel_liftingbody.jl:285-447).
    elprescribe: [(0-based index, value)]."""
    pres = sorted(elprescribe, key=lambda t: t[0])
    r = np.array(rhs, float)
    for i, v in pres:
        r = r - v * G[:, i]
    keep = np.setdiff1d(np.arange(G.shape[1]), [i for i, _ in pres])
    Gred = G[:, keep]
    tGred = np.ascontiguousarray(Gred.T)
    Gls = tGred @ Gred
    g = solve_ludiv(Gls, tGred @ r)
    out = np.zeros(G.shape[1])
    out[keep] = g
    for i, v in pres:
        out[i] = v
    return out, Gls


def gmres(A, b, memory=50, atol=None, rtol=None, itmax=None, x0=None, restart=False):
    """GMRES as the reference calls it (src/FLOWPanel_linearsolver.jl:136-147):
    Krylov.jl 0.9's gmres, whose default restart=false runs one Arnoldi process
    (modified Gram-Schmidt) with a basis that grows past `memory` (a storage
    hint), Givens rotations on the Hessenberg columns, and stops when the
    rotated residual estimate |z_{k+1}| <= atol + rtol ||r0|| (or on a
    breakdown h_{k+1,k} <= eps^(3/4), or after itmax = 2n steps).
    restart=True gives GMRES(memory), restarted from the true residual.
    Returns (x, niter, converged)."""
    eps = np.finfo(np.float64).eps
    atol = np.sqrt(eps) if atol is None else atol
    rtol = np.sqrt(eps) if rtol is None else rtol
    btol = eps ** 0.75
    n = len(b)
    itmax = 2 * n if itmax is None else itmax
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    r = b - A @ x if x0 is not None else b.copy()
    beta = np.linalg.norm(r)
    eps_stop = atol + rtol * beta
    it = 0
    if beta <= eps_stop:
        return x, 0, True
    while it < itmax:
        V = [r / beta]
        cols = []                        # rotated Hessenberg columns
        cs, sn, z = [], [], [beta]
        solved = False
        while it < itmax and not (restart and len(cols) >= memory):
            k = len(cols)
            w = A @ V[k]
            h = np.zeros(k + 2)
            for i in range(k + 1):       # modified Gram-Schmidt
                h[i] = np.dot(V[i], w)
                w = w - h[i] * V[i]
            h[k + 1] = np.linalg.norm(w)
            breakdown = h[k + 1] <= btol
            if not breakdown:
                V.append(w / h[k + 1])
            for i in range(k):
                t = cs[i] * h[i] + sn[i] * h[i + 1]
                h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1]
                h[i] = t
            den = np.hypot(h[k], h[k + 1])
            cs.append(h[k] / den)
            sn.append(h[k + 1] / den)
            h[k], h[k + 1] = den, 0.0
            z.append(-sn[k] * z[k])
            z[k] = cs[k] * z[k]
            cols.append(h)
            it += 1
            solved = abs(z[k + 1]) <= eps_stop
            if solved or breakdown:
                break
        kd = len(cols)
        R = np.zeros((kd, kd))
        for j, h in enumerate(cols):
            R[:j + 1, j] = h[:j + 1]
        y = np.linalg.solve(np.triu(R), np.asarray(z[:kd]))
        x = x + np.asarray(V[:kd]).T @ y
        r = b - A @ x
        beta = np.linalg.norm(r)
        if not restart:
            return x, it, solved
        if beta <= eps_stop:
            return x, it, True
    return x, it, False


# ----------------------------------------------------------------- post-processing
def calcfield_Cp(Us, Uref, shedding=None, correct_kuttacondition=True):
    """calcfield_Cp!: Cp = 1 - (|U|/Uref)^2 with the TE Kutta average over
    (pi, pi+1, pj, pj-1) (src/FLOWPanel_postprocess.jl:1059-1112)."""
    Us = np.asarray(Us, dtype=np.float64)
    Cp = 1 - (np.sqrt(np.sum(Us * Us, axis=1)) / Uref) ** 2
    if correct_kuttacondition and shedding is not None:
        for (pi, nia, nib, pj, nja, njb) in np.reshape(shedding, (-1, 6)):
            if pj != -1:
                ave = (Cp[pi] + Cp[pi + 1] + Cp[pj] + Cp[pj - 1]) / 4
                Cp[[pi, pi + 1, pj, pj - 1]] = ave
            else:
                ave = (Cp[pi] + Cp[pi + 1]) / 2
                Cp[[pi, pi + 1]] = ave
    return Cp


def calcfield_F(Cps, areas, normals, Uinf, rho, shedding=None, correct_kuttacondition=True):
    """calcfield_F!: F = -Cp q A n (normals already flipped by sign(CPoffset))
    with the TE override (src/FLOWPanel_postprocess.jl:1199-1307)."""
    normals = np.asarray(normals, dtype=np.float64)
    F = (-0.5 * rho * Uinf ** 2 * np.asarray(Cps) * np.asarray(areas))[:, None] * normals
    if correct_kuttacondition and shedding is not None:
        q = 0.5 * rho * Uinf ** 2
        for (pi, nia, nib, pj, nja, njb) in np.reshape(shedding, (-1, 6)):
            if pj != -1:
                idx = [pi, pi + 1, pj, pj - 1]
                ave = (Cps[pi] + Cps[pi + 1] + Cps[pj] + Cps[pj - 1]) / 4
            else:
                idx = [pi, pi + 1]
                ave = (Cps[pi] + Cps[pi + 1]) / 2
            for i in idx:
                F[i] = -ave * q * areas[i] * normals[i]
    return F


def calcfield_LDS(Fs, Lhat, Dhat, Shat=None):
    """calcfield_LDS!: project the summed force on L, D, S (src/FLOWPanel_postprocess.jl:1615-1652)."""
    Lhat, Dhat = np.asarray(Lhat, float), np.asarray(Dhat, float)
    Shat = np.cross(Lhat, Dhat) if Shat is None else np.asarray(Shat, float)
    Ftot = np.sum(np.asarray(Fs), axis=0)
    return np.stack([Lhat * np.dot(Ftot, Lhat), Dhat * np.dot(Ftot, Dhat), Shat * np.dot(Ftot, Shat)], axis=1)


# ----------------------------------------------------------------- surface velocity from grad(mu)
# calcfield_Ugradmu_cell! / _node! / calcfield_Ugradmu! of
# src/FLOWPanel_postprocess.jl:139-1042, on triangular cells. The mesh queries
# they make of GeometricTools (unvendored, version 2 per Project.toml:29) are
# restated from their use there:
#   neighbor(grid, ni, ci; preserveEdge=true) -> the cell across the edge from
#       the cell's local node ni to ni%3+1, none at a free edge;
#   get_nodal_data(grid, data; areas) -> per node, the area-weighted mean of the
#       data of the cells that contain it;
#   project_3d_2d! + get_tri_gradient! -> the in-plane gradient of the linear
#       interpolant of three nodal values, expressed in 3D.
def mesh_neighbors(mesh):
    """(N, 3) int: the cell across edge k (local nodes k -> k+1) of each
    triangle, -1 at a free edge."""
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    if np.any(np.diff(offs) != 3):
        raise ValueError("the grad(mu) schemes need triangular cells")
    owners = {}
    for c in range(mesh.npanels):
        p = pn[offs[c]:offs[c] + 3]
        for k in range(3):
            a, b = int(p[k]), int(p[(k + 1) % 3])
            owners.setdefault((min(a, b), max(a, b)), []).append((c, k))
    nb = -np.ones((mesh.npanels, 3), np.int64)
    for lst in owners.values():
        if len(lst) == 2:
            (c0, k0), (c1, k1) = lst
            nb[c0, k0] = c1
            nb[c1, k1] = c0
        elif len(lst) > 2:
            raise ValueError("an edge is shared by more than two cells")
    return nb


def nodal_data(mesh, values, areas):
    """Area-weighted mean of the cell values around every node."""
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    num = np.zeros(mesh.nnodes)
    den = np.zeros(mesh.nnodes)
    for c in range(mesh.npanels):
        for v in pn[offs[c]:offs[c + 1]]:
            num[v] += areas[c] * values[c]
            den[v] += areas[c]
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(den > 0, num / np.where(den > 0, den, 1.0), 0.0)


def _gg_term(P, tri, k, nc, cpc, cpn, gc, gn, area, hs):
    """One Green-Gauss face term of the cell scheme times hs = 0.5*sign(CPoffset)
    (postprocess.jl:189-247)."""
    ei, ej = k, (k + 1) % 3
    r1 = P[tri[ej], 0] - P[tri[ei], 0]
    r2 = P[tri[ej], 1] - P[tri[ei], 1]
    r3 = P[tri[ej], 2] - P[tri[ei], 2]
    d1 = r2 * nc[2] - r3 * nc[1]
    d2 = r3 * nc[0] - r1 * nc[2]
    d3 = r1 * nc[1] - r2 * nc[0]
    dmag = np.sqrt(d1 * d1 + d2 * d2 + d3 * d3)
    d1, d2, d3 = d1 / dmag, d2 / dmag, d3 / dmag
    vm = P[tri[ei]] - cpc
    vn = P[tri[ei]] - cpn
    r = np.array([r1, r2, r3])
    dMain = np.linalg.norm(np.cross(vm, r))
    dNear = np.linalg.norm(np.cross(vn, r))
    f = dNear / (dMain + dNear)
    face = f * gc + (1.0 - f) * gn
    mag = face * np.sqrt(r1 * r1 + r2 * r2 + r3 * r3) / area
    return np.array([hs * d1 * mag, hs * d2 * mag, hs * d3 * mag])


def ugradmu_cell(mesh, gammas, areas, normals, cps, cpsign, nb=None, maxgrad=np.inf, smooth=None, passes=0):
    """calcfield_Ugradmu_cell! (src/FLOWPanel_postprocess.jl:270-540, the
    RigidWakeBody method; without shedding rows it is the AbstractBody method
    of :139-268): Green-Gauss over the cell's edges with the inverse-distance
    face value, then the face terms of the trailing-edge cells added back.
    ``cpsign`` is sign(CPoffset) per cell (1 where CPoffset = 0)."""
    P = np.asarray(mesh.nodes, float)
    nb = mesh_neighbors(mesh) if nb is None else nb
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    out = np.zeros((mesh.npanels, 3))

    def terms(ci):
        tri = pn[offs[ci]:offs[ci] + 3]
        for k in range(3):
            n = nb[ci, k]
            if n >= 0:
                yield _gg_term(P, tri, k, normals[ci], cps[ci], cps[n], gammas[ci], gammas[n], areas[ci],
                               0.5 * cpsign[ci])

    for ci in range(mesh.npanels):
        for t in terms(ci):
            out[ci] -= t
    for (pi, nia, nib, pj, nja, njb) in np.reshape(mesh.shedding, (-1, 6)):
        for ci in ((pi, pj) if pj != -1 else (pi,)):
            for t in terms(ci):
                out[ci] += t
    if smooth is not None and passes > 0:
        smooth_cells(mesh, out, smooth, passes, nb)
    big = np.linalg.norm(out, axis=1) >= maxgrad
    out[big] = 0.0
    return out


def tri_gradient(p1, p2, p3, v1, v2, v3):
    """In-plane gradient of the linear function through (p_k, v_k)."""
    e1 = p2 - p1
    x2 = np.linalg.norm(e1)
    e1 = e1 / x2
    w = p3 - p1
    x3 = np.dot(w, e1)
    e2 = w - x3 * e1
    y3 = np.linalg.norm(e2)
    e2 = e2 / y3
    gx = (v2 - v1) / x2
    gy = (v3 - v1 - gx * x3) / y3
    return gx * e1 + gy * e2


def te_cells(mesh):
    """The trailing-edge cells of the sharp-TE node scheme: the upper cells
    pi, pi+1 and the lower cells pj, pj-1 of every shedding row (the last and
    first two loop cells of a lofted grid, postprocess.jl:705-712), in row
    order, and the trailing-edge nodes (the upper edge's nodes)."""
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    up, lo, te = [], [], []
    for (pi, nia, nib, pj, nja, njb) in np.reshape(mesh.shedding, (-1, 6)):
        for c in (pi, pi + 1):
            if 0 <= c < mesh.npanels and c not in up:
                up.append(int(c))
        if pj != -1:
            for c in (pj, pj - 1):
                if 0 <= c < mesh.npanels and c not in lo:
                    lo.append(int(c))
        for k in (nia, nib):
            v = int(pn[offs[pi] + k])
            if v not in te:
                te.append(v)
    return up, lo, te


def nodal_data_cells(mesh, values, areas, nodes, cells):
    """Nodal values at `nodes` from the given cells only: the area-weighted mean
    over those of `cells` that contain the node (GeometricTools'
    get_nodal_data_TEcells, restated in the weighting of nodal_data)."""
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    out = {}
    for v in nodes:
        num = den = 0.0
        for c in cells:
            if v in pn[offs[c]:offs[c + 1]]:
                num += areas[c] * values[c]
                den += areas[c]
        out[v] = num / den if den > 0 else 0.0
    return out


def ugradmu_node(mesh, gammas, areas, cpsign, sharpTE=False):
    """calcfield_Ugradmu_node! (src/FLOWPanel_postprocess.jl:622-748): nodal
    values as the area-weighted mean of the cells around each node, the
    cell's linear gradient of them (the nodal values take the sign of
    CPoffset), times -1/2. With sharpTE the trailing-edge cells take, at the
    trailing-edge nodes, the nodal values of their own side only: the upper
    cells first, then the lower ones (postprocess.jl:698-742)."""
    P = np.asarray(mesh.nodes, float)
    nodal = nodal_data(mesh, gammas, areas)
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    out = np.zeros((mesh.npanels, 3))

    def grad(ci, nod):
        v = pn[offs[ci]:offs[ci] + 3]
        s = cpsign[ci]
        return tri_gradient(P[v[0]], P[v[1]], P[v[2]], s * nod[v[0]], s * nod[v[1]], s * nod[v[2]])

    for ci in range(mesh.npanels):
        out[ci] = grad(ci, nodal)
    if sharpTE and mesh.nsheddings > 0:
        up, lo, te = te_cells(mesh)
        for cells in (up, lo):
            side = nodal.copy()
            for v, val in nodal_data_cells(mesh, gammas, areas, te, cells).items():
                side[v] = val
            for ci in cells:
                out[ci] = grad(ci, side)
    return -0.5 * out


def smooth_cells(mesh, out, cells, passes, nb=None):
    """smoothPass / smoothRows of calcfield_Ugradmu_cell!
    (src/FLOWPanel_postprocess.jl:501-526): `passes` times, each listed cell in
    order takes the mean of its neighbours' current values, in place."""
    nb = mesh_neighbors(mesh) if nb is None else nb
    for _ in range(passes):
        for ci in cells:
            acc = np.zeros(3)
            k = 0
            for n in nb[ci]:
                if n >= 0:
                    acc += out[n]
                    k += 1
            out[ci] = acc / k
    return out


def ugradmu(mesh, gammas, areas, normals, cps, cpsign, force_cellTE=True, anglecrit=30.0, sharpTE=False):
    """calcfield_Ugradmu! (src/FLOWPanel_postprocess.jl:825-941): the cell
    scheme, except where a cell has a free edge or a neighbour whose normal is
    more than ``anglecrit`` degrees off, which take the node scheme (with the
    cell values forced on the TE cells pi, pi+1, pj, pj-1). Returns
    (out, out_cell, out_node)."""
    import math

    nb = mesh_neighbors(mesh)
    oc = ugradmu_cell(mesh, gammas, areas, normals, cps, cpsign, nb)
    on = ugradmu_node(mesh, gammas, areas, cpsign, sharpTE=sharpTE)
    if force_cellTE:
        for (pi, nia, nib, pj, nja, njb) in np.reshape(mesh.shedding, (-1, 6)):
            on[pi] = oc[pi]
            on[pi + 1] = oc[pi + 1]
            if pj != -1:
                on[pj] = oc[pj]
                on[pj - 1] = oc[pj - 1]
    cc = math.cos(math.radians(anglecrit))
    out = np.zeros((mesh.npanels, 3))
    for ci in range(mesh.npanels):
        use_node = False
        for k in range(3):
            n = nb[ci, k]
            if n < 0 or np.dot(normals[ci], normals[n]) < cc:
                use_node = True
                break
        out[ci] = on[ci] if use_node else oc[ci]
    return out, oc, on
