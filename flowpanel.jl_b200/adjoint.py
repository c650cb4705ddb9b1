"""Reverse-mode derivatives of the GPU solve, as ``torch.autograd.Function``s.

The reference differentiates ``solve`` through ForwardDiff duals and the
ImplicitAD rule of its linear solve (src/FLOWPanel_linearsolver.jl:73,128);
the Julia drop-in exposes the same pullbacks as a ChainRulesCore ``rrule``.
Here the two device calls of the hot path are autograd Functions:

* ``PanelSolve``: Gamma = A(nodes, CPs, normals, Das, Dbs)^-1 b(Uinfs, normals).
  Backward: lambda = A^-T dGamma (``fp_adjoint_solve`` on the saved factors),
  then the reverse-mode assembly ``fp_assembly_vjp`` gives the gradients of
  lambda^T (b - A Gamma) with respect to every input.
* ``InducedVelocity``: U = Uind(Gamma, targets) of the vortex-ring body.
  Backward: ``fp_uind_vjp``.

The O(N) geometry (normals, control points, areas) and post-processing (Cp
with the Kutta average, forces, CL, CD) are written with torch (CPU, float64),
so autograd chains them around the device calls, as ForwardDiff does around
the reference's CPU code.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi

F64 = torch.float64


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64, copy=False)


class _Geom:
    """Connectivity of a mesh in the forms the torch functions index with."""

    def __init__(self, mesh):
        offs = mesh.panel_offsets
        nn = np.diff(offs)
        idx = np.zeros((mesh.npanels, 4), np.int64)
        for k in range(4):
            sel = nn > k
            idx[sel, k] = mesh.panel_nodes[offs[:-1][sel] + k]
        self.mesh = mesh
        self.idx = torch.from_numpy(idx)
        self.nn = torch.from_numpy(nn.astype(np.float64))
        self.mask = (torch.arange(4)[None, :] < self.nn[:, None]).to(F64)
        self.quad = torch.from_numpy(nn == 4)
        sh = mesh.shedding.reshape(-1, 6) if mesh.nsheddings else np.zeros((0, 6), np.int64)
        self.shedding = sh
        low = sh[:, 3] != -1
        self.k4 = torch.from_numpy(np.stack([sh[low, 0], sh[low, 0] + 1, sh[low, 3], sh[low, 3] - 1]).astype(np.int64))
        self.k2 = torch.from_numpy(np.stack([sh[~low, 0], sh[~low, 0] + 1]).astype(np.int64))


def geometry(g: _Geom, nodes, cp_off=1e-14, l=1.0):
    """Normals, control points and areas of calc_normals / calc_controlpoints /
    calc_areas (src/FLOWPanel_abstractbody.jl:635-776,905-927) as torch ops."""
    P = nodes[g.idx]                              # (N, 4, 3)
    e = P[:, 1] - P[:, 0]
    f = P[:, 2] - P[:, 0]
    t = e / torch.linalg.norm(e, dim=1, keepdim=True)
    c = torch.cross(e, f, dim=1)
    cn = torch.linalg.norm(c, dim=1, keepdim=True)
    n = c / cn
    o = torch.cross(n, t, dim=1)
    m = g.mask[:, :, None]
    cen = (P * m).sum(1) / g.nn[:, None]
    d = (P - cen[:, None, :]) * m
    x = torch.einsum("pkd,pd->p", d, t) / g.nn
    y = torch.einsum("pkd,pd->p", d, o) / g.nn
    cen = cen + x[:, None] * t + y[:, None] * o
    area = 0.5 * cn[:, 0]
    c2 = torch.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0], dim=1)
    area = area + torch.where(g.quad, 0.5 * torch.linalg.norm(c2, dim=1), torch.zeros_like(area))
    cps = cen + (cp_off * l) * n
    return n, cps, cen, area


def kutta_average(g: _Geom, Cp):
    """Cp averaged over (pi, pi+1, pj, pj-1) at each shedding edge
    (src/FLOWPanel_postprocess.jl:1075-1097)."""
    out = Cp.clone()
    if g.k4.shape[1]:
        ave = Cp[g.k4].mean(0)
        for r in range(4):
            out = out.index_put((g.k4[r],), ave)
    if g.k2.shape[1]:
        ave = Cp[g.k2].mean(0)
        for r in range(2):
            out = out.index_put((g.k2[r],), ave)
    return out


class PanelSolve(torch.autograd.Function):
    """Gamma of the vortex-ring body with Kutta wake (fp_solve_body)."""

    @staticmethod
    def forward(fctx, solver, g, nodes, cps, normals, Uinfs, Das, Dbs, kerneloffset, kernelcutoff):
        c = solver.ctx
        m = g.mesh
        c.set_geometry(_np(nodes), m.panel_offsets, m.panel_nodes, _np(cps), _np(normals))
        c.set_wake(m.shedding, _np(Das), _np(Dbs))
        x, st = c.solve_body(_capi.FP_ELEMENT_VORTEXRING, _np(Uinfs), kerneloffset, kernelcutoff, solver.opts)
        solver.stats = st.asdict()
        fctx.solver, fctx.nnodes = solver, nodes.shape[0]
        fctx.Uinfs = _np(Uinfs)
        return torch.from_numpy(np.array(x, dtype=np.float64))

    @staticmethod
    def backward(fctx, gG):
        c = fctx.solver.ctx
        c.adjoint_solve(_np(gG)[None, :])
        r = c.assembly_vjp(fctx.Uinfs, fctx.nnodes)   # lambda, Gamma from the device
        t = lambda k: torch.from_numpy(r[k])
        return (None, None, t("dnodes"), t("dcps"), t("dnormals"), t("dUinfs"), t("dDas"), t("dDbs"),
                None, None)


class InducedVelocity(torch.autograd.Function):
    """Uind of the solved vortex-ring body at targets (fp_uind), FP64."""

    @staticmethod
    def forward(fctx, solver, strengths, targets, nodes, Das, Dbs, kerneloffset, kernelcutoff):
        c = solver.ctx
        out = c.uind(_capi.FP_ELEMENT_VORTEXRING, _np(strengths), _np(targets), None, _capi.FP_PREC_FP64,
                     kerneloffset, kernelcutoff)
        fctx.solver, fctx.nnodes = solver, nodes.shape[0]
        fctx.s, fctx.x = _np(strengths).copy(), _np(targets).copy()
        return torch.from_numpy(out)

    @staticmethod
    def backward(fctx, gU):
        r = fctx.solver.ctx.uind_vjp(fctx.s, fctx.x, _np(gU), fctx.nnodes)
        t = lambda k: torch.from_numpy(r[k])
        return None, t("dstrengths"), t("dtargets"), t("dnodes"), t("dDas"), t("dDbs"), None, None


# ----------------------------------------------------------------------------- design variables
def twist_basis(nodes, nstations=13):
    """Section twist design variables: hat functions of the spanwise
    coordinate at ``nstations`` equally spaced stations, and each node's
    section quarter-chord point (leading edge + chord/4 of its section)."""
    y = nodes[:, 1]
    ys = np.linspace(y.min(), y.max(), nstations)
    phi = np.zeros((nodes.shape[0], nstations))
    k = np.clip(np.searchsorted(ys, y, side="right") - 1, 0, nstations - 2)
    s = (y - ys[k]) / (ys[k + 1] - ys[k])
    phi[np.arange(len(y)), k] = 1 - s
    phi[np.arange(len(y)), k + 1] += s
    key = np.round(y, 12)
    xqc = np.zeros(len(y))
    zqc = np.zeros(len(y))
    for v in np.unique(key):
        sel = key == v
        xs = nodes[sel, 0]
        le = np.argmin(xs)
        xqc[sel] = xs.min() + 0.25 * (xs.max() - xs.min())
        zqc[sel] = nodes[sel, 2][le]
    return phi, xqc, zqc


def apply_twist(nodes0, tau, phi, xqc, zqc):
    """Rotate each node about its section's quarter chord by the interpolated
    twist (radians; positive nose up, as the mesh generator's twist)."""
    a = torch.from_numpy(phi) @ tau
    xq, zq = torch.from_numpy(xqc), torch.from_numpy(zqc)
    dx, dz = nodes0[:, 0] - xq, nodes0[:, 2] - zq
    ca, sa = torch.cos(a), torch.sin(a)
    return torch.stack([xq + dx * ca + dz * sa, nodes0[:, 1], zq - dx * sa + dz * ca], dim=1)


# ----------------------------------------------------------------------------- objectives
def wing_coefficients(solver, g: _Geom, nodes, aoa, span, chord, rho=1.225, probe_offset=0.02,
                      kerneloffset=1e-8, kernelcutoff=1e-14, cp_offset=1e-14):
    """CL and CD of a lifting wing as the reference's solver tests compute
    them (test/runtests_solvers.jl:146-166): solve with the wake along the
    freestream, velocity at probes probe_offset*chord off the surface, Cp with
    the Kutta average, F = -Cp q A n, L and D projected on the wind axes.
    ``aoa`` in radians, |Vinf| = 1. Differentiable in ``nodes`` and ``aoa``."""
    n, cps, cen, area = geometry(g, nodes, cp_off=cp_offset)
    V = torch.stack([torch.cos(aoa), torch.zeros_like(aoa), torch.sin(aoa)])
    nsh = g.shedding.shape[0]
    Uinfs = V.expand(g.mesh.npanels, 3)
    Dw = V.expand(nsh, 3)
    gamma = PanelSolve.apply(solver, g, nodes, cps, n, Uinfs, Dw, Dw, kerneloffset, kernelcutoff)
    probes = cen + (probe_offset * chord) * n
    U = Uinfs + InducedVelocity.apply(solver, gamma, probes, nodes, Dw, Dw, kerneloffset, kernelcutoff)
    Cp = kutta_average(g, 1.0 - (U * U).sum(1))
    q = 0.5 * rho
    F = (-q * Cp * area)[:, None] * n
    Ftot = F.sum(0)
    Dhat = V / torch.linalg.norm(V)
    Shat = torch.tensor([0.0, 1.0, 0.0], dtype=F64)
    Lhat = torch.cross(Dhat, Shat, dim=0)
    nondim = q * span * chord
    return torch.dot(Ftot, Lhat) / nondim, torch.dot(Ftot, Dhat) / nondim


def induced_drag_metric(CL, CD, AR):
    """Span-efficiency-weighted induced drag J = CD / e with the span
    efficiency e = CL^2 / (pi AR CD), i.e. J = pi AR CD^2 / CL^2: the induced
    drag in units of the ideal elliptic-loading drag at the same lift. (The
    reference defines no such quantity; this is the definition used here.)"""
    return np.pi * AR * CD * CD / (CL * CL)
