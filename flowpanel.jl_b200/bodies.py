"""Host mirror of FLOWPanel.jl's body / solve / calcfield API over the C ABI.

Names, arguments and error behaviour follow the reference:
``solve(body, Uinfs, Das, Dbs; solver=...)`` (src/FLOWPanel_liftingbody.jl:172-216,
src/FLOWPanel_multibody.jl:312-364, src/FLOWPanel_nonliftingbody.jl:93-130),
``calcfield_U/Cp/F/LDS`` (src/FLOWPanel_postprocess.jl:28-110,1059-1689). The
solver object is the drop-in: ``B200Solver`` owns a device context and runs the
assembly, factorisation, solve, induced-velocity evaluation and the surface
post-processing (grad(mu) velocity, Cp, forces, L/D/S) on the GPU. Geometry
preprocessing (normals, control points) stays on the host, as in the
reference.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional

import numpy as np

from . import _capi
from .meshes import Body as BodyInfo
from .meshes import Mesh, concat


# ----------------------------------------------------------------------------- bodies
class AbstractBody:
    element = None

    def __init__(self, mesh: Mesh, CPoffset=1e-14, kerneloffset=1e-8, kernelcutoff=1e-14,
                 characteristiclength: Optional[Callable] = None, name=None):
        self.mesh = mesh
        self.ncells = mesh.npanels
        self.nnodes = mesh.nnodes
        self.nsheddings = mesh.nsheddings
        self.CPoffset = CPoffset
        self.kerneloffset = kerneloffset
        self.kernelcutoff = kernelcutoff
        self.characteristiclength = characteristiclength
        self.strength = np.zeros(self.ncells)
        self.fields: Dict[str, dict] = {}
        self.solved = False
        self.name = name or type(self).__name__
        if not mesh.bodies:
            mesh.bodies = [BodyInfo(self.name, self.kind, mesh.npanels, mesh.nsheddings, CPoffset,
                                    kerneloffset, kernelcutoff)]

    kind = "vortexring"

    # fields (src/FLOWPanel_abstractbody.jl:358-430)
    def add_field(self, name, ftype, data, entry):
        self.fields[name] = {"field_name": name, "field_type": ftype, "field_data": data, "entry_type": entry}

    def get_field(self, name):
        return self.fields[name]

    def check_field(self, name):
        return name in self.fields

    def _cp_off_vector(self, off):
        """Per-panel control-point offsets: a plain body uses ``off`` as given; a
        MultiBody multiplies it by each member's sign(CPoffset)
        (src/FLOWPanel_multibody.jl:664-676)."""
        return np.full(self.ncells, float(off))

    def _l_vector(self, characteristiclength):
        if characteristiclength is None:
            return np.ones(self.ncells)
        return np.array([float(characteristiclength(self.mesh.nodes.T, self.mesh.panel(i)))
                         for i in range(self.ncells)])


class NonLiftingBody(AbstractBody):
    """NonLiftingBody{E} (src/FLOWPanel_nonliftingbody.jl:32-72) with E one of
    "ConstantSource" (the default), "ConstantDoublet" or
    "ConstantSource+ConstantDoublet" (the reference's
    Union{ConstantSource, ConstantDoublet}, two strengths per panel)."""
    _ELEMENTS = {"ConstantSource": ("source", _capi.FP_ELEMENT_SOURCE),
                 "ConstantDoublet": ("doublet", _capi.FP_ELEMENT_VORTEXRING),
                 "ConstantSource+ConstantDoublet": ("source+doublet", _capi.FP_ELEMENT_SOURCE_DOUBLET)}
    kind = "source"
    element = _capi.FP_ELEMENT_SOURCE

    def __init__(self, mesh: Mesh, *args, element="ConstantSource", **kwargs):
        if element not in self._ELEMENTS:
            raise ValueError(f"unknown element {element}; expected one of {list(self._ELEMENTS)}")
        self.kind, self.element = self._ELEMENTS[element]
        super().__init__(mesh, *args, **kwargs)
        if self.kind == "source+doublet":
            self.strength = np.zeros((self.ncells, 2))


class RigidWakeBody(AbstractBody):
    """RigidWakeBody{VortexRing, 1} (src/FLOWPanel_liftingbody.jl:43-134); with
    watertight=True, RigidWakeBody{VortexRing, 2}, solved by least squares with
    prescribed strengths (:236-447)."""
    kind = "vortexring"
    element = _capi.FP_ELEMENT_VORTEXRING

    def __init__(self, mesh: Mesh, *args, watertight=False, **kwargs):
        self.watertight = watertight
        super().__init__(mesh, *args, **kwargs)


def calc_elprescribe(body: AbstractBody):
    """The default prescribed strengths of a least-squares solve, 0-based:
    the first panel of a watertight body at 0 (calc_elprescribe,
    src/FLOWPanel_liftingbody.jl:283), and for a MultiBody the first panel of
    each watertight member (src/FLOWPanel_multibody.jl:565-600)."""
    if isinstance(body, MultiBody):
        out, k = [], 0
        for b in body.bodies:
            if getattr(b, "watertight", False):
                out.append((k, 0.0))
            k += b.ncells
        return out
    return [(0, 0.0)] if getattr(body, "watertight", False) else []


class MultiBody(AbstractBody):
    """MultiBody of vortex-ring bodies (src/FLOWPanel_multibody.jl:19-79): the
    bodies' panels are concatenated in order; G's column blocks follow them."""
    kind = "vortexring"
    element = _capi.FP_ELEMENT_VORTEXRING

    def __init__(self, bodies: List[AbstractBody], names=None):
        kinds = {b.kind for b in bodies}
        if len(kinds) != 1:
            raise ValueError("MultiBody: all bodies must use the same element type")
        offs = {(b.kerneloffset, b.kernelcutoff) for b in bodies}
        if len(offs) != 1:
            raise ValueError("MultiBody: all bodies must share kerneloffset and kernelcutoff")
        self.bodies = bodies
        mesh = concat([b.mesh for b in bodies])
        for info, b in zip(mesh.bodies, bodies):
            info.CPoffset = b.CPoffset
        b0 = bodies[0]
        super().__init__(mesh, b0.CPoffset, b0.kerneloffset, b0.kernelcutoff, None, "MultiBody")
        self.kind = b0.kind
        self.element = b0.element

    def _cp_off_vector(self, off):
        out = np.empty(self.ncells)
        k = 0
        for b in self.bodies:
            s = np.sign(b.CPoffset) if b.CPoffset != 0 else 1.0
            out[k:k + b.ncells] = s * off
            k += b.ncells
        return out

    def _l_vector(self, characteristiclength):
        if characteristiclength is not None:
            return super()._l_vector(characteristiclength)
        return np.concatenate([b._l_vector(b.characteristiclength) for b in self.bodies])

    def _default_off(self):
        return np.concatenate([np.full(b.ncells, b.CPoffset) for b in self.bodies])


# ----------------------------------------------------------------------------- geometry
def _panel_arrays(mesh: Mesh):
    """Dense (N, 4) node index array (triangles repeat no node: nn recorded)."""
    offs = mesh.panel_offsets
    nn = np.diff(offs)
    idx = np.zeros((mesh.npanels, 4), np.int64)
    for k in range(4):
        sel = nn > k
        idx[sel, k] = mesh.panel_nodes[offs[:-1][sel] + k]
    return idx, nn


def _frame(mesh: Mesh):
    idx, nn = _panel_arrays(mesh)
    P = mesh.nodes
    e = P[idx[:, 1]] - P[idx[:, 0]]
    f = P[idx[:, 2]] - P[idx[:, 0]]
    t = e / np.linalg.norm(e, axis=1)[:, None]
    c = np.cross(e, f)
    n = c / np.linalg.norm(c, axis=1)[:, None]
    o = np.cross(n, t)
    return t, o, n, idx, nn


def calc_normals(body: AbstractBody, flipbyCPoffset=False):
    """Unit normals (N, 3) (src/FLOWPanel_abstractbody.jl:738-776)."""
    _, _, n, _, _ = _frame(body.mesh)
    if flipbyCPoffset:
        if isinstance(body, MultiBody):
            s = body._cp_off_vector(1.0)
            n = n * s[:, None]
        else:
            n = n * (np.sign(body.CPoffset) if body.CPoffset != 0 else 1.0)
    return n


def calc_controlpoints(body: AbstractBody, normals=None, off=None, characteristiclength=None):
    """Control points (N, 3): vertex mean, in-plane centroid correction, then
    + off * l * n (src/FLOWPanel_abstractbody.jl:635-694)."""
    t, o, n, idx, nn = _frame(body.mesh)
    normals = n if normals is None else normals
    P = body.mesh.nodes
    mask = (np.arange(4)[None, :] < nn[:, None]).astype(float)
    pts = P[idx] * mask[:, :, None]
    c = pts.sum(axis=1) / nn[:, None]
    d = (P[idx] - c[:, None, :]) * mask[:, :, None]
    x = np.einsum("pkd,pd->p", d, t) / nn
    y = np.einsum("pkd,pd->p", d, o) / nn
    c = c + x[:, None] * t + y[:, None] * o
    if off is None:
        offv = body._default_off() if isinstance(body, MultiBody) else np.full(body.ncells, body.CPoffset)
        l = body._l_vector(body.characteristiclength if not isinstance(body, MultiBody) else None)
    else:
        offv = body._cp_off_vector(off)
        l = body._l_vector(characteristiclength)
    return c + (offv * l)[:, None] * normals


def calc_areas(body: AbstractBody):
    """Panel areas (fan of triangles from the first node)."""
    idx, nn = _panel_arrays(body.mesh)
    P = body.mesh.nodes
    a = 0.5 * np.linalg.norm(np.cross(P[idx[:, 1]] - P[idx[:, 0]], P[idx[:, 2]] - P[idx[:, 0]]), axis=1)
    q = nn == 4
    a[q] += 0.5 * np.linalg.norm(np.cross(P[idx[q, 2]] - P[idx[q, 0]], P[idx[q, 3]] - P[idx[q, 0]]), axis=1)
    return a


# ----------------------------------------------------------------------------- solver
class B200Solver:
    """The GPU solver object passed as ``solver=`` (the drop-in of
    src/FLOWPanel_linearsolver.jl:24-157's solvers, owning assembly too).

    method: "ludiv" | "backslash" (LU, same on the device) | "gmres"
    precision: "fp64" (plain) | "mixed" (FP32 factors with a static row order
        + FP64 refinement) | "mixed_gepp" (FP32 factors pivoted as the FP64
        form + FP64 refinement) | "bf16" (BF16 tensor-core operands, GMRES-IR
        with FP64 residuals; the largest meshes)
    autotune: before the first LU solve of each problem size, time the
        factorisation's knob settings on the assembled AIC (fp_autotune) and
        keep the fastest for this solver
    """

    def __init__(self, method="ludiv", precision="fp64", device=0, ir_tol=1e-12, ir_maxiter=10,
                 gmres_memory=50, atol=None, rtol=None, itmax=0, autotune=False):
        if method not in ("ludiv", "backslash", "gmres"):
            raise ValueError(f"unknown method {method}")
        if precision not in ("fp64", "mixed", "mixed_gepp", "bf16"):
            raise ValueError(f"unknown precision {precision}")
        self.method, self.precision = method, precision
        self.opts = _capi.make_opts("gmres" if method == "gmres" else "ludiv", precision, ir_tol, ir_maxiter,
                                    gmres_memory, -1.0 if atol is None else atol,
                                    -1.0 if rtol is None else rtol, itmax)
        self.ctx = _capi.Context(device)
        self.stats = None
        self._geom_of = None
        self.autotune = autotune
        self.tuned = {}   # (N, precision) -> knob values chosen by fp_autotune

    def load(self, body: AbstractBody, normals=None, CPs=None):
        m = body.mesh
        if normals is None:
            normals = calc_normals(body)
        if CPs is None:
            CPs = calc_controlpoints(body, normals)
        self.ctx.set_geometry(m.nodes, m.panel_offsets, m.panel_nodes, CPs, normals)
        self._geom_of = id(body)

    def close(self):
        self.ctx.close()


def solve(body: AbstractBody, Uinfs, Das=None, Dbs=None, solver: Optional[B200Solver] = None,
          elprescribe=None):
    """solve(body, Uinfs[, Das, Dbs]; solver): assemble, factor and solve on the
    GPU, then store the strengths and the fields like the reference. A
    source+doublet NonLiftingBody follows its reference method
    (src/FLOWPanel_nonliftingbody.jl:425-600): sigma = -Uinf . n and
    mu = the potential of the sources of strength -sigma at the control points;
    like the reference it returns mu and stores nothing. A watertight
    vortex-ring body (or a MultiBody with watertight members, or any
    ``elprescribe`` given: [(0-based index, value), ...]) is solved by least
    squares (fp_solve_ls, src/FLOWPanel_liftingbody.jl:236-447)."""
    Uinfs = np.asarray(Uinfs, dtype=np.float64)
    if Uinfs.shape != (body.ncells, 3):
        raise ValueError(f"Invalid Uinfs; expected size ({body.ncells}, 3), got {Uinfs.shape}")
    if body.kind == "source+doublet":
        normals = calc_normals(body)
        CPs = calc_controlpoints(body, normals)
        sigma = -np.einsum("ij,ij->i", normals, Uinfs)
        solver = solver or B200Solver()
        solver.load(body, normals, CPs)
        return solver.ctx.phi(_capi.FP_ELEMENT_SOURCE, -sigma, CPs, None, body.kerneloffset)
    lifting = body.kind == "vortexring"
    if lifting:
        if Das is None or Dbs is None:
            raise ValueError("lifting bodies need Das and Dbs")
        Das, Dbs = np.asarray(Das, float), np.asarray(Dbs, float)
        if Das.shape != (body.nsheddings, 3):
            raise ValueError(f"Invalid Das; expected size ({body.nsheddings}, 3), got {Das.shape}")
        if Dbs.shape != (body.nsheddings, 3):
            raise ValueError(f"Invalid Dbs; expected size ({body.nsheddings}, 3), got {Dbs.shape}")
    solver = solver or B200Solver()
    solver.load(body)
    if lifting and body.nsheddings:
        solver.ctx.set_wake(body.mesh.shedding, Das, Dbs)
    elif lifting:
        solver.ctx.set_wake(np.zeros((0, 6), np.int32), np.zeros((0, 3)), np.zeros((0, 3)))
    ls = lifting and (elprescribe is not None or getattr(body, "watertight", False) or
                      (isinstance(body, MultiBody) and any(getattr(b, "watertight", False) for b in body.bodies)))
    if ls:
        pres = calc_elprescribe(body) if elprescribe is None else list(elprescribe)
        x, st = solver.ctx.solve_ls(Uinfs, pres, body.kerneloffset, body.kernelcutoff)
    else:
        if solver.autotune and solver.method != "gmres" and solver.precision in ("fp64", "mixed", "bf16"):
            key = (body.ncells, solver.precision)
            if key not in solver.tuned:
                prec = {"fp64": _capi.FP_PREC_FP64, "mixed": _capi.FP_PREC_MIXED, "bf16": _capi.FP_PREC_BF16}
                solver.ctx.assemble(body.element, body.kerneloffset, body.kernelcutoff,
                                    _capi.FP_PREC_MIXED if solver.precision == "mixed" else _capi.FP_PREC_FP64)
                solver.tuned[key] = solver.ctx.autotune(prec[solver.precision])
        x, st = solver.ctx.solve_body(body.element, Uinfs, body.kerneloffset, body.kernelcutoff, solver.opts)
    solver.stats = st.asdict()
    body.strength = np.array(x, dtype=np.float64)
    body.solved = True
    body.add_field("Uinf", "vector", Uinfs, "cell")
    if lifting:
        body.add_field("Da", "vector", Das, "system")
        body.add_field("Db", "vector", Dbs, "system")
        body.add_field("Gamma", "scalar", body.strength, "cell")
    elif body.kind == "doublet":
        body.add_field("mu", "scalar", body.strength, "cell")
    else:
        body.add_field("sigma", "scalar", body.strength, "cell")
    body._solver = solver
    return body


def solve_batch(bodies: List[AbstractBody], Uinfs, Das=None, Dbs=None, method="ludiv", precision="mixed",
                device=0, nslots=4, batch=None):
    """Solve many bodies of one element type concurrently on one device
    (fp_batch_solve: nslots device contexts, largest bodies first). Each
    body's strengths and fields are stored as ``solve`` stores them, and each
    equals the result of solving that body alone. Uinfs, Das, Dbs are lists
    with one entry per body. Returns the per-body statistics."""
    if not bodies:
        return []
    kinds = {b.kind for b in bodies}
    if len(kinds) != 1:
        raise ValueError("solve_batch: all bodies must use the same element type")
    lifting = bodies[0].kind == "vortexring"
    problems = []
    for i, b in enumerate(bodies):
        U = np.asarray(Uinfs[i], dtype=np.float64)
        if U.shape != (b.ncells, 3):
            raise ValueError(f"Invalid Uinfs of body {i}; expected size ({b.ncells}, 3), got {U.shape}")
        p = dict(nodes=b.mesh.nodes, panel_offsets=b.mesh.panel_offsets, panel_nodes=b.mesh.panel_nodes, Uinfs=U)
        if isinstance(b, MultiBody) or b.CPoffset != 1e-14 or b.characteristiclength is not None:
            normals = calc_normals(b)
            p.update(normals=normals, cps=calc_controlpoints(b, normals))
        # else: the library's worker threads form them (the default offset 1e-14, l = 1)
        if lifting:
            p.update(shedding=b.mesh.shedding, Das=np.asarray(Das[i], float), Dbs=np.asarray(Dbs[i], float))
        problems.append(p)
    opts = _capi.make_opts("gmres" if method == "gmres" else "ludiv", precision)
    own = batch is None
    batch = batch or _capi.Batch(device, nslots)
    try:
        xs, stats = batch.solve(bodies[0].element, problems, bodies[0].kerneloffset, bodies[0].kernelcutoff, opts)
    finally:
        if own:
            batch.close()
    for i, (b, x) in enumerate(zip(bodies, xs)):
        b.strength = x
        b.solved = True
        b.add_field("Uinf", "vector", problems[i]["Uinfs"], "cell")
        if lifting:
            b.add_field("Da", "vector", problems[i]["Das"], "system")
            b.add_field("Db", "vector", problems[i]["Dbs"], "system")
            b.add_field("Gamma", "scalar", x, "cell")
        else:
            b.add_field("sigma", "scalar", x, "cell")
    return stats


def _field_solver(body: AbstractBody, solver: Optional[B200Solver]):
    """A solver whose context holds the body's geometry (and wake)."""
    solver = solver or getattr(body, "_solver", None) or B200Solver()
    if solver._geom_of != id(body):
        solver.load(body)
        if body.kind == "vortexring" and body.nsheddings:
            Da = body.get_field("Da")["field_data"]
            Db = body.get_field("Db")["field_data"]
            solver.ctx.set_wake(body.mesh.shedding, Da, Db)
    return solver


def Uind(body: AbstractBody, targets, out, solver: Optional[B200Solver] = None, precision="fp64"):
    """Uind!: add the velocity induced by the solved body at targets (M, 3) to out
    (src/FLOWPanel_abstractbody.jl:101-110)."""
    if not body.solved:
        raise RuntimeError("Source body hasn't been solved yet. Please call `solve(...)` function first.")
    solver = _field_solver(body, solver)
    prec = _capi.FP_PREC_FP64 if precision == "fp64" else _capi.FP_PREC_MIXED
    return solver.ctx.uind(body.element, body.strength, targets, out, prec,
                           body.kerneloffset, body.kernelcutoff)


def phi(body: AbstractBody, targets, out, solver: Optional[B200Solver] = None):
    """phi!: add the potential induced by the solved body at targets (M, 3) to
    out (M,) (src/FLOWPanel_abstractbody.jl:118-127): sources, doublets, both,
    or vortex rings with the wake's semi-infinite doublets."""
    if not body.solved:
        raise RuntimeError("Body hasn't been solved yet. Please call `solve()` function first.")
    solver = _field_solver(body, solver)
    return solver.ctx.phi(body.element, body.strength, targets, out, body.kerneloffset)


def calcfield_U(sourcebody: AbstractBody, targetbody: AbstractBody, offset=None,
                characteristiclength=None, fieldname="U", addfield=True, solver=None):
    """calcfield_U: freestream + induced velocity at the (offset) control points
    of targetbody (src/FLOWPanel_postprocess.jl:28-110)."""
    if not sourcebody.solved:
        raise RuntimeError("Source body hasn't been solved yet. Please call `solve(...)` function first.")
    if not targetbody.check_field("Uinf"):
        raise RuntimeError("Target body doesn't have freestream field `\"Uinf\"`.")
    Uinfs = np.asarray(targetbody.get_field("Uinf")["field_data"], float)
    normals = calc_normals(targetbody)
    cps = calc_controlpoints(targetbody, normals, off=offset, characteristiclength=characteristiclength) \
        if offset is not None else calc_controlpoints(targetbody, normals)
    out = np.array(Uinfs, dtype=np.float64, copy=True)
    out = Uind(sourcebody, cps, out, solver)
    if addfield:
        targetbody.add_field(fieldname, "vector", out, "cell")
    return out


def _cpoffset_cells(body: AbstractBody):
    """CPoffset of every panel (each member's own for a MultiBody)."""
    if isinstance(body, MultiBody):
        return body._default_off()
    return np.full(body.ncells, float(body.CPoffset))


def _doublet_strength(body: AbstractBody, Gammai=0):
    if not body.solved:
        raise RuntimeError("Body hasn't been solved yet. Please call `solve()` function first.")
    s = np.asarray(body.strength, float)
    if s.ndim == 2:
        return np.ascontiguousarray(s[:, Gammai if body.kind != "source+doublet" else 1])
    return s


def calcfield_Ugradmu(body: AbstractBody, sharpTE=False, force_cellTE=True, anglecrit=30.0, Gammai=0,
                      fieldname="Ugradmu", addfield=True, solver: Optional[B200Solver] = None, want_parts=False):
    """calcfield_Ugradmu: surface velocity -1/2 grad(mu) of a solved body with
    triangular panels, the cell scheme except where a cell has a free edge or
    a neighbour more than ``anglecrit`` degrees off, which take the node scheme
    (src/FLOWPanel_postprocess.jl:825-1042), on the device (fp_ugradmu_ex).
    Returns (N, 3); with ``want_parts`` also the cell and node fields.
    ``sharpTE``: the node scheme's trailing-edge cells take one-sided nodal
    values at the trailing-edge nodes (see calcfield_Ugradmu_node)."""
    g = _doublet_strength(body, Gammai)
    solver = _field_solver(body, solver)
    out, oc, on = solver.ctx.ugradmu(_capi.FP_UGRADMU_COMBINED, g, _cpoffset_cells(body), anglecrit, force_cellTE,
                                     want_parts=True, sharpTE=sharpTE)
    if addfield:
        body.add_field(fieldname, "vector", out, "cell")
    return (out, oc, on) if want_parts else out


def smooth_rows_cells(smoothRows, ndivscells):
    """The cells that smoothRows names, in the order the smoothing visits them
    (src/FLOWPanel_postprocess.jl:500-503: ``for i in smoothRows, j in
    1:NDIVS[2]``, cell ``linc[i, j]``): ``ndivscells`` = (n1, n2), the cell
    grid of the triangulated loft (n1 along its first, split dimension),
    column-major; rows are 1-based as in the reference, 0 meaning none."""
    n1, n2 = (int(v) for v in ndivscells)
    rows = [int(i) for i in np.atleast_1d(smoothRows)]
    if not rows or rows[0] == 0:
        return np.zeros(0, np.int32)
    if any(i < 1 or i > n1 for i in rows):
        raise ValueError(f"smoothRows must lie in 1..{n1}")
    return np.asarray([(i - 1) + n1 * j for i in rows for j in range(n2)], np.int32)


def calcfield_Ugradmu_cell(body: AbstractBody, Gammai=0, maxgrad=np.inf, fieldname="Ugradmu", addfield=True,
                           solver: Optional[B200Solver] = None, smoothPass=0, smoothRows=(0,), ndivscells=None,
                           smooth_cells=None):
    """calcfield_Ugradmu_cell (src/FLOWPanel_postprocess.jl:139-616): Green-Gauss
    gradient with the inverse-distance face value; the trailing-edge cells'
    face terms are added back; with ``smoothPass`` > 0 the cells of
    ``smoothRows`` (placed on the loft's cell grid ``ndivscells``, see
    smooth_rows_cells) or an explicit ``smooth_cells`` list are smoothed
    (:499-526); then rows whose norm reaches ``maxgrad`` are zeroed."""
    g = _doublet_strength(body, Gammai)
    solver = _field_solver(body, solver)
    if smooth_cells is None and smoothPass and np.atleast_1d(smoothRows)[0] != 0:
        if ndivscells is None:
            raise ValueError("smoothRows needs the loft's cell grid: pass ndivscells=(n1, n2) or smooth_cells")
        smooth_cells = smooth_rows_cells(smoothRows, ndivscells)
    out = solver.ctx.ugradmu(_capi.FP_UGRADMU_CELL, g, _cpoffset_cells(body), maxgrad=maxgrad,
                             smooth_cells=smooth_cells, smooth_pass=int(smoothPass))
    if addfield:
        body.add_field(fieldname, "vector", out, "cell")
    return out


def calcfield_Ugradmu_node(body: AbstractBody, Gammai=0, sharpTE=False, fieldname="Ugradmu", addfield=True,
                           solver: Optional[B200Solver] = None):
    """calcfield_Ugradmu_node (src/FLOWPanel_postprocess.jl:622-819): -1/2 the
    linear gradient of the area-weighted nodal values. With ``sharpTE``
    (:698-742) the trailing-edge cells (each shedding row's upper cells pi,
    pi+1 and lower cells pj, pj-1: the last and first two loop cells of a
    loft, :705-708) take at the trailing-edge nodes (the upper edge's nodes)
    the area-weighted nodal value over their own side's cells only."""
    g = _doublet_strength(body, Gammai)
    solver = _field_solver(body, solver)
    out = solver.ctx.ugradmu(_capi.FP_UGRADMU_NODE, g, _cpoffset_cells(body), sharpTE=sharpTE)
    if addfield:
        body.add_field(fieldname, "vector", out, "cell")
    return out


def addfields(body: AbstractBody, sourcefieldname, targetfieldname):
    """addfields: add field ``sourcefieldname`` into ``targetfieldname``
    (src/FLOWPanel_abstractbody.jl addfields)."""
    src = np.asarray(body.get_field(sourcefieldname)["field_data"], float)
    tgt = body.get_field(targetfieldname)
    tgt["field_data"] = np.asarray(tgt["field_data"], float) + src
    return body


def calcfield_Cp(body: AbstractBody, Uref, U_fieldname="U", Us=None, correct_kuttacondition=True,
                 clip=None, fieldname="Cp", addfield=True, solver: Optional[B200Solver] = None):
    """calcfield_Cp!: Cp = 1 - (|U|/Uref)^2, Kutta average over (pi, pi+1, pj, pj-1)
    of each shedding row in order (src/FLOWPanel_postprocess.jl:1059-1112), on
    the device (fp_calcfield_cp); ``clip`` is applied afterwards on the host."""
    if Us is None:
        if not body.check_field(U_fieldname):
            raise RuntimeError(f"Field {U_fieldname} not found; Please run "
                               f"`calcfield_U(args...; fieldname={U_fieldname}, optargs...)`")
        Us = body.get_field(U_fieldname)["field_data"]
    Us = np.asarray(Us, float)
    solver = _field_solver(body, solver)
    Cp = solver.ctx.calcfield_cp(Us, Uref, correct_kuttacondition and body.kind == "vortexring")
    if clip is not None:
        Cp = np.array([clip(v) for v in Cp])
    if addfield:
        body.add_field(fieldname, "scalar", Cp, "cell")
    return Cp


def calcfield_F(body: AbstractBody, Uinf, rho, Cp_fieldname="Cp", correct_kuttacondition=True,
                fieldname="F", addfield=True, solver: Optional[B200Solver] = None):
    """calcfield_F!: F = -Cp (rho Uinf^2 / 2) A n with normals flipped by
    sign(CPoffset) and the TE override (src/FLOWPanel_postprocess.jl:1199-1392),
    on the device (fp_calcfield_f)."""
    if not body.check_field(Cp_fieldname):
        raise RuntimeError(f"Field {Cp_fieldname} not found; Please run "
                           f"`calcfield_Cp(args...; fieldname={Cp_fieldname}, optargs...)`")
    Cps = np.asarray(body.get_field(Cp_fieldname)["field_data"], float)
    solver = _field_solver(body, solver)
    F = solver.ctx.calcfield_f(Cps, Uinf, rho, _cpoffset_cells(body),
                               correct_kuttacondition and body.kind == "vortexring")
    if addfield:
        body.add_field(fieldname, "vector", F, "cell")
    return F


def calcfield_LDS(body: AbstractBody, Lhat, Dhat, Shat=None, F_fieldname="F", addfield=True,
                  solver: Optional[B200Solver] = None):
    """calcfield_LDS!: lift, drag and sideslip vectors (columns) from the summed
    force (src/FLOWPanel_postprocess.jl:1615-1689), on the device
    (fp_calcfield_lds)."""
    Lhat, Dhat = np.asarray(Lhat, float), np.asarray(Dhat, float)
    Shat = np.cross(Lhat, Dhat) if Shat is None else np.asarray(Shat, float)
    for v, nm in ((Lhat, "Lhat"), (Dhat, "Dhat"), (Shat, "Shat")):
        if abs(np.linalg.norm(v) - 1) > 2 * np.finfo(float).eps:
            raise ValueError(f"{nm}={v} is not a unitary vector")
    if not body.check_field(F_fieldname):
        raise RuntimeError(f"Field {F_fieldname} not found; Please run "
                           f"`calcfield_F(args...; fieldname={F_fieldname}, optargs...)`")
    Fs = np.asarray(body.get_field(F_fieldname)["field_data"], float)
    solver = _field_solver(body, solver)
    out = solver.ctx.calcfield_lds(Fs, Lhat, Dhat, Shat)
    if addfield:
        body.add_field("L", "vector", out[:, 0], "system")
        body.add_field("D", "vector", out[:, 1], "system")
        body.add_field("S", "vector", out[:, 2], "system")
    return out


def surface_loads(body: AbstractBody, magVinf, rho, Lhat, Dhat, Shat=None, ugradmu=None,
                  correct_kuttacondition=True, solver: Optional[B200Solver] = None, addfield=True):
    """The post-processing sequence of the reference's examples in one pass on
    the device (examples/sweptwing_solverbenchmark.jl:14-66): calcfield_U at the
    control points, + calcfield_Ugradmu (when ``ugradmu``), calcfield_Cp with
    Uref = magVinf, calcfield_F with Uinf = magVinf and rho, calcfield_LDS.
    Returns the 3 x 3 L/D/S matrix and stores the U, Cp, F, L, D, S fields.
    ``ugradmu`` defaults to True for bodies with doublet strengths (vortex
    rings, doublets) and False for source bodies, which have none."""
    if ugradmu is None:
        ugradmu = body.kind != "source"
    if not body.solved:
        raise RuntimeError("Body hasn't been solved yet. Please call `solve()` function first.")
    Lhat, Dhat = np.asarray(Lhat, float), np.asarray(Dhat, float)
    Shat = np.cross(Lhat, Dhat) if Shat is None else np.asarray(Shat, float)
    Uinfs = np.asarray(body.get_field("Uinf")["field_data"], float)
    solver = _field_solver(body, solver)
    U, Cp, F, LDS = solver.ctx.surface_loads(body.element, body.strength, Uinfs, magVinf, rho, Lhat, Dhat, Shat,
                                             _cpoffset_cells(body), body.kerneloffset, body.kernelcutoff,
                                             ugradmu, correct_kuttacondition and body.kind == "vortexring")
    if addfield:
        body.add_field("U", "vector", U, "cell")
        body.add_field("Cp", "scalar", Cp, "cell")
        body.add_field("F", "vector", F, "cell")
        body.add_field("L", "vector", LDS[:, 0], "system")
        body.add_field("D", "vector", LDS[:, 1], "system")
        body.add_field("S", "vector", LDS[:, 2], "system")
    return LDS
