"""Synthetic panel meshes for the benchmark and test workloads.

Meshing stays on the host in FLOWPanel.jl (GeometricTools lofts and
revolutions, src/FLOWPanel_abstractliftingbody.jl:73-176,
src/FLOWPanel_utils.jl:68-150). These generators produce the same kind of
structured surface meshes directly, in the flat layout the C ABI takes:

* ``nodes``          (nnodes, 3) float64  == Julia's 3 x nnodes column-major;
* ``panel_offsets``  (npanels+1,) int32, ``panel_nodes`` int32, 0-based (CSR);
* ``shedding``       (nsh, 6) int32 rows (pi, nia, nib, pj, nja, njb), 0-based,
  nia/nib/nja/njb local to the panel, pj == -1 for no lower side
  (the 6 x nsh matrix of src/FLOWPanel_liftingbody.jl:24-31).

Panel node order makes ``(p2-p1) x (p3-p1)`` point out of the body, so every
body here uses a positive ``CPoffset``. Wing contours run from the upper
trailing edge over the leading edge to the lower trailing edge, chordwise index
fastest, so the reference's Kutta average over (pi, pi+1, pj, pj-1)
(src/FLOWPanel_postprocess.jl:1075-1097) averages the two panels on each side
of the trailing edge.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List

import numpy as np


@dataclass
class Body:
    name: str
    kind: str            # "source" | "vortexring"
    ncells: int
    nsheddings: int
    CPoffset: float = 1e-14
    kerneloffset: float = 1e-8
    kernelcutoff: float = 1e-14


@dataclass
class Mesh:
    nodes: np.ndarray
    panel_offsets: np.ndarray
    panel_nodes: np.ndarray
    shedding: np.ndarray = field(default_factory=lambda: np.zeros((0, 6), np.int32))
    bodies: List[Body] = field(default_factory=list)

    @property
    def npanels(self) -> int:
        return len(self.panel_offsets) - 1

    @property
    def nnodes(self) -> int:
        return self.nodes.shape[0]

    @property
    def nsheddings(self) -> int:
        return int(self.shedding.shape[0])

    def panel(self, i):
        return self.panel_nodes[self.panel_offsets[i]:self.panel_offsets[i + 1]]

    def cpoffset_sign(self):
        """Per-panel sign(CPoffset) (MultiBody rule, src/FLOWPanel_multibody.jl:664-676)."""
        s = np.empty(self.npanels)
        k = 0
        for b in self.bodies:
            s[k:k + b.ncells] = np.sign(b.CPoffset) if b.CPoffset != 0 else 1.0
            k += b.ncells
        return s

    def cpoffset(self):
        s = np.empty(self.npanels)
        k = 0
        for b in self.bodies:
            s[k:k + b.ncells] = b.CPoffset
            k += b.ncells
        return s


def concat(meshes: List[Mesh]) -> Mesh:
    """MultiBody: concatenate bodies; G's column blocks follow body order
    (src/FLOWPanel_multibody.jl:502-530)."""
    nodes, offs, pn, sh, bodies = [], [0], [], [], []
    noff, poff = 0, 0
    for m in meshes:
        nodes.append(m.nodes)
        pn.append(m.panel_nodes + noff)
        offs.extend((m.panel_offsets[1:] + offs[-1]).tolist())
        s = m.shedding.copy()
        if len(s):
            s[:, 0] += poff
            s[:, 3] = np.where(s[:, 3] >= 0, s[:, 3] + poff, -1)
        sh.append(s)
        bodies.extend(m.bodies)
        noff += m.nnodes
        poff += m.npanels
    return Mesh(np.concatenate(nodes), np.asarray(offs, np.int32), np.concatenate(pn).astype(np.int32),
                np.concatenate(sh).astype(np.int32) if sh else np.zeros((0, 6), np.int32), bodies)


def _quad_grid(P, drop_degenerate=True, tol=1e-14):
    """Quads of a structured (ni+1) x (nj+1) node grid P[i, j] (contour i, span j).
    Panel (i, j) = [n(i,j), n(i,j+1), n(i+1,j+1), n(i+1,j)]; coincident
    consecutive nodes (poles) are dropped so that such panels become triangles."""
    ni, nj = P.shape[0] - 1, P.shape[1] - 1
    nodes = P.reshape(-1, 3)
    idx = np.arange((ni + 1) * (nj + 1)).reshape(ni + 1, nj + 1)
    offs, pn = [0], []
    for j in range(nj):
        for i in range(ni):
            q = [idx[i, j], idx[i, j + 1], idx[i + 1, j + 1], idx[i + 1, j]]
            if drop_degenerate:
                keep = []
                for k in range(4):
                    a, b = q[k], q[(k + 1) % 4]
                    if np.linalg.norm(nodes[a] - nodes[b]) > tol:
                        keep.append(a)
                q = keep
            pn.extend(q)
            offs.append(len(pn))
    return nodes.copy(), np.asarray(offs, np.int32), np.asarray(pn, np.int32)


# ------------------------------------------------------------------ sphere
def sphere(R=1.0, ntheta=30, nphi=60, CPoffset=1e-14):
    """Body of revolution: sphere of radius R centred at the origin, polar axis z;
    ntheta polar x nphi azimuthal cells (pole rows are triangles). Constant-source
    body as in examples/sphere.jl."""
    th = np.linspace(0.0, np.pi, ntheta + 1)
    ph = np.linspace(0.0, 2 * np.pi, nphi + 1)
    T, PH = np.meshgrid(th, ph, indexing="ij")
    P = np.stack([R * np.sin(T) * np.cos(PH), R * np.sin(T) * np.sin(PH), R * np.cos(T)], axis=-1)
    P[0, :] = [0, 0, R]
    P[-1, :] = [0, 0, -R]
    P[:, -1] = P[:, 0]
    # contour i along theta, "span" j along phi: (p2-p1) x (p3-p1) ~ e_phi x e_theta = -e_r,
    # so reverse phi to point outwards.
    P = P[:, ::-1].copy()
    nodes, offs, pn = _quad_grid(P)
    m = Mesh(nodes, offs, pn)
    m.bodies = [Body("sphere", "source", m.npanels, 0, CPoffset)]
    return m


def triangulate(m: Mesh) -> Mesh:
    """Split every quad into two triangles along its first diagonal (the
    reference always meshes structured grids as triangles,
    src/FLOWPanel_nonliftingbody.jl:834,855). Shedding rows are re-mapped to
    the triangle that keeps the trailing-edge edge."""
    offs, pn, newidx = [0], [], []
    for i in range(m.npanels):
        p = list(m.panel(i))
        if len(p) == 4:
            newidx.append(len(offs) - 1)
            pn.extend([p[0], p[1], p[2]]); offs.append(len(pn))
            pn.extend([p[0], p[2], p[3]]); offs.append(len(pn))
        else:
            newidx.append(len(offs) - 1)
            pn.extend(p); offs.append(len(pn))
    sh = []
    for (pi, nia, nib, pj, nja, njb) in m.shedding:
        def remap(pp, a, b):
            p = list(m.panel(pp))
            ga, gb = p[a], p[b]
            base = newidx[pp]
            for t in (base, base + 1):
                tri = pn[offs[t]:offs[t + 1]]
                if ga in tri and gb in tri:
                    return t, tri.index(ga), tri.index(gb)
            raise ValueError("edge lost in triangulation")
        ti, ta, tb = remap(pi, nia, nib)
        if pj >= 0:
            tj, tc, td = remap(pj, nja, njb)
        else:
            tj, tc, td = -1, 0, 0
        sh.append((ti, ta, tb, tj, tc, td))
    out = Mesh(m.nodes.copy(), np.asarray(offs, np.int32), np.asarray(pn, np.int32),
               np.asarray(sh, np.int32).reshape(-1, 6))
    out.bodies = [Body(b.name, b.kind, 0, b.nsheddings, b.CPoffset, b.kerneloffset, b.kernelcutoff)
                  for b in m.bodies]
    # recount cells per body
    k = 0
    for b, ob in zip(out.bodies, m.bodies):
        b.ncells = sum(2 if len(m.panel(i)) == 4 else 1 for i in range(k, k + ob.ncells))
        k += ob.ncells
    return out


# ------------------------------------------------------------------ airfoils and wings
def naca4_contour(code="0012", n_half=50, closed_te=True):
    """NACA 4-digit section with cosine spacing, as a closed contour from the
    upper trailing edge over the leading edge to the lower trailing edge;
    returns (2*n_half+1, 2) points (x, z) on a unit chord."""
    m = int(code[0]) / 100.0
    p = int(code[1]) / 10.0
    t = int(code[2:]) / 100.0
    k = np.arange(n_half + 1)
    x = 0.5 * (1 - np.cos(np.pi * k / n_half))          # LE -> TE
    a4 = -0.1036 if closed_te else -0.1015
    yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 + a4 * x ** 4)
    if m > 0:
        yc = np.where(x < p, m / p ** 2 * (2 * p * x - x ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x - x ** 2))
        dyc = np.where(x < p, 2 * m / p ** 2 * (p - x), 2 * m / (1 - p) ** 2 * (p - x))
    else:
        yc = np.zeros_like(x)
        dyc = np.zeros_like(x)
    th = np.arctan(dyc)
    xu, zu = x - yt * np.sin(th), yc + yt * np.cos(th)
    xl, zl = x + yt * np.sin(th), yc - yt * np.cos(th)
    if closed_te:
        zu[-1] = zl[-1] = yc[-1]
        xu[-1] = xl[-1] = 1.0
    upper = np.stack([xu[::-1], zu[::-1]], axis=1)       # TE -> LE
    lower = np.stack([xl[1:], zl[1:]], axis=1)           # LE(excl) -> TE
    return np.concatenate([upper, lower])


def wing_half(contour, y0, y1, nspan, chord0, chord1, xle0, xle1, twist0=0.0, twist1=0.0,
              zle0=0.0, zle1=0.0, name="wing", CPoffset=1e-14):
    """Loft one wing panel between spanwise stations y0 < y1 (linear
    interpolation of chord, leading-edge position and twist about the quarter
    chord). Returns a lifting Mesh with one shedding edge per spanwise strip."""
    nc = contour.shape[0] - 1
    ys = np.linspace(y0, y1, nspan + 1)
    s = (ys - y0) / (y1 - y0)
    P = np.zeros((nc + 1, nspan + 1, 3))
    for j, sj in enumerate(s):
        c = chord0 + (chord1 - chord0) * sj
        xle = xle0 + (xle1 - xle0) * sj
        zle = zle0 + (zle1 - zle0) * sj
        tw = np.deg2rad(twist0 + (twist1 - twist0) * sj)
        xc = (contour[:, 0] - 0.25) * c
        zc = contour[:, 1] * c
        xr = xc * np.cos(tw) + zc * np.sin(tw)
        zr = -xc * np.sin(tw) + zc * np.cos(tw)
        P[:, j, 0] = xle + 0.25 * c + xr
        P[:, j, 1] = ys[j]
        P[:, j, 2] = zle + zr
    nodes, offs, pn = _quad_grid(P, drop_degenerate=False)
    sh = np.zeros((nspan, 6), np.int32)
    for j in range(nspan):
        sh[j] = (j * nc + 0, 1, 0, j * nc + nc - 1, 3, 2)
    m = Mesh(nodes, offs, pn, sh)
    m.bodies = [Body(name, "vortexring", m.npanels, nspan, CPoffset)]
    return m


def discretize_ndivs(NDIVS, length=1.0):
    """Node positions 0..length of the NDIVS sections [(fraction, ncells,
    expansion, central), ...] of GeometricTools' discretisation, as
    simplewing's ``span_NDIVS`` and ``rfl_NDIVS`` give them
    (src/FLOWPanel_utils.jl:110-125): each section covers ``fraction`` of the
    length with ``ncells`` cells whose lengths grow linearly from the first to
    the last by the factor ``expansion`` (the lofted swept wing of
    examples/sweptwing.jl pins this: 15 cells at expansion 10 grow by equal
    steps from 1 to 10); ``central`` mirrors the growth about the section's
    middle (cells grow from both ends towards it by ``expansion``)."""
    pts = [0.0]
    x0 = 0.0
    tot = sum(float(f) for f, *_ in NDIVS)
    for frac, n, r, central in NDIVS:
        L = length * float(frac) / tot
        n = int(n)
        if central and n > 1:
            h = n // 2
            w = _ramp(h, r) if h > 0 else np.zeros(0)
            mid = [1.0 * r] if n % 2 else []
            w = np.concatenate([w, mid, w[::-1]])
        else:
            w = _ramp(n, r)
        w = w / w.sum() * L
        pts.extend((x0 + np.cumsum(w)).tolist())
        x0 += L
    out = np.asarray(pts)
    out[-1] = length
    return out


def _ramp(n, r):
    """n cell weights growing linearly from 1 to r."""
    if n == 1:
        return np.ones(1)
    return 1.0 + (float(r) - 1.0) * np.arange(n) / (n - 1)


def rediscretize_airfoil(x, y, NDIVS_up, NDIVS_lo, spline_k=5, spline_s=1e-8, nsamples=100_000):
    """Re-discretise an airfoil contour (GeometricTools' rediscretize_airfoil,
    as simplewing calls it with rflspl_s, src/FLOWPanel_utils.jl:76-147):
    the contour, from the trailing edge over one surface to the leading edge
    (the point of least x) and back over the other, is split there; each
    surface is splined as y(x) with the smoothing spline of FITPACK (curfit,
    order ``spline_k``, smoothing ``spline_s``: the library both
    GeometricTools' Dierckx and scipy's UnivariateSpline wrap) and
    re-discretised by arc length from the leading edge with the NDIVS
    sections (discretize_ndivs), the arc length measured on ``nsamples``
    chords of the curve. Returns (K, 2): the trailing edge (from the second
    surface's spline), the second surface from the trailing edge to before
    the leading edge, the leading edge (first surface), then the first
    surface up to before the trailing edge -- the closed loop of the
    reference's lofted sections. With the reference's RAE 101 file and
    rfl_NDIVS this reproduces the section of its lofted swept-wing mesh to
    1e-9 of the chord."""
    from scipy.interpolate import UnivariateSpline

    x = np.asarray(x, float)
    y = np.asarray(y, float)
    ile = int(np.argmin(x))
    first = np.stack([x[:ile + 1][::-1], y[:ile + 1][::-1]], axis=1)    # LE -> TE
    second = np.stack([x[ile:], y[ile:]], axis=1)                        # LE -> TE

    def surface(pts, NDIVS):
        sp = UnivariateSpline(pts[:, 0], pts[:, 1], k=spline_k, s=spline_s)
        xs = np.linspace(pts[0, 0], pts[-1, 0], nsamples + 1)
        ys = sp(xs)
        L = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(xs), np.diff(ys)))])
        xn = np.interp(discretize_ndivs(NDIVS) * L[-1], L, xs)
        return np.stack([xn, sp(xn)], axis=1)

    a = surface(first, NDIVS_up)
    b = surface(second, NDIVS_lo)
    return np.concatenate([b[::-1][:-1], a[:-1]])


def revolution_liftbody(profile, NDIVS_theta, name="body", CPoffset=0.0, kind="vortexring"):
    """Lifting body of revolution about the x axis (generate_revolution_liftbody,
    src/FLOWPanel_abstractliftingbody.jl:124-176): ``profile`` (K, 2) is the
    closed contour (x axial, r radial; first point = last point, kept as two
    nodes: the grid loops in the azimuth only), revolved over NDIVS_theta
    equal azimuthal steps (the reference's start angle, 270 deg, is a
    multiple of the step for any NDIVS_theta dividing 360 into whole degrees
    of that kind, and only permutes the stations). Nodes station-major, K per
    station; triangles per strip and profile edge k as in simplewing, (a, b,
    c) and (c, d, a) with a = (j, k), b = (j, k+1), c = (j+1, k+1),
    d = (j+1, k), the azimuth running so that the normals point away from the
    contour's interior (into the flow). Shedding rows as the reference sets
    them for a closed contour: per strip, pi = the first triangle of the
    last profile quad, pj = the second triangle of the first, local nodes
    (3, 2) of each (1-based)."""
    P = np.asarray(profile, float)
    K = P.shape[0]
    nq = K - 1
    th = 2 * np.pi * np.arange(NDIVS_theta) / NDIVS_theta

    def build(sign):
        t = sign * th
        nodes = np.zeros((NDIVS_theta, K, 3))
        nodes[:, :, 0] = P[None, :, 0]
        nodes[:, :, 1] = P[None, :, 1] * np.cos(t)[:, None]
        nodes[:, :, 2] = P[None, :, 1] * np.sin(t)[:, None]
        return nodes.reshape(-1, 3)

    def tris():
        pn = []
        for j in range(NDIVS_theta):
            j1 = (j + 1) % NDIVS_theta
            for k in range(nq):
                a_, b_, c_, d_ = j * K + k, j * K + k + 1, j1 * K + k + 1, j1 * K + k
                pn += [a_, b_, c_, c_, d_, a_]
        return np.asarray(pn, np.int32)

    pn = tris()
    nodes = build(1.0)
    # orientation: the normal of a triangle a quarter of the way round the
    # contour against the direction from the contour's centroid (at that
    # azimuth) to the triangle
    q = 3 * 2 * (nq // 4)
    tri = nodes[pn[q:q + 3]]
    nrm = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    cen = P[:-1].mean(axis=0)
    ref = np.array([cen[0], cen[1], 0.0])
    if np.dot(nrm, tri.mean(axis=0) - ref) < 0:
        nodes = build(-1.0)
    npan = len(pn) // 3
    sh = np.asarray([(2 * nq - 2 + 2 * nq * j, 2, 1, 1 + 2 * nq * j, 2, 1) for j in range(NDIVS_theta)], np.int32)
    m = Mesh(nodes, np.arange(0, 3 * npan + 1, 3, dtype=np.int32), pn, sh)
    m.bodies = [Body(name, kind, npan, len(sh), CPoffset)]
    return m


def simplewing(section, b, ar, tr=1.0, lambda_=0.0, gamma=0.0, span_NDIVS=((1.0, 35, 20.0, True),),
               b_low=-1.0, b_up=1.0, name="wing", CPoffset=0.0, kind="vortexring"):
    """The lofted wing of simplewing (src/FLOWPanel_utils.jl:68-150): tip chord
    b/ar, root chord (b/ar)/tr, leading edge swept by ``lambda_`` and raised
    by ``gamma`` (degrees), chord and leading edge linear in |semi-span
    position| s (s = 0 at the root, 1 at the tips), stations at s in
    [b_low, b_up] from ``span_NDIVS`` (discretize_ndivs, first cell at
    b_low), untwisted.

    ``section`` (K, 2) is the re-discretised airfoil on a unit chord as a
    closed loop of K distinct points, x/c and z/c, starting at the trailing
    edge along the lower surface (the layout of the reference's lofted
    meshes). Nodes: station-major, K per station; triangles: per span strip,
    per loop edge k, (a, b, c) and (c, d, a) with a = (j, k), b = (j, k+1),
    c = (j+1, k+1), d = (j+1, k) -- the split of the reference's triangulated
    loft (GridTriangleSurface with dimsplit = 1). Shedding rows as
    generate_loft_liftbody sets them (src/FLOWPanel_abstractliftingbody.jl:
    85-100): per span strip j, pi = the first triangle of the loop's last
    quad, pj = the second triangle of its first quad, local nodes (3, 2) of
    each (1-based), i.e. 0-based rows (2K-2 + 2Kj, 2, 1, 1 + 2Kj, 2, 1)."""
    sec = np.asarray(section, float)
    K = sec.shape[0]
    semispan = b / 2
    c_tip = b / ar
    c_root = c_tip / tr
    t = discretize_ndivs(span_NDIVS)
    s = b_low + (b_up - b_low) * t
    a = np.abs(s)
    chord = c_root + (c_tip - c_root) * a
    xle = a * semispan * np.tan(np.deg2rad(lambda_))
    zle = a * semispan * np.tan(np.deg2rad(gamma))
    nst = len(s)
    nodes = np.zeros((nst, K, 3))
    nodes[:, :, 0] = xle[:, None] + chord[:, None] * sec[None, :, 0]
    nodes[:, :, 1] = (s * semispan)[:, None]
    nodes[:, :, 2] = zle[:, None] + chord[:, None] * sec[None, :, 1]
    pn = []
    for j in range(nst - 1):
        for k in range(K):
            a_, b_ = j * K + k, j * K + (k + 1) % K
            c_, d_ = (j + 1) * K + (k + 1) % K, (j + 1) * K + k
            pn += [a_, b_, c_, c_, d_, a_]
    npan = len(pn) // 3
    sh = np.asarray([(2 * K - 2 + 2 * K * j, 2, 1, 1 + 2 * K * j, 2, 1) for j in range(nst - 1)], np.int32)
    m = Mesh(nodes.reshape(-1, 3), np.arange(0, 3 * npan + 1, 3, dtype=np.int32), np.asarray(pn, np.int32), sh)
    m.bodies = [Body(name, kind, npan, len(sh), CPoffset)]
    return m


def swept_wing(naca="0012", n_chord=100, n_span=120, chord=1.0, b=5.0, sweep=45.0, taper=1.0,
               twist_root=0.0, twist_tip=0.0):
    """Swept wing as a MultiBody of two halves lofted from the root outwards on
    each side (the practice of examples/sweptwing.jl:88-130). ``n_chord`` cells
    around the section, ``n_span`` cells over the whole span. Root chord
    ``chord``, tip chord ``chord*taper``, aspect ratio b/c_tip."""
    assert n_chord % 2 == 0 and n_span % 2 == 0
    cont = naca4_contour(naca, n_chord // 2)
    tl = np.tan(np.deg2rad(sweep))
    half = b / 2
    ct = chord * taper
    left = wing_half(cont, -half, 0.0, n_span // 2, ct, chord, half * tl, 0.0, twist_tip, twist_root, name="L")
    right = wing_half(cont, 0.0, half, n_span // 2, chord, ct, 0.0, half * tl, twist_root, twist_tip, name="R")
    return concat([left, right])


def random_wings(n=64, seed=0, pmin=2000, pmax=8000):
    """Batch of wings drawn from ``numpy.random.default_rng(seed)``: sweep U[0,45] deg,
    aspect ratio U[4,10], taper U[0.3,1], linear twist U[-4,0] deg at the tip,
    chordwise cells U{40..80} (even), spanwise U{50..100} (even); draws outside
    [pmin, pmax] panels are rejected. Draw order: sweep, AR, taper, twist, nc, ns."""
    rng = np.random.default_rng(seed)
    out, params = [], []
    while len(out) < n:
        sweep = rng.uniform(0, 45)
        ar = rng.uniform(4, 10)
        taper = rng.uniform(0.3, 1)
        twist = rng.uniform(-4, 0)
        nc = 2 * int(rng.integers(20, 41))
        ns = 2 * int(rng.integers(25, 51))
        if not (pmin <= nc * ns <= pmax):
            continue
        ct = 1.0 * taper
        b = ar * ct
        out.append(swept_wing("0012", nc, ns, 1.0, b, sweep, taper, 0.0, twist))
        params.append(dict(sweep=sweep, ar=ar, taper=taper, twist=twist, n_chord=nc, n_span=ns, b=b))
    return out, params


def prolate_ellipsoid(L=10.0, rmax=0.6, nx=120, ntheta=80, tail=0.9):
    """Fuselage: prolate ellipsoid along x with semi-axes (L/2, rmax, rmax),
    nx axial x ntheta circumferential cells, polar angle from the nose up to
    ``tail*pi``. The tail is left open: a closed vortex-ring surface makes the
    direct vortex-ring system singular (src/FLOWPanel_liftingbody.jl:86-91),
    an open base keeps it well posed. The nose row is triangles."""
    th = np.linspace(0.0, tail * np.pi, nx + 1)
    ph = np.linspace(0.0, 2 * np.pi, ntheta + 1)
    T, PH = np.meshgrid(th, ph, indexing="ij")
    a = L / 2
    P = np.stack([a * np.cos(T), rmax * np.sin(T) * np.cos(PH), rmax * np.sin(T) * np.sin(PH)], axis=-1)
    P[0, :] = [a, 0, 0]
    P[:, -1] = P[:, 0]
    nodes, offs, pn = _quad_grid(P)
    k = nx // 2                                   # a mid-body panel of the first strip
    p = nodes[pn[offs[k]:offs[k + 1]]]
    n = np.cross(p[1] - p[0], p[2] - p[0])
    c = p.mean(axis=0)
    if np.dot(n, c - np.array([c[0], 0.0, 0.0])) < 0:
        P = P[:, ::-1].copy()
        nodes, offs, pn = _quad_grid(P)
    m = Mesh(nodes, offs, pn)
    m.bodies = [Body("fuselage", "vortexring", m.npanels, 0)]
    return m


def wing_body(fuse_nx=120, fuse_nt=80, wing_nc=150, wing_ns=180, AR=8.0, taper=0.4,
              sweep=40.0, croot=1.5):
    """Wing-body: prolate ellipsoid fuselage (L=10 m, r=0.6 m) and a swept NACA 2412
    wing (AR = b^2/S with S = b (croot+ctip)/2) whose root sections sit inside
    the fuselage at y = +-0 (no intersection meshing)."""
    fuse = prolate_ellipsoid(10.0, 0.6, fuse_nx, fuse_nt)
    ct = croot * taper
    b = AR * (croot + ct) / 2
    wing = swept_wing("2412", wing_nc, wing_ns, croot, b, sweep, taper)
    # place the wing root quarter chord near the fuselage mid-length, low wing
    wing.nodes = wing.nodes + np.array([-1.0, 0.0, -0.2])
    return concat([fuse, wing])


def _point_triangle_distance(P, A, B, C):
    """Distances from points P (k, 3) to triangles (A, B, C) (k, 3 each), row by
    row (closest-point regions of the triangle: vertices, edges, face)."""
    ab, ac, ap = B - A, C - A, P - A
    d1, d2 = np.einsum("ij,ij->i", ab, ap), np.einsum("ij,ij->i", ac, ap)
    bp, cp = P - B, P - C
    d3, d4 = np.einsum("ij,ij->i", ab, bp), np.einsum("ij,ij->i", ac, bp)
    d5, d6 = np.einsum("ij,ij->i", ab, cp), np.einsum("ij,ij->i", ac, cp)
    va = d3 * d6 - d5 * d4
    vb = d5 * d2 - d1 * d6
    vc = d1 * d4 - d3 * d2
    denom = va + vb + vc
    with np.errstate(divide="ignore", invalid="ignore"):
        v = vb / denom
        w = vc / denom
    Q = A + ab * v[:, None] + ac * w[:, None]   # interior projection
    # edge and vertex regions
    def seg(X, Y):
        d = Y - X
        t = np.clip(np.einsum("ij,ij->i", P - X, d) / np.maximum(np.einsum("ij,ij->i", d, d), 1e-300), 0, 1)
        return X + d * t[:, None]
    inside = (va >= 0) & (vb >= 0) & (vc >= 0) & (denom > 0)
    cands = [seg(A, B), seg(B, C), seg(C, A)]
    dist = np.min([np.linalg.norm(P - q, axis=1) for q in cands], axis=0)
    dq = np.linalg.norm(P - Q, axis=1)
    return np.where(inside, np.minimum(dq, dist), dist)


def panel_distance(mesh: Mesh, P, panels):
    """Distance from each point P[i] to panel panels[i] (triangles and planar
    quads, the quad as two triangles)."""
    offs = mesh.panel_offsets
    nn = offs[panels + 1] - offs[panels]
    i0 = mesh.panel_nodes[offs[panels]]
    i1 = mesh.panel_nodes[offs[panels] + 1]
    i2 = mesh.panel_nodes[offs[panels] + 2]
    X = mesh.nodes
    d = _point_triangle_distance(P, X[i0], X[i1], X[i2])
    q = nn == 4
    if q.any():
        i3 = mesh.panel_nodes[offs[panels[q]] + 3]
        d[q] = np.minimum(d[q], _point_triangle_distance(P[q], X[i0[q]], X[i2[q]], X[i3]))
    return d


def probe_box(mesh: Mesh, n=1_000_000, lo=(-6.0, -6.0, -2.0), hi=(6.0, 6.0, 2.0), min_dist=0.01, seed=5):
    """n probe points uniform in the box [lo, hi] from default_rng(seed),
    rejecting points closer than min_dist to any panel (exact point-to-panel
    distance for the points near the surface). Draws in batches until n
    points are kept; returns (n, 3)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    offs = mesh.panel_offsets
    cen = np.add.reduceat(mesh.nodes[mesh.panel_nodes], offs[:-1], axis=0) / np.diff(offs)[:, None]
    rad = np.zeros(mesh.npanels)
    for k in range(4):
        sel = np.diff(offs) > k
        idx = mesh.panel_nodes[offs[:-1][sel] + k]
        rad[sel] = np.maximum(rad[sel], np.linalg.norm(mesh.nodes[idx] - cen[sel], axis=1))
    R = rad.max() + min_dist
    tree = cKDTree(cen)
    kept = []
    total = 0
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    while total < n:
        P = lo + (hi - lo) * rng.random((max(n - total, 1) + n // 10 + 16, 3))
        near = tree.query_ball_point(P, R)
        ok = np.ones(len(P), bool)
        cand = [(i, j) for i, lst in enumerate(near) if lst for j in lst]
        if cand:
            ci = np.array([c[0] for c in cand])
            cj = np.array([c[1] for c in cand])
            d = panel_distance(mesh, P[ci], cj)
            bad = np.unique(ci[d < min_dist])
            ok[bad] = False
        P = P[ok]
        kept.append(P)
        total += len(P)
    return np.concatenate(kept)[:n]
