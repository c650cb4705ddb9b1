"""Unstructured surface meshes: file readers and the trailing-edge detection.

FLOWPanel.jl reads meshes through GeoIO (VTK ``.vtu``, Gmsh ``.msh``) into a
``Meshes.SimpleMesh`` wrapped by ``GeometricTools.GridTriangleSurface``, and
builds the wake's shedding matrix with ``calc_shedding``
(src/FLOWPanel_liftingbody.jl:928-1071; test/runtests_meshes.jl:190-230,
test/runtests_meshes2.jl:68-93). Here the same inputs become the flat
``Mesh`` the C ABI takes (nodes, CSR panels, 0-based shedding rows):

* :func:`read_vtu` -- VTK XML UnstructuredGrid (ascii, base64 or appended raw
  data, optionally zlib-compressed, 32- or 64-bit headers);
* :func:`read_msh` -- Gmsh ASCII 2.2 and 4.1 (surface elements only);
* :func:`write_vtu` -- the inverse of :func:`read_vtu` (appended raw, zlib);
* :func:`read_stl` (ASCII or binary, facet vertices welded into nodes) and
  :func:`read_obj` (Wavefront OBJ), two more of the formats GeoIO reads;
* :func:`calc_shedding` -- the shedding matrix of an unstructured mesh from a
  sampled trailing-edge line.

Node and cell order are kept as in the file: the Kutta averages of
``calcfield_Cp``/``calcfield_F`` use the neighbours ``pi+1`` and ``pj-1`` by
index (src/FLOWPanel_postprocess.jl:1083-1097), as in the reference.
"""
from __future__ import annotations

import base64
import struct
import xml.etree.ElementTree as ET
import zlib
from typing import Sequence

import numpy as np

from .meshes import Body, Mesh

_VTK_TYPES = {
    "Int8": np.int8, "UInt8": np.uint8, "Int16": np.int16, "UInt16": np.uint16,
    "Int32": np.int32, "UInt32": np.uint32, "Int64": np.int64, "UInt64": np.uint64,
    "Float32": np.float32, "Float64": np.float64,
}
_VTK_TRIANGLE, _VTK_POLYGON, _VTK_QUAD = 5, 7, 9


def _mesh_from_cells(nodes, cells, kind="vortexring", name="mesh", CPoffset=1e-14):
    offs = np.zeros(len(cells) + 1, np.int32)
    offs[1:] = np.cumsum([len(c) for c in cells])
    pn = np.concatenate([np.asarray(c, np.int32) for c in cells]) if cells else np.zeros(0, np.int32)
    m = Mesh(np.ascontiguousarray(nodes, dtype=np.float64), offs, pn)
    m.bodies = [Body(name, kind, m.npanels, 0, CPoffset)]
    return m


# ----------------------------------------------------------------------------- VTK XML
def _vtu_block(raw: bytes, pos: int, header: type, compressed: bool):
    """Decode one appended-raw data array starting at ``pos``; returns bytes."""
    hs = np.dtype(header).itemsize
    if not compressed:
        (nbytes,) = struct.unpack_from("<" + ("Q" if hs == 8 else "I"), raw, pos)
        return raw[pos + hs: pos + hs + nbytes]
    fmt = "<" + ("Q" if hs == 8 else "I")
    nblocks, bsize, last = (struct.unpack_from(fmt, raw, pos + k * hs)[0] for k in range(3))
    sizes = [struct.unpack_from(fmt, raw, pos + (3 + k) * hs)[0] for k in range(nblocks)]
    p = pos + (3 + nblocks) * hs
    out = []
    for k, s in enumerate(sizes):
        out.append(zlib.decompress(raw[p:p + s]))
        p += s
    data = b"".join(out)
    expect = bsize * (nblocks - 1) + (last if last else bsize) if nblocks else 0
    if len(data) != expect:
        raise ValueError("read_vtu: compressed block sizes do not add up")
    return data


def _vtu_inline_binary(text: str, header: type, compressed: bool):
    hs = np.dtype(header).itemsize
    s = "".join(text.split())
    if not compressed:
        raw = base64.b64decode(s)
        return raw[hs:hs + struct.unpack_from("<" + ("Q" if hs == 8 else "I"), raw, 0)[0]]
    # the header is base64-encoded on its own, then the compressed blocks
    fmt = "<" + ("Q" if hs == 8 else "I")
    first = base64.b64decode(s[:((3 * hs + 2) // 3) * 4])
    nblocks = struct.unpack_from(fmt, first, 0)[0]
    hlen = ((3 + nblocks) * hs + 2) // 3 * 4
    head = base64.b64decode(s[:hlen])
    bsize, last = struct.unpack_from(fmt, head, hs)[0], struct.unpack_from(fmt, head, 2 * hs)[0]
    sizes = [struct.unpack_from(fmt, head, (3 + k) * hs)[0] for k in range(nblocks)]
    body = base64.b64decode(s[hlen:])
    out, p = [], 0
    for sz in sizes:
        out.append(zlib.decompress(body[p:p + sz]))
        p += sz
    return b"".join(out)


def read_vtu(path, kind="vortexring", name=None, CPoffset=1e-14) -> Mesh:
    """Read the surface cells (triangles, quads, polygons of 3-4 nodes) of a VTK
    XML UnstructuredGrid file, in file order. Points become ``nodes``; other
    cell types (vertices, lines) are skipped."""
    with open(path, "rb") as f:
        blob = f.read()
    # appended data follows the first '_' after <AppendedData ...>; it is not XML
    app = blob.find(b"<AppendedData")
    raw, xml_bytes = b"", blob
    if app >= 0:
        start = blob.find(b"_", blob.find(b">", app)) + 1
        end = blob.rfind(b"</AppendedData>")
        raw = blob[start:end]
        xml_bytes = blob[:app] + b"<AppendedData/></VTKFile>"
    root = ET.fromstring(xml_bytes)
    if root.get("type") != "UnstructuredGrid":
        raise ValueError(f"read_vtu: {path} is not a VTK UnstructuredGrid file")
    header = np.uint64 if root.get("header_type", "UInt32") == "UInt64" else np.uint32
    compressed = root.get("compressor") is not None
    if root.get("byte_order", "LittleEndian") != "LittleEndian":
        raise ValueError("read_vtu: big-endian files are not supported")
    piece = root.find("UnstructuredGrid/Piece")

    def array(elem):
        dt = _VTK_TYPES[elem.get("type")]
        fmt = elem.get("format", "ascii")
        if fmt == "ascii":
            return np.array(elem.text.split(), dtype=dt)
        if fmt == "binary":
            return np.frombuffer(_vtu_inline_binary(elem.text, header, compressed), dtype=dt)
        return np.frombuffer(_vtu_block(raw, int(elem.get("offset")), header, compressed), dtype=dt)

    pts = array(piece.find("Points/DataArray")).astype(np.float64).reshape(-1, 3)
    cells = {e.get("Name"): e for e in piece.findall("Cells/DataArray")}
    conn = array(cells["connectivity"]).astype(np.int64)
    offs = array(cells["offsets"]).astype(np.int64)
    types = array(cells["types"]).astype(np.int64)
    out, lo = [], 0
    for hi, t in zip(offs, types):
        c = conn[lo:hi]
        lo = hi
        if t in (_VTK_TRIANGLE, _VTK_QUAD, _VTK_POLYGON) and 3 <= len(c) <= 4:
            out.append(c)
        elif t in (_VTK_TRIANGLE, _VTK_QUAD, _VTK_POLYGON):
            raise ValueError(f"read_vtu: polygon with {len(c)} nodes (3 or 4 supported)")
    return _mesh_from_cells(pts, out, kind, name or str(path), CPoffset)


def write_vtu(path, mesh: Mesh, compress=True):
    """Write ``mesh`` as a VTK XML UnstructuredGrid with appended raw data
    (UInt64 headers, zlib blocks when ``compress``)."""
    nn = np.diff(mesh.panel_offsets)
    types = np.where(nn == 3, _VTK_TRIANGLE, _VTK_QUAD).astype(np.uint8)
    arrays = [("Float64", "Points", 3, np.ascontiguousarray(mesh.nodes, np.float64)),
              ("Int64", "connectivity", 1, mesh.panel_nodes.astype(np.int64)),
              ("Int64", "offsets", 1, mesh.panel_offsets[1:].astype(np.int64)),
              ("UInt8", "types", 1, types)]
    blobs, heads, off = [], [], 0
    for tname, name, nc, a in arrays:
        data = a.tobytes()
        if compress:
            z = zlib.compress(data)
            b = struct.pack("<QQQQ", 1, len(data), len(data), len(z)) + z
        else:
            b = struct.pack("<Q", len(data)) + data
        heads.append((tname, name, nc, off))
        blobs.append(b)
        off += len(b)
    da = ['<DataArray type="%s" Name="%s" NumberOfComponents="%d" format="appended" offset="%d"/>' % h
          for h in heads]
    comp = ' compressor="vtkZLibDataCompressor"' if compress else ""
    xml = ('<?xml version="1.0" encoding="utf-8"?>\n'
           '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64"%s>\n'
           '  <UnstructuredGrid>\n    <Piece NumberOfPoints="%d" NumberOfCells="%d">\n'
           '      <Points>\n        %s\n      </Points>\n      <Cells>\n        %s\n        %s\n        %s\n'
           '      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding="raw">\n   _'
           % (comp, mesh.nnodes, mesh.npanels, da[0], da[1], da[2], da[3]))
    with open(path, "wb") as f:
        f.write(xml.encode())
        for b in blobs:
            f.write(b)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")


# ----------------------------------------------------------------------------- Gmsh
_GMSH_NODES = {2: 3, 3: 4}      # 3-node triangle, 4-node quadrangle


def read_msh(path, kind="vortexring", name=None, CPoffset=1e-14) -> Mesh:
    """Read the triangles and quadrangles of a Gmsh ASCII mesh (format 2.2 or
    4.1), in file order; node tags are mapped to 0-based indices in the order
    the nodes appear."""
    with open(path, "r") as f:
        lines = f.read().split("\n")
    pos = {}
    k = 0
    while k < len(lines):
        s = lines[k].strip()
        if s.startswith("$") and not s.startswith("$End"):
            pos[s[1:]] = k
        k += 1
    if "MeshFormat" not in pos:
        raise ValueError(f"read_msh: {path} has no $MeshFormat section")
    version = float(lines[pos["MeshFormat"] + 1].split()[0])
    if lines[pos["MeshFormat"] + 1].split()[1] != "0":
        raise ValueError("read_msh: binary Gmsh files are not supported")
    tags, xyz, cells = [], [], []
    if version >= 4.0:
        k = pos["Nodes"] + 1
        nblocks = int(lines[k].split()[0]); k += 1
        for _ in range(nblocks):
            _, _, parametric, n = (int(v) for v in lines[k].split()); k += 1
            tags.extend(int(lines[k + i]) for i in range(n)); k += n
            for i in range(n):
                v = lines[k + i].split()
                xyz.append([float(v[0]), float(v[1]), float(v[2])])
            k += n
        k = pos["Elements"] + 1
        nblocks = int(lines[k].split()[0]); k += 1
        for _ in range(nblocks):
            _, _, etype, n = (int(v) for v in lines[k].split()); k += 1
            if etype in _GMSH_NODES:
                for i in range(n):
                    v = lines[k + i].split()
                    cells.append([int(t) for t in v[1:1 + _GMSH_NODES[etype]]])
            k += n
    else:
        k = pos["Nodes"] + 1
        n = int(lines[k]); k += 1
        for i in range(n):
            v = lines[k + i].split()
            tags.append(int(v[0]))
            xyz.append([float(v[1]), float(v[2]), float(v[3])])
        k = pos["Elements"] + 1
        n = int(lines[k]); k += 1
        for i in range(n):
            v = [int(t) for t in lines[k + i].split()]
            etype, ntags = v[1], v[2]
            if etype in _GMSH_NODES:
                cells.append(v[3 + ntags:3 + ntags + _GMSH_NODES[etype]])
    index = {t: i for i, t in enumerate(tags)}
    try:
        cells = [[index[t] for t in c] for c in cells]
    except KeyError as e:
        raise ValueError(f"read_msh: element references unknown node tag {e}") from None
    return _mesh_from_cells(np.asarray(xyz, np.float64).reshape(-1, 3), cells, kind, name or str(path), CPoffset)


# ----------------------------------------------------------------------------- STL / OBJ
def weld_nodes(points, tolerance=0.0):
    """Merge points closer than ``tolerance`` (exact duplicates when 0); returns
    (unique nodes in first-appearance order, index of each input point)."""
    points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    if tolerance <= 0.0:
        _, first, inv = np.unique(points, axis=0, return_index=True, return_inverse=True)
    else:
        from scipy.spatial import cKDTree
        pairs = cKDTree(points).query_pairs(tolerance, output_type="ndarray")
        root = np.arange(len(points))

        def find(i):
            while root[i] != i:
                root[i] = root[root[i]]
                i = root[i]
            return i
        for i, j in pairs:
            ri, rj = find(i), find(j)
            if ri != rj:
                root[max(ri, rj)] = min(ri, rj)
        lab = np.array([find(i) for i in range(len(points))])
        _, first, inv = np.unique(lab, return_index=True, return_inverse=True)
    inv = np.asarray(inv).ravel()
    order = np.argsort(first, kind="stable")          # first-appearance order
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    return points[np.sort(first)], rank[inv]


def read_stl(path, kind="vortexring", name=None, CPoffset=1e-14, tolerance=0.0) -> Mesh:
    """Read an STL file (ASCII or binary) as triangles in file order; the
    per-facet vertices are welded into shared nodes (exact duplicates, or
    within ``tolerance``), so neighbouring facets share their edges."""
    with open(path, "rb") as f:
        blob = f.read()
    tris = None
    if len(blob) >= 84:
        ntri = struct.unpack_from("<I", blob, 80)[0]
        if 84 + 50 * ntri == len(blob):
            rec = np.frombuffer(blob, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]),
                                count=ntri, offset=84)
            tris = rec["v"].astype(np.float64).reshape(-1, 3)
    if tris is None:
        text = blob.decode("ascii", errors="replace").split()
        if not text or text[0].lower() != "solid":
            raise ValueError(f"read_stl: {path} is neither binary nor ASCII STL")
        vs = [[float(text[i + 1]), float(text[i + 2]), float(text[i + 3])]
              for i, t in enumerate(text) if t.lower() == "vertex"]
        if len(vs) % 3:
            raise ValueError("read_stl: facets must have three vertices")
        tris = np.asarray(vs, np.float64).reshape(-1, 3)
    nodes, idx = weld_nodes(tris, tolerance)
    cells = idx.reshape(-1, 3).tolist()
    return _mesh_from_cells(nodes, cells, kind, name or str(path), CPoffset)


def read_obj(path, kind="vortexring", name=None, CPoffset=1e-14) -> Mesh:
    """Read the vertices and the 3- and 4-vertex faces of a Wavefront OBJ file
    (``f`` entries may carry /texture/normal indices; negative indices count
    from the end)."""
    nodes, cells = [], []
    with open(path, "r") as f:
        for line in f:
            p = line.split()
            if not p:
                continue
            if p[0] == "v":
                nodes.append([float(p[1]), float(p[2]), float(p[3])])
            elif p[0] == "f":
                ids = []
                for tok in p[1:]:
                    i = int(tok.split("/")[0])
                    ids.append(i - 1 if i > 0 else len(nodes) + i)
                if not 3 <= len(ids) <= 4:
                    raise ValueError(f"read_obj: face with {len(ids)} vertices (3 or 4 supported)")
                cells.append(ids)
    return _mesh_from_cells(np.asarray(nodes, np.float64).reshape(-1, 3), cells, kind, name or str(path), CPoffset)


# ----------------------------------------------------------------------------- trailing edge
def identify_edge(nodes, line, tolerance):
    """Nodes closer than ``tolerance`` to a sampled line, as (node, sample)
    pairs ordered along the line: each node is paired with the first sample
    (in the line's order) that lies within the tolerance, ties broken by node
    index (the ``identifyedge`` step of calc_shedding,
    src/FLOWPanel_liftingbody.jl:950-952)."""
    from scipy.spatial import cKDTree

    nodes = np.asarray(nodes, float)
    line = np.asarray(line, float)
    tree = cKDTree(line)
    near = tree.query_ball_point(nodes, tolerance)
    pairs = [(i, min(lst)) for i, lst in enumerate(near) if lst]
    pairs.sort(key=lambda p: (p[1], p[0]))
    return pairs


def _edge_table(mesh: Mesh):
    """(min node, max node) -> list of (cell, local edge k) for the edge from
    local node k to k+1."""
    table = {}
    offs, pn = mesh.panel_offsets, mesh.panel_nodes
    for c in range(mesh.npanels):
        p = pn[offs[c]:offs[c + 1]]
        n = len(p)
        for k in range(n):
            a, b = int(p[k]), int(p[(k + 1) % n])
            table.setdefault((min(a, b), max(a, b)), []).append((c, k))
    return table


def calc_shedding(mesh: Mesh, trailingedge, periodic=False, tolerance=1e2 * np.finfo(float).eps):
    """Shedding matrix (nsh, 6) of an unstructured mesh from a trailing-edge
    line sampled by the points ``trailingedge`` (k, 3), sorted along the edge
    (calc_shedding, src/FLOWPanel_liftingbody.jl:942-1071):

    nodes within ``tolerance`` of the line, in line order; consecutive pairs
    (a, b) that are an edge of the mesh; pi = the panel that runs a -> b in its
    node order, pj = the one that runs b -> a (-1 on a single-sided edge, where
    pi is the panel that exists); (nia, nib) = local indices of (b, a) in pi,
    (nja, njb) = local indices of (a, b) in pj (-1, -1 when pj = -1).
    Returns 0-based rows."""
    te = [n for n, _ in identify_edge(mesh.nodes, np.asarray(trailingedge, float).reshape(-1, 3), tolerance)]
    if not te:
        return np.zeros((0, 6), np.int32)
    if periodic:
        te.append(te[0])
    table = _edge_table(mesh)
    offs, pn = mesh.panel_offsets, mesh.panel_nodes

    def local(c, node):
        p = list(pn[offs[c]:offs[c + 1]])
        return p.index(node)

    def runs(c, a, b):
        p = list(pn[offs[c]:offs[c + 1]])
        n = len(p)
        return any(p[k] == a and p[(k + 1) % n] == b for k in range(n))

    rows = []
    for a, b in zip(te[:-1], te[1:]):
        owners = table.get((min(a, b), max(a, b)))
        if not owners:
            continue
        cs = [c for c, _ in owners]
        if len(cs) > 2:
            raise ValueError(f"calc_shedding: edge ({a}, {b}) is shared by more than two panels")
        if len(cs) == 1:
            pi, pj = cs[0], -1
        elif runs(cs[0], a, b):
            pi, pj = cs[0], cs[1]
        elif runs(cs[1], a, b):
            pi, pj = cs[1], cs[0]
        else:
            raise ValueError("Logic error: Could not match panel to node pair")
        nia, nib = local(pi, b), local(pi, a)
        nja, njb = (local(pj, a), local(pj, b)) if pj != -1 else (-1, -1)
        rows.append((pi, nia, nib, pj, nja, njb))
    return np.asarray(rows, np.int32).reshape(-1, 6)


def lifting_mesh(mesh: Mesh, shedding, name=None, CPoffset=1e-14, kerneloffset=1e-8,
                 kernelcutoff=1e-14) -> Mesh:
    """The mesh as one vortex-ring body with the given shedding rows."""
    out = Mesh(mesh.nodes, mesh.panel_offsets, mesh.panel_nodes, np.asarray(shedding, np.int32).reshape(-1, 6))
    out.bodies = [Body(name or (mesh.bodies[0].name if mesh.bodies else "mesh"), "vortexring", mesh.npanels,
                       out.nsheddings, CPoffset, kerneloffset, kernelcutoff)]
    return out


def sample_line(points: Sequence, n: int, sortdir=None):
    """``n`` evenly spaced samples on each segment of the polyline ``points``
    (consecutive segments share their joint), optionally sorted by the
    projection on ``sortdir`` (the trailing-edge construction of
    test/runtests_meshes.jl:198-206 and test/runtests_meshes2.jl:77-85)."""
    pts = np.asarray(points, float)
    segs = []
    for k in range(len(pts) - 1):
        t = np.linspace(0.0, 1.0, n)[:, None]
        s = pts[k] + t * (pts[k + 1] - pts[k])
        segs.append(s if k == 0 else s[1:])
    line = np.concatenate(segs)
    if sortdir is not None:
        line = line[np.argsort(line @ np.asarray(sortdir, float), kind="stable")]
    return line
