"""Mesh ingestion (VTK .vtu, Gmsh .msh) and the trailing-edge detection of
calc_shedding (src/FLOWPanel_liftingbody.jl:942-1071) on CPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the reference checkout's example data, when FLOWPANEL_REFERENCE names a checkout
# (the fixture comparison below is skipped otherwise)
REF_DATA = os.path.join(os.environ.get("FLOWPANEL_REFERENCE", ""), "examples", "data") \
    if os.environ.get("FLOWPANEL_REFERENCE") else ""

# trailing edges of test/runtests_meshes.jl:198-206 (left half; the right one mirrors y)
TE_X1 = {"L": [1.74244, -1.2446, 1.38094e-07], "R": [1.74244, 1.2446, 1.38094e-07]}
TE_X2 = [0.49784, -1.38178e-16, 1.38094e-07]
SPANDIR = {"L": [0, 1, 0], "R": [0, -1, 0]}


def fixture_mesh(fp, side):
    z = np.load(os.path.join(GOLDEN, "sweptwing_vtu.npz"))
    m = fp.meshes.Mesh(z[f"nodes_{side}"], z[f"offsets_{side}"], z[f"pnodes_{side}"])
    m.bodies = [fp.meshes.Body(side, "vortexring", m.npanels, 0)]
    return m


def te_line(fp, side, n=1000):
    return fp.meshio.sample_line([TE_X1[side], TE_X2], n, SPANDIR[side])


def test_vtu_roundtrip(fp, tmp_path):
    m = fp.meshes.triangulate(fp.meshes.swept_wing("0012", 12, 8))
    quads = fp.meshes.swept_wing("0012", 10, 6)
    for mesh in (m, quads):
        for compress in (True, False):
            path = tmp_path / f"w{compress}{mesh.npanels}.vtu"
            fp.meshio.write_vtu(path, mesh, compress=compress)
            r = fp.meshio.read_vtu(path)
            assert np.array_equal(r.nodes, mesh.nodes)
            assert np.array_equal(r.panel_offsets, mesh.panel_offsets)
            assert np.array_equal(r.panel_nodes, mesh.panel_nodes)


def test_vtu_ascii_and_base64(fp, tmp_path):
    """Inline ascii and inline base64 (uncompressed, UInt32 headers) arrays."""
    import base64
    import struct
    pts = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], float)
    conn = np.array([0, 1, 2, 0, 2, 3], np.int32)

    def b64(a):
        raw = a.tobytes()
        return base64.b64encode(struct.pack("<I", len(raw)) + raw).decode()
    xml = f"""<?xml version="1.0"?>
<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">
  <UnstructuredGrid><Piece NumberOfPoints="4" NumberOfCells="3">
    <Points><DataArray type="Float64" NumberOfComponents="3" format="binary">{b64(pts)}</DataArray></Points>
    <Cells>
      <DataArray type="Int32" Name="connectivity" format="ascii">0 1 2 0 2 3 0 1</DataArray>
      <DataArray type="Int32" Name="offsets" format="ascii">3 6 8</DataArray>
      <DataArray type="UInt8" Name="types" format="ascii">5 5 3</DataArray>
    </Cells>
  </Piece></UnstructuredGrid>
</VTKFile>"""
    path = tmp_path / "a.vtu"
    path.write_text(xml)
    m = fp.meshio.read_vtu(path)
    assert np.array_equal(m.nodes, pts)
    assert m.npanels == 2                      # the line cell (type 3) is skipped
    assert np.array_equal(m.panel_nodes, conn)


def test_msh_formats(fp, tmp_path):
    v41 = """$MeshFormat
4.1 0 8
$EndMeshFormat
$Nodes
1 4 10 13
2 1 0 4
10
11
12
13
0 0 0
1 0 0
1 1 0
0 1 0
$EndNodes
$Elements
2 3 1 3
1 1 1 1
1 10 11
2 1 2 2
2 10 11 12
3 10 12 13
$EndElements
"""
    v22 = """$MeshFormat
2.2 0 8
$EndMeshFormat
$Nodes
4
7 0 0 0
8 1 0 0
9 1 1 0
5 0 1 0
$EndNodes
$Elements
3
1 15 2 0 1 7
2 2 2 0 1 7 8 9
3 3 2 0 1 7 8 9 5
$EndElements
"""
    (tmp_path / "a.msh").write_text(v41)
    (tmp_path / "b.msh").write_text(v22)
    a = fp.meshio.read_msh(tmp_path / "a.msh")
    b = fp.meshio.read_msh(tmp_path / "b.msh")
    assert a.npanels == 2 and np.array_equal(a.panel_nodes, [0, 1, 2, 0, 2, 3])
    assert b.npanels == 2 and np.array_equal(np.diff(b.panel_offsets), [3, 4])
    assert np.array_equal(b.panel_nodes, [0, 1, 2, 0, 1, 2, 3])
    assert np.allclose(a.nodes, b.nodes)
    # a trailing-edge line mesh (line elements only, as the Cessna example's
    # TE files): its nodes are the points of the line, it has no panels
    line = """$MeshFormat
4.1 0 8
$EndMeshFormat
$Nodes
1 3 1 3
1 1 0 3
1
2
3
0 0 0
0.5 0 0
1 0 0
$EndNodes
$Elements
1 2 1 2
1 1 1 2
1 1 2
2 2 3
$EndElements
"""
    (tmp_path / "te.msh").write_text(line)
    te = fp.meshio.read_msh(tmp_path / "te.msh")
    assert te.npanels == 0 and te.nnodes == 3 and np.allclose(te.nodes[:, 0], [0, 0.5, 1])


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA),
                    reason="set FLOWPANEL_REFERENCE to a FLOWPanel.jl checkout to compare the fixtures")
def test_fixtures_match_reference_files(fp):
    for side, f in (("L", "sweptwing-left000.vtu"), ("R", "sweptwing-right000.vtu")):
        m = fp.meshio.read_vtu(os.path.join(REF_DATA, f))
        g = fixture_mesh(fp, side)
        assert np.array_equal(m.nodes, g.nodes) and np.array_equal(m.panel_nodes, g.panel_nodes)
    m = fp.meshio.read_msh(os.path.join(REF_DATA, "sweptwing-openvsp.msh"))
    z = np.load(os.path.join(GOLDEN, "sweptwing_openvsp.npz"))
    assert np.array_equal(m.nodes, z["nodes"]) and np.array_equal(m.panel_nodes, z["pnodes"])


@pytest.mark.parametrize("side", ["L", "R"])
def test_calc_shedding_vtu_wing(fp, side):
    """One shedding row per spanwise strip; pi runs a -> b, pj runs b -> a; the
    local indices name the trailing-edge nodes."""
    m = fixture_mesh(fp, side)
    line = te_line(fp, side)
    span = np.ptp(line @ np.asarray(SPANDIR[side], float))
    sh = fp.meshio.calc_shedding(m, line, tolerance=0.001 * span)
    assert sh.shape == (15, 6)
    te = [n for n, _ in fp.meshio.identify_edge(m.nodes, line, 0.001 * span)]
    assert len(te) == 16
    # TE nodes ordered along the span direction
    s = m.nodes[te] @ np.asarray(SPANDIR[side], float)
    assert np.all(np.diff(s) > 0)
    for r, (pi, nia, nib, pj, nja, njb) in enumerate(sh):
        a, b = te[r], te[r + 1]
        P = list(m.panel(pi))
        Q = list(m.panel(pj))
        assert P[nia] == b and P[nib] == a and Q[nja] == a and Q[njb] == b
        assert any(P[k] == a and P[(k + 1) % 3] == b for k in range(3))
        assert any(Q[k] == b and Q[(k + 1) % 3] == a for k in range(3))


def test_calc_shedding_single_sided_and_periodic(fp):
    """A free trailing edge gives pj = -1; ``periodic`` closes the node loop."""
    nodes = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], float)
    m = fp.meshes.Mesh(nodes, np.array([0, 3, 6], np.int32), np.array([0, 1, 2, 0, 2, 3], np.int32))
    sh = fp.meshio.calc_shedding(m, fp.meshio.sample_line([[1, 0, 0], [1, 1, 0]], 101), tolerance=1e-3)
    assert sh.tolist() == [[0, 2, 1, -1, -1, -1]]
    sq = fp.meshio.sample_line([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], 101)
    sh = fp.meshio.calc_shedding(m, sq, periodic=True, tolerance=1e-3)
    assert len(sh) == 4 and sh[-1][0] == 1   # the closing edge (3, 0) belongs to the second triangle
    assert len(fp.meshio.calc_shedding(m, np.array([[5.0, 5.0, 5.0]]), tolerance=1e-3)) == 0


def test_calc_shedding_errors_and_ties(fp):
    """An edge of three panels is refused; nodes at the same sample keep node order."""
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0], [0.5, 0, 1]], float)
    m = fp.meshes.Mesh(nodes, np.array([0, 3, 6, 9], np.int32),
                       np.array([0, 1, 2, 1, 0, 3, 0, 1, 4], np.int32))
    with pytest.raises(ValueError, match="more than two panels"):
        fp.meshio.calc_shedding(m, fp.meshio.sample_line([[0, 0, 0], [1, 0, 0]], 11), tolerance=1e-3)
    pairs = fp.meshio.identify_edge(np.array([[0, 0, 0], [0, 0, 1e-9], [1, 0, 0]], float),
                                    np.array([[0, 0, 0], [1, 0, 0]], float), 1e-6)
    assert pairs == [(0, 0), (1, 0), (2, 1)]


def test_vtu_polygon_cells(fp, tmp_path):
    """VTK_POLYGON cells of 3 and 4 nodes are panels; larger polygons are refused."""
    pts = " ".join(str(v) for v in [0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0, 2, 0, 0, 2, 1, 0])
    def vtu(conn, offs, types):
        return f"""<?xml version="1.0"?>
<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">
  <UnstructuredGrid><Piece NumberOfPoints="6" NumberOfCells="{len(types.split())}">
    <Points><DataArray type="Float32" NumberOfComponents="3" format="ascii">{pts}</DataArray></Points>
    <Cells>
      <DataArray type="Int64" Name="connectivity" format="ascii">{conn}</DataArray>
      <DataArray type="Int64" Name="offsets" format="ascii">{offs}</DataArray>
      <DataArray type="UInt8" Name="types" format="ascii">{types}</DataArray>
    </Cells>
  </Piece></UnstructuredGrid>
</VTKFile>"""
    (tmp_path / "p.vtu").write_text(vtu("0 1 2 3 1 4 5 2", "4 8", "7 9"))
    m = fp.meshio.read_vtu(tmp_path / "p.vtu")
    assert m.npanels == 2 and np.array_equal(np.diff(m.panel_offsets), [4, 4])
    (tmp_path / "q.vtu").write_text(vtu("0 1 4 5 2 3", "6", "7"))
    with pytest.raises(ValueError, match="polygon with 6 nodes"):
        fp.meshio.read_vtu(tmp_path / "q.vtu")


def test_stl_and_obj(fp, O, tmp_path):
    """STL (ASCII and binary, vertices welded) and OBJ faces give the mesh back."""
    import struct
    m = fp.meshes.triangulate(fp.meshes.sphere(1.0, 6, 8))
    P = m.nodes
    tri = m.panel_nodes.reshape(-1, 3)
    lines = ["solid s"]
    for t in tri:
        lines += ["facet normal 0 0 0", "outer loop"] + ["vertex %.17g %.17g %.17g" % tuple(P[i]) for i in t] + \
                 ["endloop", "endfacet"]
    (tmp_path / "a.stl").write_text("\n".join(lines + ["endsolid s"]))
    b = bytearray(80) + struct.pack("<I", len(tri))
    for t in tri:
        b += struct.pack("<3f", 0, 0, 0) + struct.pack("<9f", *P[t].astype(np.float32).ravel()) + b"\0\0"
    (tmp_path / "b.stl").write_bytes(bytes(b))
    for f, tol in (("a.stl", 0.0), ("b.stl", 1e-6)):
        r = fp.meshio.read_stl(tmp_path / f, tolerance=tol)
        assert r.npanels == len(tri)
        # the welded mesh is watertight like the original: every edge has two panels
        assert (O.mesh_neighbors(r) >= 0).all()
        assert np.abs(r.nodes[r.panel_nodes] - P[m.panel_nodes]).max() < 1e-6
    obj = ["v %.17g %.17g %.17g" % tuple(p) for p in P] + \
          ["f " + " ".join(f"{i + 1}/1/1" for i in t) for t in tri[:-1]] + \
          ["f " + " ".join(str(i - m.nnodes) for i in tri[-1])]
    (tmp_path / "c.obj").write_text("\n".join(obj))
    r = fp.meshio.read_obj(tmp_path / "c.obj")
    assert np.array_equal(r.panel_nodes, m.panel_nodes) and np.array_equal(r.nodes, P)
