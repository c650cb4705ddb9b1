"""Regenerate the mesh fixtures of this folder from FLOWPanel.jl's example data.

Run from the repository root where the reference checkout is available:

    python tests/golden/make_fixtures.py /path/to/FLOWPanel.jl

* ``sweptwing_vtu.npz``: the two half-wing meshes of
  examples/data/sweptwing-{left,right}000.vtu (768 nodes, 1,440 triangles
  each), read with ``meshio.read_vtu``; used by test/runtests_meshes.jl:190-230.
* ``sweptwing_openvsp.npz``: the OpenVSP wing of
  examples/data/sweptwing-openvsp.msh (Gmsh 4.1; 6,398 nodes, 12,792
  triangles), read with ``meshio.read_msh``; used by
  test/runtests_meshes2.jl:45-93.

* ``airfoils.npz``: the airfoil contours examples/data/airfoil-rae101.csv
  (RAE 101, the swept wing of test/runtests_solvers.jl and
  examples/sweptwing.jl) and examples/data/naca662015.csv (NACA 66-2015, the
  duct of test/runtests_solvers2.jl), (x, y) in file order.

Nodes are float64, cells int32 CSR (0-based), both in file order.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402


def main(ref):
    ge.load_package()
    import flowpanel_b200.meshio as mio

    data = os.path.join(ref, "examples", "data")
    out = {}
    for side, f in (("L", "sweptwing-left000.vtu"), ("R", "sweptwing-right000.vtu")):
        m = mio.read_vtu(os.path.join(data, f))
        out[f"nodes_{side}"] = m.nodes
        out[f"offsets_{side}"] = m.panel_offsets
        out[f"pnodes_{side}"] = m.panel_nodes
    np.savez_compressed(os.path.join(HERE, "sweptwing_vtu.npz"), **out)
    np.savez_compressed(os.path.join(HERE, "airfoils.npz"),
                        rae101=np.loadtxt(os.path.join(data, "airfoil-rae101.csv"), delimiter=",", skiprows=1),
                        naca662015=np.loadtxt(os.path.join(data, "naca662015.csv"), delimiter=",", skiprows=1))
    m = mio.read_msh(os.path.join(data, "sweptwing-openvsp.msh"))
    np.savez_compressed(os.path.join(HERE, "sweptwing_openvsp.npz"), nodes=m.nodes, offsets=m.panel_offsets,
                        pnodes=m.panel_nodes)


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("FLOWPANEL_REFERENCE"):
        sys.exit("usage: make_fixtures.py /path/to/FLOWPanel.jl  (or set FLOWPANEL_REFERENCE)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["FLOWPANEL_REFERENCE"])
