"""B200-native (sm_100a) panel-method hot path of FLOWPanel.jl.

Host mirror of the reference's ``solve`` / ``calcfield_*`` API over the C ABI
of ``include/flowpanel_b200.h`` (kernels in ``csrc/``); synthetic workload
meshes in ``meshes``, mesh files and trailing-edge detection in ``meshio``. Import name: ``flowpanel_b200`` (loaded from this
directory by ``__graft_entry__.load_package``).
"""
from . import _capi, meshes, meshio  # noqa: F401
from .bodies import (B200Solver, MultiBody, NonLiftingBody, RigidWakeBody, Uind, addfields,  # noqa: F401
                     calc_areas, calc_controlpoints, calc_normals, calcfield_Cp, calcfield_F,
                     calcfield_LDS, calcfield_U, calcfield_Ugradmu, calcfield_Ugradmu_cell, smooth_rows_cells,
                     calcfield_Ugradmu_node, phi, solve, solve_batch, surface_loads)

__all__ = ["B200Solver", "MultiBody", "NonLiftingBody", "RigidWakeBody", "solve", "solve_batch", "Uind", "phi",
           "calcfield_U",
           "calcfield_Cp", "calcfield_F", "calcfield_LDS", "calcfield_Ugradmu", "calcfield_Ugradmu_cell", "smooth_rows_cells",
           "calcfield_Ugradmu_node", "addfields", "surface_loads", "calc_normals", "calc_controlpoints",
           "calc_areas", "meshes", "meshio"]


def __getattr__(name):
    # the reverse-mode module imports torch; load it on first use
    if name == "adjoint":
        import importlib
        return importlib.import_module(__name__ + ".adjoint")
    raise AttributeError(name)
