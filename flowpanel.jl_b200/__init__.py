"""B200-native (sm_100a) panel-method hot path of FLOWPanel.jl.

Host mirror of the reference's ``solve`` / ``calcfield_*`` API over the C ABI
of ``include/flowpanel_b200.h`` (kernels in ``csrc/``); synthetic workload
meshes in ``meshes``. Import name: ``flowpanel_b200`` (loaded from this
directory by ``__graft_entry__.load_package``).
"""
from . import _capi, meshes  # noqa: F401
from .bodies import (B200Solver, MultiBody, NonLiftingBody, RigidWakeBody, Uind,  # noqa: F401
                     calc_areas, calc_controlpoints, calc_normals, calcfield_Cp, calcfield_F,
                     calcfield_LDS, calcfield_U, phi, solve, solve_batch)

__all__ = ["B200Solver", "MultiBody", "NonLiftingBody", "RigidWakeBody", "solve", "solve_batch", "Uind", "phi",
           "calcfield_U",
           "calcfield_Cp", "calcfield_F", "calcfield_LDS", "calc_normals", "calc_controlpoints",
           "calc_areas", "meshes"]


def __getattr__(name):
    # the reverse-mode module imports torch; load it on first use
    if name == "adjoint":
        import importlib
        return importlib.import_module(__name__ + ".adjoint")
    raise AttributeError(name)
