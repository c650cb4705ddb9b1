"""The C-ABI library loads and exports every symbol include/flowpanel_b200.h declares (CPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "flowpanel_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fp_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("fp_ctx_create", "fp_set_geometry", "fp_set_wake", "fp_assemble", "fp_factor", "fp_solve",
              "fp_solve_body", "fp_uind", "fp_adjoint_solve"):
        assert s in syms


def test_library_exports_every_declared_symbol(fp):
    path = fp._capi.LIB_PATH
    if not os.path.exists(path):
        pytest.skip("CUDA library not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(fp._capi.EXPORTS) == set(declared_symbols())


def test_no_device_is_a_clean_error(fp):
    """Without a GPU the library reports an error instead of running anything on the CPU."""
    path = fp._capi.LIB_PATH
    if not os.path.exists(path):
        pytest.skip("CUDA library not built")
    lib = fp._capi.lib()
    if lib.fp_device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(fp._capi.FlowPanelError):
        fp._capi.Context(0)


def test_binding_constants_match_header(fp):
    """Every integer #define of include/flowpanel_b200.h that the Python binding
    also defines has the same value there, and every fp_set_tuning knob
    (FP_TUNE_*) is defined in the binding."""
    src = open(os.path.join(ROOT, "include", "flowpanel_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    defs = {k: int(v) for k, v in re.findall(r"^\s*#define\s+(FP_\w+)\s+(-?\d+)\s*$", src, flags=re.M)}
    assert any(k.startswith("FP_TUNE_") for k in defs)
    cap = fp._capi
    for k, v in defs.items():
        if k.startswith("FP_TUNE_"):
            assert hasattr(cap, k), k
        if hasattr(cap, k):
            assert getattr(cap, k) == v, (k, getattr(cap, k), v)
    knobs = sorted(v for k, v in defs.items() if k.startswith("FP_TUNE_"))
    assert knobs == list(range(len(knobs)))   # knob numbers are dense from 0
