"""ctypes bindings of include/flowpanel_b200.h (the library's C ABI).

The library is loaded from ``_build/libflowpanel_b200.so`` inside this
package. There is no CPU fallback: without the library (or without a GPU)
every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libflowpanel_b200.so")

FP_OK, FP_EINVAL, FP_ESINGULAR, FP_ENOCONV, FP_ECUDA, FP_ETIMEOUT, FP_ESTATE = range(7)
FP_ELEMENT_SOURCE, FP_ELEMENT_VORTEXRING, FP_ELEMENT_SOURCE_DOUBLET = 0, 1, 2
FP_PREC_FP64, FP_PREC_MIXED, FP_PREC_MIXED_GEPP, FP_PREC_BF16 = 0, 1, 2, 3
_PRECISIONS = {"fp64": FP_PREC_FP64, "mixed": FP_PREC_MIXED, "mixed_gepp": FP_PREC_MIXED_GEPP, "bf16": FP_PREC_BF16}
FP_SOLVER_LU, FP_SOLVER_GMRES = 0, 1
FP_STAGE_ASSEMBLE, FP_STAGE_FACTOR, FP_STAGE_SOLVE, FP_STAGE_UIND, FP_STAGE_ADJOINT, FP_STAGE_VJP, FP_STAGE_POST, FP_STAGE_PHI = range(8)
FP_UGRADMU_COMBINED, FP_UGRADMU_CELL, FP_UGRADMU_NODE = 0, 1, 2

# every symbol the header declares
EXPORTS = ("fp_ctx_create", "fp_ctx_destroy", "fp_last_error", "fp_device_count", "fp_set_geometry",
           "fp_set_wake", "fp_assemble", "fp_get_aic", "fp_set_rhs", "fp_factor", "fp_solve",
           "fp_solve_body", "fp_uind", "fp_adjoint_solve", "fp_last_kernel_ms", "fp_measure_fma_peak",
           "fp_kernel_launches", "fp_tc_selftest", "fp_lu_solve_noalloc", "fp_assembly_vjp",
           "fp_uind_vjp", "fp_kernel_timing", "fp_kernel_timing_read", "fp_batch_create",
           "fp_batch_destroy", "fp_batch_last_error", "fp_batch_solve", "fp_trace", "fp_trace_read", "fp_phi", "fp_solve_ls",
           "fp_ugradmu", "fp_ugradmu_ex", "fp_calcfield_cp", "fp_calcfield_f", "fp_calcfield_lds", "fp_surface_loads",
           "fp_set_tuning", "fp_autotune")
FP_TUNE_TC_STAGES, FP_TUNE_LU_OVERLAP, FP_TUNE_TC_TILES, FP_TUNE_GRAPH, FP_TUNE_TC_SMEM = 0, 1, 2, 3, 4
FP_TUNE_FP64_DMMA, FP_TUNE_TC_SPLIT, FP_TUNE_TC_RED, FP_TUNE_ASM32, FP_TUNE_TC_NARROW = 5, 6, 7, 8, 9
FP_TUNE_TRS2 = 10
FP_TUNE_PANEL_GEMM = 11
FP_TUNE_TC_BF16X3 = 12
FP_TUNE_TC_PREFETCH = 13
FP_TUNE_PDL = 14
FP_TUNE_LU_SPLIT = 15
FP_TUNE_LU_FUSE = 16
FP_TUNE_U12_WIDE = 17
FP_TUNE_L21_ASYNC = 18
FP_TUNE_U12_ASYNC = 19
FP_TUNE_REST_SPLIT = 20
FP_TUNE_PDIAG_LINV = 21


class SolveOpts(C.Structure):
    _fields_ = [("solver", C.c_int), ("precision", C.c_int), ("ir_tol", C.c_double),
                ("ir_maxiter", C.c_int), ("gmres_memory", C.c_int), ("gmres_atol", C.c_double),
                ("gmres_rtol", C.c_double), ("gmres_itmax", C.c_int), ("gmres_restart", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("ms_assemble", C.c_double), ("ms_factor", C.c_double), ("ms_solve", C.c_double),
                ("ir_iters", C.c_int), ("gmres_iters", C.c_int), ("used_gmres", C.c_int),
                ("gepp_certified", C.c_int), ("max_abs_L", C.c_double), ("rel_residual", C.c_double)]

    def asdict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BodyDesc(C.Structure):
    _fields_ = [("nodes", C.POINTER(C.c_double)), ("nnodes", C.c_int64),
                ("panel_offsets", C.POINTER(C.c_int32)), ("panel_nodes", C.POINTER(C.c_int32)),
                ("npanels", C.c_int64), ("cps", C.POINTER(C.c_double)), ("normals", C.POINTER(C.c_double)),
                ("shedding", C.POINTER(C.c_int32)), ("nsh", C.c_int64), ("Das", C.POINTER(C.c_double)),
                ("Dbs", C.POINTER(C.c_double)), ("Uinfs", C.POINTER(C.c_double)), ("x", C.POINTER(C.c_double))]


class FlowPanelError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not found: build the CUDA library first "
                               "(python flowpanel.jl_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.fp_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.fp_ctx_destroy.argtypes = [vp]
        L.fp_last_error.argtypes = [vp]
        L.fp_last_error.restype = C.c_char_p
        L.fp_device_count.argtypes = []
        L.fp_set_geometry.argtypes = [vp, _dp, C.c_int64, _ip, _ip, C.c_int64, _dp, _dp, _dp]
        L.fp_set_wake.argtypes = [vp, _ip, C.c_int64, _dp, _dp]
        L.fp_assemble.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_int]
        L.fp_get_aic.argtypes = [vp, _dp]
        L.fp_set_rhs.argtypes = [vp, _dp, C.c_int64]
        L.fp_factor.argtypes = [vp, C.c_int]
        L.fp_set_tuning.argtypes = [vp, C.c_int, C.c_int]
        L.fp_autotune.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.fp_solve.argtypes = [vp, _dp, C.c_int64, C.POINTER(SolveOpts), C.POINTER(Stats)]
        L.fp_solve_body.argtypes = [vp, C.c_int, C.c_double, C.c_double, _dp, C.c_int64,
                                    C.POINTER(SolveOpts), _dp, C.POINTER(Stats)]
        L.fp_uind.argtypes = [vp, C.c_int, _dp, _dp, C.c_int64, _dp, C.c_int, C.c_double, C.c_double]
        L.fp_phi.argtypes = [vp, C.c_int, _dp, _dp, C.c_int64, _dp, C.c_double]
        L.fp_ugradmu.argtypes = [vp, C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_double, _dp, _dp, _dp]
        L.fp_ugradmu_ex.argtypes = [vp, C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_double, C.c_int, _ip,
                                    C.c_int64, C.c_int, _dp, _dp, _dp]
        L.fp_calcfield_cp.argtypes = [vp, _dp, C.c_double, C.c_int, _dp]
        L.fp_calcfield_f.argtypes = [vp, _dp, _dp, C.c_double, C.c_double, C.c_int, _dp]
        L.fp_calcfield_lds.argtypes = [vp, _dp, _dp, _dp, _dp, _dp]
        L.fp_surface_loads.argtypes = [vp, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double,
                                       C.c_double, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp]
        L.fp_solve_ls.argtypes = [vp, C.c_double, C.c_double, _dp, C.c_int64, C.POINTER(C.c_int64), _dp, _dp,
                                  C.POINTER(Stats)]
        L.fp_adjoint_solve.argtypes = [vp, _dp, C.c_int64, _dp]
        L.fp_lu_solve_noalloc.argtypes = [vp, C.c_void_p, C.c_int64, C.c_int64]
        L.fp_assembly_vjp.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.fp_uind_vjp.argtypes = [vp, _dp, _dp, C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp]
        L.fp_batch_create.argtypes = [C.c_int, C.c_int, C.POINTER(vp)]
        L.fp_batch_destroy.argtypes = [vp]
        L.fp_batch_last_error.argtypes = [vp]
        L.fp_batch_last_error.restype = C.c_char_p
        L.fp_batch_solve.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_int64, C.POINTER(BodyDesc),
                                     C.POINTER(SolveOpts), C.POINTER(Stats)]
        L.fp_trace.argtypes = [vp, C.c_int]
        L.fp_trace_read.argtypes = [vp, C.c_int64, _ip, _ip, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.POINTER(C.c_int64)]
        L.fp_kernel_timing.argtypes = [vp, C.c_int]
        L.fp_kernel_timing_read.argtypes = [vp, C.POINTER(C.c_int64), _dp, _dp, _dp]
        L.fp_last_kernel_ms.argtypes = [vp, C.c_int, _dp, C.POINTER(C.c_int)]
        L.fp_measure_fma_peak.argtypes = [C.c_int, C.c_int, _dp]
        L.fp_kernel_launches.argtypes = [vp, C.POINTER(C.c_int64)]
        L.fp_tc_selftest.argtypes = [C.c_int, C.c_int64, C.c_int64, C.c_int, _dp, _dp, _dp]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _strengths(s):
    """Strengths as the ABI takes them: N values, or N x 2 column-major (all
    sources, then all doublets) for a source+doublet body."""
    s = np.asarray(s, dtype=np.float64)
    return np.ascontiguousarray(s.T).ravel() if s.ndim == 2 else _f64(s)


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def make_opts(solver="ludiv", precision="fp64", ir_tol=1e-12, ir_maxiter=10, gmres_memory=50,
              gmres_atol=-1.0, gmres_rtol=-1.0, gmres_itmax=0, gmres_restart=False):
    """fp_solve_opts. GMRES defaults to the reference's Krylov.jl gmres (no
    restart: gmres_memory only sizes the first basis storage);
    gmres_restart=True gives GMRES(gmres_memory)."""
    return SolveOpts(FP_SOLVER_GMRES if solver == "gmres" else FP_SOLVER_LU,
                     _PRECISIONS[precision], ir_tol, ir_maxiter,
                     gmres_memory, gmres_atol, gmres_rtol, gmres_itmax, 1 if gmres_restart else 0)


class Context:
    """One device context of the library (one CUDA stream)."""

    def __init__(self, device=0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.fp_ctx_create(int(device), C.byref(h))
        if rc:
            raise FlowPanelError(rc, f"fp_ctx_create failed on device {device}")
        self.h = h
        self.N = 0
        self.nsh = 0

    def close(self):
        if getattr(self, "h", None):
            self._L.fp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc:
            raise FlowPanelError(rc, self._L.fp_last_error(self.h).decode())

    def set_geometry(self, nodes, panel_offsets, panel_nodes, cps=None, normals=None, cp_offset=None):
        nodes = _f64(nodes)
        offs = np.ascontiguousarray(panel_offsets, dtype=np.int32)
        pn = np.ascontiguousarray(panel_nodes, dtype=np.int32)
        cps, normals, cp_offset = _f64(cps), _f64(normals), _f64(cp_offset)
        self._chk(self._L.fp_set_geometry(self.h, _d(nodes), nodes.shape[0], _i(offs), _i(pn), len(offs) - 1,
                                          _d(cps), _d(normals), _d(cp_offset)))
        self.N = len(offs) - 1
        self.nsh = 0

    def set_wake(self, shedding, Das, Dbs):
        sh = np.ascontiguousarray(np.reshape(shedding, (-1, 6)), dtype=np.int32)
        Das, Dbs = _f64(np.reshape(Das, (-1, 3))), _f64(np.reshape(Dbs, (-1, 3)))
        self._chk(self._L.fp_set_wake(self.h, _i(sh), sh.shape[0], _d(Das), _d(Dbs)))
        self.nsh = sh.shape[0]

    def assemble(self, element, kerneloffset=1e-8, kernelcutoff=1e-14, precision=FP_PREC_FP64):
        self._chk(self._L.fp_assemble(self.h, element, kerneloffset, kernelcutoff, precision))

    def get_aic(self):
        G = np.empty((self.N, self.N), order="F")
        self._chk(self._L.fp_get_aic(self.h, G.ctypes.data_as(_dp)))
        return G

    def set_rhs(self, Uinfs):
        U = _f64(Uinfs)
        k = U.size // (3 * self.N)
        self._chk(self._L.fp_set_rhs(self.h, _d(U), k))
        return k

    def factor(self, precision=FP_PREC_FP64):
        self._chk(self._L.fp_factor(self.h, precision))

    def solve(self, k=1, opts=None):
        x = np.empty((k, self.N))
        st = Stats()
        self._chk(self._L.fp_solve(self.h, _d(x), k, C.byref(opts) if opts is not None else None, C.byref(st)))
        return (x[0] if k == 1 else x), st

    def solve_device(self, k=1, opts=None):
        """Solve without copying the solution back (it stays in HBM)."""
        st = Stats()
        self._chk(self._L.fp_solve(self.h, None, k, C.byref(opts) if opts is not None else None, C.byref(st)))
        return st

    def solve_body(self, element, Uinfs, kerneloffset=1e-8, kernelcutoff=1e-14, opts=None):
        U = _f64(Uinfs)
        k = U.size // (3 * self.N)
        x = np.empty((k, self.N))
        st = Stats()
        self._chk(self._L.fp_solve_body(self.h, element, kerneloffset, kernelcutoff, _d(U), k,
                                        C.byref(opts) if opts is not None else None, _d(x), C.byref(st)))
        return (x[0] if k == 1 else x), st

    def uind(self, element, strengths, targets, out=None, precision=FP_PREC_FP64, kerneloffset=1e-8,
             kernelcutoff=1e-14):
        targets = _f64(np.reshape(targets, (-1, 3)))
        m = targets.shape[0]
        out = np.zeros((m, 3)) if out is None else np.ascontiguousarray(out, dtype=np.float64)
        self._chk(self._L.fp_uind(self.h, element, _d(_strengths(strengths)), _d(targets), m, _d(out),
                                  precision, kerneloffset, kernelcutoff))
        return out

    def solve_ls(self, Uinfs, elprescribe, kerneloffset=1e-8, kernelcutoff=1e-14):
        """Least-squares solve of a watertight vortex-ring body (fp_solve_ls);
        elprescribe: [(index (0-based), value), ...]. Returns (Gamma, Stats)."""
        U = _f64(np.reshape(Uinfs, (-1, 3)))
        idx = np.ascontiguousarray([int(i) for i, _ in elprescribe], dtype=np.int64)
        val = np.ascontiguousarray([float(v) for _, v in elprescribe], dtype=np.float64)
        x = np.zeros(U.shape[0])
        st = Stats()
        self._chk(self._L.fp_solve_ls(self.h, kerneloffset, kernelcutoff, _d(U), len(idx),
                                      idx.ctypes.data_as(C.POINTER(C.c_int64)), _d(val), _d(x), C.byref(st)))
        return x, st

    def phi(self, element, strengths, targets, out=None, kerneloffset=1e-8):
        """Potential at targets (M, 3) added to out (M,) (fp_phi). strengths: N, or
        (N, 2) (sources, doublets) for FP_ELEMENT_SOURCE_DOUBLET."""
        targets = _f64(np.reshape(targets, (-1, 3)))
        m = targets.shape[0]
        out = np.zeros(m) if out is None else np.ascontiguousarray(out, dtype=np.float64)
        self._chk(self._L.fp_phi(self.h, element, _d(_strengths(strengths)), _d(targets), m, _d(out),
                                 kerneloffset))
        return out

    def ugradmu(self, scheme, strength, cp_offset=None, anglecrit=30.0, force_cellTE=True, maxgrad=np.inf,
                out=None, want_parts=False, sharpTE=False, smooth_cells=None, smooth_pass=0):
        """grad(mu) surface velocity (fp_ugradmu_ex) of the loaded triangular
        body: scheme FP_UGRADMU_COMBINED / _CELL / _NODE; returns out (N, 3),
        with (out, out_cell, out_node) when want_parts (combined scheme only).
        sharpTE: the node scheme's one-sided trailing-edge nodal values;
        smooth_cells / smooth_pass: the cell scheme's smoothRows cells (in
        order) and smoothPass."""
        g = _f64(strength)
        n = g.shape[0]
        out = np.zeros((n, 3)) if out is None else np.ascontiguousarray(out, dtype=np.float64)
        oc = np.zeros((n, 3)) if want_parts else None
        on = np.zeros((n, 3)) if want_parts else None
        sc = np.ascontiguousarray(np.zeros(0) if smooth_cells is None else smooth_cells, dtype=np.int32)
        self._chk(self._L.fp_ugradmu_ex(self.h, scheme, _d(g), _d(_f64(cp_offset)), float(anglecrit),
                                        int(bool(force_cellTE)), float(maxgrad), int(bool(sharpTE)),
                                        sc.ctypes.data_as(_ip) if sc.size else None, int(sc.size),
                                        int(smooth_pass), _d(out), _d(oc), _d(on)))
        return (out, oc, on) if want_parts else out

    def calcfield_cp(self, Us, Uref, correct_kutta=True, out=None):
        Us = _f64(np.reshape(Us, (-1, 3)))
        out = np.zeros(Us.shape[0]) if out is None else np.ascontiguousarray(out, dtype=np.float64)
        self._chk(self._L.fp_calcfield_cp(self.h, _d(Us), float(Uref), int(bool(correct_kutta)), _d(out)))
        return out

    def calcfield_f(self, Cps, Uinf, rho, cp_offset=None, correct_kutta=True, out=None):
        Cps = _f64(Cps)
        out = np.zeros((Cps.shape[0], 3)) if out is None else np.ascontiguousarray(out, dtype=np.float64)
        self._chk(self._L.fp_calcfield_f(self.h, _d(Cps), _d(_f64(cp_offset)), float(Uinf), float(rho),
                                         int(bool(correct_kutta)), _d(out)))
        return out

    def calcfield_lds(self, Fs, Lhat, Dhat, Shat, out=None):
        """Returns the 3 x 3 matrix of lift, drag and sideslip vectors (columns)."""
        Fs = _f64(np.reshape(Fs, (-1, 3)))
        o = np.zeros(9) if out is None else np.ascontiguousarray(np.asarray(out, float).T).ravel()
        self._chk(self._L.fp_calcfield_lds(self.h, _d(Fs), _d(_f64(Lhat)), _d(_f64(Dhat)), _d(_f64(Shat)),
                                           _d(o)))
        return o.reshape(3, 3).T.copy()

    def surface_loads(self, element, strengths, Uinfs, Uref, rho, Lhat, Dhat, Shat, cp_offset=None,
                      kerneloffset=1e-8, kernelcutoff=1e-14, ugradmu=True, correct_kutta=True, want_U=True):
        """fp_surface_loads: (U, Cp, F, LDS) of the solved body."""
        U0 = _f64(np.reshape(Uinfs, (-1, 3)))
        n = U0.shape[0]
        U = np.empty((n, 3)) if want_U else None
        Cp = np.empty(n)
        F = np.empty((n, 3))
        lds = np.empty(9)
        self._chk(self._L.fp_surface_loads(self.h, element, _d(_strengths(strengths)), _d(U0), _d(_f64(cp_offset)),
                                           kerneloffset, kernelcutoff, int(bool(ugradmu)), float(Uref), float(rho),
                                           _d(_f64(Lhat)), _d(_f64(Dhat)), _d(_f64(Shat)),
                                           int(bool(correct_kutta)), _d(U), _d(Cp), _d(F), _d(lds)))
        return U, Cp, F, lds.reshape(3, 3).T.copy()

    def adjoint_solve(self, ybar):
        ybar = _f64(np.atleast_2d(ybar))
        lam = np.empty_like(ybar)
        self._chk(self._L.fp_adjoint_solve(self.h, _d(ybar), ybar.shape[0], _d(lam)))
        return lam

    def assembly_vjp(self, Uinfs, nnodes, lam=None, gamma=None):
        """Gradient of lambda^T (b - A Gamma) (see fp_assembly_vjp); lam / gamma
        None use the device-resident adjoint / primal solutions. Returns a dict
        of dnodes (nnodes, 3), dcps, dnormals, dUinfs (N, 3), dDas, dDbs (nsh, 3)."""
        n = self.N
        U = _f64(np.reshape(Uinfs, (n, 3)))
        nsh = self.nsh
        out = {"dnodes": np.zeros((nnodes, 3)), "dcps": np.zeros((n, 3)), "dnormals": np.zeros((n, 3)),
               "dUinfs": np.zeros((n, 3)), "dDas": np.zeros((max(nsh, 1), 3)), "dDbs": np.zeros((max(nsh, 1), 3))}
        self._chk(self._L.fp_assembly_vjp(self.h, _d(_f64(lam)), _d(_f64(gamma)), _d(U), _d(out["dnodes"]),
                                          _d(out["dcps"]), _d(out["dnormals"]), _d(out["dUinfs"]),
                                          _d(out["dDas"]), _d(out["dDbs"])))
        out["dDas"], out["dDbs"] = out["dDas"][:nsh], out["dDbs"][:nsh]
        return out

    def uind_vjp(self, strengths, targets, wbar, nnodes):
        """Gradient of sum_i wbar_i . Uind(targets_i) (see fp_uind_vjp)."""
        X = _f64(np.reshape(targets, (-1, 3)))
        W = _f64(np.reshape(wbar, (-1, 3)))
        m = X.shape[0]
        nsh = self.nsh
        out = {"dtargets": np.zeros((m, 3)), "dstrengths": np.zeros(self.N), "dnodes": np.zeros((nnodes, 3)),
               "dDas": np.zeros((max(nsh, 1), 3)), "dDbs": np.zeros((max(nsh, 1), 3))}
        self._chk(self._L.fp_uind_vjp(self.h, _d(_f64(strengths)), _d(X), m, _d(W), _d(out["dtargets"]),
                                      _d(out["dstrengths"]), _d(out["dnodes"]), _d(out["dDas"]), _d(out["dDbs"])))
        out["dDas"], out["dDbs"] = out["dDas"][:nsh], out["dDbs"][:nsh]
        return out

    def lu_solve_noalloc(self, dev_ptr, ldb, k=1):
        """In-place FP64 solve of the N x k column-major device array at
        ``dev_ptr`` (an integer address on this context's device) with the
        factors of the last ``factor(FP_PREC_FP64)``; the library allocates
        no device memory for it."""
        self._chk(self._L.fp_lu_solve_noalloc(self.h, C.c_void_p(dev_ptr), ldb, k))

    def trace(self, enable=True):
        """Record a timeline of the next factorisations (fp_trace)."""
        self._chk(self._L.fp_trace(self.h, 1 if enable else 0))

    def trace_read(self):
        """(tags, streams, t0_ms, t1_ms) of the last traced factorisation."""
        n = C.c_int64()
        self._chk(self._L.fp_trace_read(self.h, 0, None, None, None, None, C.byref(n)))
        k = n.value
        tags, streams = np.zeros(k, np.int32), np.zeros(k, np.int32)
        t0, t1 = np.zeros(k, np.float32), np.zeros(k, np.float32)
        self._chk(self._L.fp_trace_read(self.h, k, _i(tags), _i(streams), t0.ctypes.data_as(C.POINTER(C.c_float)),
                                        t1.ctypes.data_as(C.POINTER(C.c_float)), C.byref(n)))
        return tags, streams, t0, t1

    def autotune(self, precision, reps=2):
        """fp_autotune: pick the fastest factorisation knobs for the assembled
        AIC (cached per size and precision); returns the 10 knob values."""
        out = (C.c_int * 10)()
        self._chk(self._L.fp_autotune(self.h, int(precision), int(reps), out))
        return list(out)

    def set_tuning(self, knob, value):
        """fp_set_tuning: one of the FP_TUNE_* knobs (include/flowpanel_b200.h)."""
        self._chk(self._L.fp_set_tuning(self.h, int(knob), int(value)))

    def kernel_timing(self, enable=True):
        """Per-launch event timing of the factorisation's trailing update."""
        self._chk(self._L.fp_kernel_timing(self.h, 1 if enable else 0))

    def kernel_timing_read(self):
        n, ms, fl, el = C.c_int64(), C.c_double(), C.c_double(), C.c_double()
        self._chk(self._L.fp_kernel_timing_read(self.h, C.byref(n), C.byref(ms), C.byref(fl), C.byref(el)))
        return n.value, ms.value, fl.value, el.value

    def kernel_launches(self):
        n = C.c_int64()
        self._chk(self._L.fp_kernel_launches(self.h, C.byref(n)))
        return n.value

    def last_kernel_ms(self, stage):
        ms = C.c_double()
        n = C.c_int()
        self._chk(self._L.fp_last_kernel_ms(self.h, stage, C.byref(ms), C.byref(n)))
        return ms.value, n.value


def measure_fma_peak(device=0, fp64=True, tensor=False):
    """Sustained FMA throughput (TFLOP/s) of the FP64 or FP32 pipe, or with
    ``tensor`` of the FP64 tensor path (mma.sync m8n8k4 .f64)."""
    t = C.c_double()
    rc = lib().fp_measure_fma_peak(int(device), 2 if tensor else (1 if fp64 else 0), C.byref(t))
    if rc:
        raise FlowPanelError(rc, "fp_measure_fma_peak failed")
    return t.value


def tc_selftest(m, n, k, device=0):
    """(err_tc, err_simt, ms_tc) of the tensor-core FP32 update against FP64 (see the header)."""
    a, b, t = C.c_double(), C.c_double(), C.c_double()
    rc = lib().fp_tc_selftest(int(device), int(m), int(n), int(k), C.byref(a), C.byref(b), C.byref(t))
    if rc:
        raise FlowPanelError(rc, "fp_tc_selftest failed")
    return a.value, b.value, t.value


class Batch:
    """nslots device contexts solving many bodies concurrently (fp_batch_*)."""

    def __init__(self, device=0, nslots=4):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.fp_batch_create(int(device), int(nslots), C.byref(h))
        if rc:
            raise FlowPanelError(rc, f"fp_batch_create failed on device {device}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self._L.fp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, element, problems, kerneloffset=1e-8, kernelcutoff=1e-14, opts=None):
        """problems: list of dicts with nodes, panel_offsets, panel_nodes, Uinfs (N, 3)
        and optionally cps, normals, shedding, Das, Dbs. Returns (strengths list, stats list)."""
        keep, descs, outs = [], [], []
        for p in problems:
            nodes = _f64(p["nodes"])
            offs = np.ascontiguousarray(p["panel_offsets"], dtype=np.int32)
            pn = np.ascontiguousarray(p["panel_nodes"], dtype=np.int32)
            n = len(offs) - 1
            U = _f64(np.reshape(p["Uinfs"], (n, 3)))
            cps, normals = _f64(p.get("cps")), _f64(p.get("normals"))
            sh = p.get("shedding")
            sh = np.ascontiguousarray(np.reshape(sh, (-1, 6)), dtype=np.int32) if sh is not None else None
            Da = _f64(np.reshape(p["Das"], (-1, 3))) if p.get("Das") is not None else None
            Db = _f64(np.reshape(p["Dbs"], (-1, 3))) if p.get("Dbs") is not None else None
            x = np.zeros(n)
            keep.append((nodes, offs, pn, U, cps, normals, sh, Da, Db, x))
            outs.append(x)
            descs.append(BodyDesc(_d(nodes), nodes.shape[0], _i(offs), _i(pn), n, _d(cps), _d(normals), _i(sh),
                                  0 if sh is None else sh.shape[0], _d(Da), _d(Db), _d(U), _d(x)))
        arr = (BodyDesc * len(descs))(*descs)
        st = (Stats * len(descs))()
        rc = self._L.fp_batch_solve(self.h, element, kerneloffset, kernelcutoff, len(descs), arr,
                                    C.byref(opts) if opts is not None else None, st)
        if rc:
            raise FlowPanelError(rc, self._L.fp_batch_last_error(self.h).decode())
        return outs, [s.asdict() for s in st]
