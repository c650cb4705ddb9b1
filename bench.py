#!/usr/bin/env python
"""Benchmark: 12k-panel swept-wing solve on B200, mixed precision vs plain FP64.

Workload (one "step"): the 12,000-panel NACA 0012 swept wing (100 chordwise x
120 spanwise quads, 45 deg sweep, AR 5, rigid wake, AoA 4.2 deg) solved end to
end on the device: AIC assembly + factorisation + solve (mixed: FP32 factors,
3xTF32 tensor-core update, FP64 refinement to ||r||/||b|| <= 1e-12).

  value   device ms per mixed-precision solve, inputs (mesh, RHS) resident in HBM
  e2e     the same through fp_solve_body with host buffers (H2D of Uinfs, D2H of Gamma)
  extras  FP64 plain-solve ms, the ratio, |dCL| of mixed vs FP64, per-stage times

The reference arm (--impl reference) times the CPU restatement of the
reference solve (OpenMP assembly as in the reference's threaded loop, LAPACK
LU via scipy) on the host cores, on the same configuration.

Run: python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU runs are replicas (the dense solve does not shard): every rank
solves its own wing; value = slowest rank's ms per step / N.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

METRIC = "12k-panel wing solve ms, mixed vs FP64 on B200 at |dCL|<=1e-7; adjoint/primal"
N_CHORD, N_SPAN, AOA = 100, 120, 4.2
B_SPAN, AR = 5.0, 5.0   # span and aspect ratio b/c_tip (chord 1)


def wing_problem(fp, n_chord=N_CHORD, n_span=N_SPAN):
    w = fp.meshes.swept_wing("0012", n_chord, n_span, 1.0, B_SPAN, 45.0, 1.0)
    body = fp.RigidWakeBody(w)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(AOA)
    V = np.array([np.cos(a), 0.0, np.sin(a)])
    D = np.tile(V, (w.nsheddings, 1))
    U = np.tile(V, (w.npanels, 1))
    return w, body, normals, cps, V, D, U


def lift_coefficient(fp, body, gamma, V, Uinfs, D, solver, chord=B_SPAN / AR, sref=B_SPAN ** 2 / AR,
                     with_drag=False):
    """CL as test/runtests_solvers.jl:146-166: probes 0.02*c off the surface,
    Cp with the Kutta average, F = -Cp q A n, L projected on cross(D, S);
    with_drag also returns CD and the Cp field."""
    body.strength = gamma
    body.solved = True
    body.add_field("Uinf", "vector", Uinfs, "cell")
    body.add_field("Da", "vector", D, "system")
    body.add_field("Db", "vector", D, "system")
    fp.calcfield_U(body, body, offset=0.02, characteristiclength=lambda *a: chord,
                   fieldname="Uoff", solver=solver)
    Cp = fp.calcfield_Cp(body, 1.0, U_fieldname="Uoff")
    fp.calcfield_F(body, 1.0, 1.225)
    Dhat = V / np.linalg.norm(V)
    Shat = np.array([0.0, 1.0, 0.0])
    Lhat = np.cross(Dhat, Shat)
    LDS = fp.calcfield_LDS(body, Lhat, Dhat)
    nondim = 0.5 * 1.225 * 1.0 * sref
    L, Dr = LDS[:, 0], LDS[:, 1]
    CL = float(np.sign(np.dot(L, Lhat)) * np.linalg.norm(L) / nondim)
    if not with_drag:
        return CL
    CD = float(np.sign(np.dot(Dr, Dhat)) * np.linalg.norm(Dr) / nondim)
    return CL, CD, np.array(Cp, copy=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def batch_throughput(fp, device, nwings=64, nslots=8, reps=2):
    """Config 3b: 64 wings drawn from default_rng(0) (sweep U[0,45], AR U[4,10],
    taper U[0.3,1], tip twist U[-4,0], 2k-8k panels), mixed precision, solved
    by fp_batch_solve with nslots device contexts against the same solves
    one at a time (one slot). Wall time of the whole batch, host set-up
    included. Returns a dict."""
    cap = fp._capi
    wings, params = fp.meshes.random_wings(nwings, seed=0)
    bodies = [fp.RigidWakeBody(w) for w in wings]
    V = np.array([np.cos(np.deg2rad(AOA)), 0.0, np.sin(np.deg2rad(AOA))])
    Us = [np.tile(V, (b.ncells, 1)) for b in bodies]
    Ds = [np.tile(V, (b.nsheddings, 1)) for b in bodies]
    out = {"config": f"{nwings} wings from default_rng(0), {min(b.ncells for b in bodies)}-"
                     f"{max(b.ncells for b in bodies)} panels ({sum(b.ncells for b in bodies)} total), mixed",
           "nslots": nslots}
    for label, slots in (("sequential", 1), ("batched", nslots)):
        batch = cap.Batch(device, slots)
        fp.solve_batch(bodies, Us, Ds, Ds, precision="mixed", batch=batch)   # warm-up, buffers sized
        best = 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            fp.solve_batch(bodies, Us, Ds, Ds, precision="mixed", batch=batch)
            best = min(best, time.perf_counter() - t0)
        batch.close()
        out[f"{label}_s"] = best
        out[f"{label}_wings_per_s"] = nwings / best
    out["speedup"] = out["sequential_s"] / out["batched_s"]
    return out


def surface_loads_timing(fp, reps=5):
    """The post-processing of the reference's examples on the triangulated
    12k wing (100 x 60 quads split in 12,000 triangles, the reference's cell
    type): U at the control points, + grad(mu), Cp with the Kutta average, F
    and L/D/S in one fp_surface_loads call. Device time of the call's
    kernels (median of reps) and the induced-velocity share of it."""
    cap = fp._capi
    m = fp.meshes.triangulate(fp.meshes.swept_wing("0012", N_CHORD, N_SPAN // 2, chord=1.0, b=B_SPAN, sweep=45.0))
    body = fp.RigidWakeBody(m)
    V = np.array([np.cos(np.deg2rad(AOA)), 0.0, np.sin(np.deg2rad(AOA))])
    D = np.tile(V, (m.nsheddings, 1))
    solver = fp.B200Solver(precision="mixed")
    fp.solve(body, np.tile(V, (m.npanels, 1)), D, D, solver=solver)
    Shat = np.array([0.0, 1.0, 0.0])
    Lhat = np.cross(V, Shat)
    ms, ug = [], []
    for k in range(reps + 2):
        fp.surface_loads(body, 1.0, 1.225, Lhat, V, Shat, solver=solver)
        t, launches = solver.ctx.last_kernel_ms(cap.FP_STAGE_POST)
        solver.ctx.ugradmu(cap.FP_UGRADMU_COMBINED, body.strength, None)
        if k >= 2:
            ms.append(t)
            ug.append(solver.ctx.last_kernel_ms(cap.FP_STAGE_POST)[0])
    solver.close()
    return {"config": f"triangulated swept wing, {m.npanels} triangles, {m.nsheddings} shedding edges",
            "surface_loads_ms": float(np.median(ms)), "launches": launches,
            "ugradmu_ms": float(np.median(ug))}


TRACE_TAGS = {0: "diagonal block", 1: "L21 (rows below)", 2: "U12 (next panel)", 3: "U12 (columns beyond)",
              4: "tcgen05 update", 5: "split A", 6: "split B", 7: "SIMT update", 8: "panel inverses"}


def factor_timeline(ctx, cap, prec):
    """One traced factorisation (outside the timed region): per kernel tag and
    stream, launches and summed device time, and each stream's busy time.
    Stream 0 carries the panel chain (the critical path)."""
    ctx.trace(True)
    ctx.factor(prec)
    ctx.trace(False)
    tags, streams, t0, t1 = ctx.trace_read()
    out = {"span_ms": float(t1.max() - t0.min()) if len(t0) else 0.0, "kernels": []}
    for s in (0, 1, 2, 3):
        sel = streams == s
        if s >= 2 and not sel.any():
            continue
        out[f"stream{s}_busy_ms"] = float(np.sum(t1[sel] - t0[sel]))
        for tg in sorted(set(tags[sel].tolist())):
            m = sel & (tags == tg)
            out["kernels"].append({"stream": s, "kernel": TRACE_TAGS.get(int(tg), str(tg)),
                                   "launches": int(m.sum()), "ms": float(np.sum(t1[m] - t0[m])),
                                   "avg_us": float(1e3 * np.mean(t1[m] - t0[m]))})
    return out


def cusolver_reference(n, reps=3):
    """cuSOLVER getrf on the same box through torch.linalg.lu_factor (the
    library LU the reference's CuArray path calls, src/FLOWPanel_linearsolver.jl:73,179),
    on a diagonally weighted random matrix of the wing's size: a comparison
    line for the hand-written factorisations, not part of the product."""
    import torch
    out = {}
    g = torch.Generator(device="cuda").manual_seed(0)
    for name, dt in (("dgetrf_fp64", torch.float64), ("sgetrf_fp32", torch.float32)):
        A = torch.rand((n, n), generator=g, device="cuda", dtype=dt) + n * torch.eye(n, device="cuda", dtype=dt)
        torch.linalg.lu_factor(A.clone())
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            B = A.clone()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.linalg.lu_factor(B)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        out[name + "_ms"] = float(np.median(ms))
        del A, B
    torch.cuda.empty_cache()
    out["n"] = n
    out["how"] = "torch.linalg.lu_factor (cuSOLVER getrf, partial pivoting), CUDA events, median of 3"
    return out


def least_squares_timing(fp, device, reps=3):
    """Least squares of a watertight lifting body (RigidWakeBody{VortexRing, 2},
    the reference's duct: NACA 66-2015 ring wing re-discretised with 10 cells a
    section per surface and revolved in 60 and in 120 azimuthal steps, 7,200 and
    14,400 triangles): device ms of fp_solve_ls (assembly, then the prescribed
    strength folded into the right-hand side, the FP64 Gram matrix of the
    reduced AIC, its LU and the solve), median of reps; the Gram product's
    share and rate (N^3 flops for the symmetric N x N product)."""
    cap = fp._capi
    c = np.load(os.path.join(ROOT, "tests", "golden", "airfoils.npz"))["naca662015"]
    nd = [(0.25, 10, 10.0, False), (0.50, 10, 1.0, True), (0.25, 10, 0.1, False)]
    S = fp.meshes.rediscretize_airfoil(c[:, 0], c[:, 1], nd, nd)
    S = np.concatenate([S, S[:1]])
    d, ar = 2 * 0.835, 0.6
    P = S * d * ar
    P[:, 1] += d / 2
    a = np.deg2rad(5.0)
    V = np.array([np.cos(a), 0.0, np.sin(a)])
    out = {"config": "duct (test/runtests_solvers2.jl), NACA 66-2015 ring wing, least squares, FP64", "cases": []}
    for ntheta in (60, 120):
        m = fp.meshes.revolution_liftbody(P, ntheta, name="duct", CPoffset=1e-14)
        body = fp.RigidWakeBody(m, watertight=True, CPoffset=1e-14, characteristiclength=lambda *x: d * ar)
        normals = fp.calc_normals(body)
        cps = fp.calc_controlpoints(body, normals)
        ctx = cap.Context(device)
        ctx.set_geometry(m.nodes, m.panel_offsets, m.panel_nodes, cps, normals)
        D = np.tile(V, (m.nsheddings, 1))
        ctx.set_wake(m.shedding, D, D)
        U = np.tile(V, (m.npanels, 1))
        ms = []
        for r in range(reps + 1):
            x, st = ctx.solve_ls(U, [(0, 0.0)])
            if r > 0:
                ms.append(st.ms_assemble + st.ms_factor)
        ctx.close()
        n = m.npanels
        out["cases"].append({"n_panels": n, "ms": float(np.median(ms)),
                             "gram_gflop": float(n) ** 3 / 1e9})
    return out


def potential_timing(fp, device, nprobes=100_000, reps=3):
    """Potential of the solved 12k wing (doublet panels and the wake's
    semi-infinite doublets, fp_phi) at nprobes points uniform in a box around
    it: device ms of the kernel (FP_STAGE_PHI), median of reps."""
    cap = fp._capi
    w, body, normals, cps, V, D, U = wing_problem(fp)
    ctx = cap.Context(device)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    x, _ = ctx.solve_body(cap.FP_ELEMENT_VORTEXRING, U, opts=cap.make_opts("ludiv", "fp64"))
    rng = np.random.default_rng(3)
    lo, hi = w.nodes.min(axis=0) - 0.5, w.nodes.max(axis=0) + 0.5
    T = lo + (hi - lo) * rng.random((nprobes, 3))
    ms = []
    for r in range(reps + 1):
        ctx.phi(cap.FP_ELEMENT_VORTEXRING, x, T)
        if r > 0:
            ms.append(ctx.last_kernel_ms(cap.FP_STAGE_PHI)[0])
    ctx.close()
    return {"config": f"12k wing doublets + wake, {nprobes} probes in its bounding box + 0.5 m, FP64",
            "ms": float(np.median(ms)), "probes_per_s": nprobes / (float(np.median(ms)) * 1e-3)}


def sphere_timing(fp, device, reps=5):
    """Config 1: the 1,800-panel source sphere (30 x 60 cells, pole rows as
    triangles), FP64 assembly + LU + solve through fp_solve_body, device ms."""
    cap = fp._capi
    s = fp.meshes.sphere(1.0, 30, 60)
    body = fp.NonLiftingBody(s)
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    U = np.tile([1.0, 0.0, 0.0], (s.npanels, 1))
    ctx = cap.Context(device)
    ctx.set_geometry(s.nodes, s.panel_offsets, s.panel_nodes, cps, normals)
    ms = []
    for i in range(reps + 2):
        _, st = ctx.solve_body(cap.FP_ELEMENT_SOURCE, U, opts=cap.make_opts("ludiv", "fp64"))
        if i >= 2:
            ms.append(st.ms_assemble + st.ms_factor + st.ms_solve)
    ctx.close()
    return {"config": f"sphere R=1, 30x60 cells = {s.npanels} source panels, FP64", "ms_per_solve": float(np.median(ms)),
            "solves_per_s": 1e3 / float(np.median(ms))}


def aoa_sweep_timing(ctx, cap, w, normals, opts, reps=3):
    """Config 3a: the 12k wing at AoA -10..+10 deg in 1 deg steps, 21
    right-hand sides on one factorisation (fixed wake), mixed: assembly +
    factorisation + refinement of all 21, device ms."""
    aoas = np.arange(-10.0, 10.5, 1.0)
    Us = np.stack([np.tile([np.cos(np.deg2rad(a)), 0.0, np.sin(np.deg2rad(a))], (w.npanels, 1)) for a in aoas])
    ms = []
    for i in range(reps + 1):
        ctx.assemble(cap.FP_ELEMENT_VORTEXRING, 1e-8, 1e-14, cap.FP_PREC_MIXED)
        ctx.set_rhs(Us)
        ctx.factor(cap.FP_PREC_MIXED)
        st = ctx.solve_device(len(aoas), opts)
        if i >= 1:
            ms.append(st.ms_assemble + st.ms_factor + st.ms_solve)
    return {"config": f"12k wing, {len(aoas)} AoA right-hand sides (-10..+10 deg) on one factorisation, mixed",
            "ms": float(np.median(ms)), "ms_per_rhs": float(np.median(ms)) / len(aoas),
            "ir_iters": st.ir_iters, "rel_residual": st.rel_residual}


def measured_peak(key, fallback):
    """A peak from MEASURED_PEAKS.json (driver-measured on this pool), else
    the stated fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)[key]), f"of measured ({key}, MEASURED_PEAKS.json)"
    except Exception:
        return fallback, "of fallback"


def profile_traffic(kernel):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per updated
    output element of `kernel`, from the committed ncu summary
    profiles/<kernel>*.txt (a line 'traffic_bytes_per_C_element: <bytes>');
    the bench scales it to its own average launch (traffic grows with the
    m x n elements each launch updates)."""
    d = os.path.join(ROOT, "profiles")
    try:
        for name in sorted(os.listdir(d)):
            if name.startswith(kernel) and name.endswith(".txt"):
                with open(os.path.join(d, name)) as fh:
                    for line in fh:
                        if line.startswith("traffic_bytes_per_C_element:"):
                            return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import datetime

    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, ws, dist


def max_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_reference_solve(fp, O, nthreads, sample="full"):
    """One reference solve on the host: OpenMP assembly (threads over panels,
    src/FLOWPanel_liftingbody.jl:476-478) + LAPACK LU + solve. Returns ms."""
    w, body, normals, cps, V, D, U = wing_problem(fp)
    t0 = time.perf_counter()
    G = O.assemble_vortexring(w, cps, normals, D, D, nthreads=nthreads)
    b = O.rhs_noflowthrough(U, normals)
    x = O.solve_ludiv(G, b)
    t1 = time.perf_counter()
    return (t1 - t0) * 1e3, x


def run_reference(args, rank, ws, dist):
    if rank != 0:
        return
    fp = ge.load_package()
    O = ge.load_oracle()
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    times = []
    for i in range(args.warmup + args.steps):
        ms, _ = cpu_reference_solve(fp, O, ncores)
        if i >= args.warmup:
            times.append(ms)
    v = float(np.mean(times))
    line = {"metric": METRIC, "value": v, "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"swept wing NACA0012 {N_CHORD}x{N_SPAN}=12000 vortex-ring panels, "
                                   "rigid wake, AoA 4.2, FP64 assembly + LAPACK LU", "n_panels": 12000},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "ms", "cores": ncores, "kind": "port",
                             "sample": "full 12k-panel solve per step (assembly + dgetrf + dgetrs)"},
            "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, ws, dist):
    fp = ge.load_package()
    cap = fp._capi
    device = int(os.environ.get("LOCAL_RANK", "0"))
    w, body, normals, cps, V, D, U = wing_problem(fp, args.n_chord, args.n_span)
    N = w.npanels
    ctx = cap.Context(device)
    ctx.set_geometry(w.nodes, w.panel_offsets, w.panel_nodes, cps, normals)
    ctx.set_wake(w.shedding, D, D)
    ctx.set_rhs(U)
    VR = cap.FP_ELEMENT_VORTEXRING
    opts = {p: cap.make_opts("ludiv", p) for p in ("fp64", "mixed")}

    def device_step(prec):
        p = cap.FP_PREC_MIXED if prec == "mixed" else cap.FP_PREC_FP64
        ctx.assemble(VR, 1e-8, 1e-14, p)
        ctx.factor(p)
        st = ctx.solve_device(1, opts[prec])
        return st.ms_assemble + st.ms_factor + st.ms_solve, st

    # warm-up
    for _ in range(args.warmup):
        for prec in (("mixed", "fp64") if args.precision == "both" else (args.precision,)):
            device_step(prec)
    launches0 = ctx.kernel_launches()
    res = {}
    precs = ("mixed", "fp64") if args.precision == "both" else (args.precision,)
    ktime = {}
    with ClockSampler(device) as clk:
        for prec in precs:
            barrier(dist)
            tot, stages = 0.0, np.zeros(3)
            for _ in range(args.steps):
                ms, st = device_step(prec)
                tot += ms
                stages += [st.ms_assemble, st.ms_factor, st.ms_solve]
            res[prec] = (max_over_ranks(dist, tot / args.steps), stages / args.steps, st)
    launches = ctx.kernel_launches() - launches0
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "launches": launches,
                              **{p: {"ms": res[p][0], "stages": res[p][1].tolist(), "ir_iters": res[p][2].ir_iters}
                                 for p in res}}), flush=True)
        ctx.close()
        return
    ms_mixed, stg_m, st_m = res["mixed"]
    ms_fp64, stg_d, st_d = res["fp64"]
    # per-launch device times of the trailing update (roofline), from one more
    # step of each form with the launch events on, outside the timed region
    # (the events themselves cost the factorisation about 0.5 ms)
    for prec in precs:
        ctx.kernel_timing(True)
        device_step(prec)
        ktime[prec] = ctx.kernel_timing_read()
        ctx.kernel_timing(False)

    # adjoint of each form: A^T lambda = ybar on the saved factors + the
    # reverse-mode assembly (gradient w.r.t. nodes, CPs, normals, Uinf, wake)
    ybar = np.random.default_rng(7).standard_normal(N)
    adj = {}
    for prec in ("mixed", "fp64"):
        device_step(prec)
        a_ms = v_ms = 0.0
        for i in range(args.warmup + args.steps):
            ctx.adjoint_solve(ybar[None, :])
            ctx.assembly_vjp(U, w.nodes.shape[0])
            if i >= args.warmup:
                a_ms += ctx.last_kernel_ms(cap.FP_STAGE_ADJOINT)[0]
                v_ms += ctx.last_kernel_ms(cap.FP_STAGE_VJP)[0]
        adj[prec] = (max_over_ranks(dist, a_ms / args.steps), max_over_ranks(dist, v_ms / args.steps))

    # e2e through the public C ABI with host buffers
    e2e = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        x_m, st = ctx.solve_body(VR, U, opts=opts["mixed"])
        t1 = time.perf_counter()
        if i >= args.warmup:
            e2e.append((t1 - t0) * 1e3)
    e2e_ms = max_over_ranks(dist, float(np.mean(e2e)))
    x_d, _ = ctx.solve_body(VR, U, opts=opts["fp64"])

    if rank != 0:
        ctx.close()
        return
    # the mixed factorisation's timeline (one traced run, outside the timed region)
    ctx.assemble(VR, 1e-8, 1e-14, cap.FP_PREC_MIXED)
    timeline = factor_timeline(ctx, cap, cap.FP_PREC_MIXED)
    # config 3a: 21 AoA right-hand sides on one factorisation
    aoa = aoa_sweep_timing(ctx, cap, w, normals, opts["mixed"])
    ctx.set_rhs(U)
    # config 1: the 1,800-panel source sphere
    sphere = sphere_timing(fp, device)
    # the least-squares solve of watertight bodies and the potential field
    lsq = least_squares_timing(fp, device)
    pot = potential_timing(fp, device)
    # cuSOLVER getrf of the same size, for comparison with the hand-written LUs
    try:
        cusolver = cusolver_reference(N)
    except Exception as e:   # torch without CUDA: no comparison line
        cusolver = {"unavailable": str(e)[:200]}
    # accuracy gate: CL of the mixed and FP64 strengths (same post-processing)
    solver = fp.B200Solver("ludiv", "fp64", device=device)
    CLm = lift_coefficient(fp, body, x_m, V, U, D, solver)
    CLd = lift_coefficient(fp, body, x_d, V, U, D, solver)
    rel_gamma = float(np.linalg.norm(x_m - x_d) / np.linalg.norm(x_d))
    # roofline of the dominant kernel of the mixed solve, the tcgen05 3xTF32
    # trailing update: algorithmic flops (2 m n k per launch) over its summed
    # per-launch device time in the timed region
    tc_launches, tc_ms, tc_flops, tc_elems = ktime["mixed"]
    tc_tflops = tc_flops / (tc_ms * 1e-3) / 1e12 if tc_ms > 0 else 0.0
    peak_tc, peak_src = measured_peak("bf16_tflops", 1590.0)
    peak_hbm, hbm_src = measured_peak("hbm_gbs", 6650.0)
    per_elem = profile_traffic("k_tc_gemm_sub")   # DRAM bytes per updated C element, from ncu
    traffic = per_elem * tc_elems / tc_launches if (per_elem and tc_launches) else None
    # with K = 128 the update does 2 x 128 flops per C element against 8 bytes
    # of C read-modify-write (32 flop/B), under the ridge point of its BF16
    # pairs (bf16 peak / 3 MMAs a flop over HBM, ~86 flop/B): HBM is the bound
    # that applies
    tc_gbs = 8.0 * tc_elems / (tc_ms * 1e-3) / 1e9 if tc_ms > 0 else 0.0
    # the critical path: the panel chain on stream 0, led by the diagonal
    # block (one CTA, dependent elimination steps)
    diag = next((k for k in timeline["kernels"] if k["stream"] == 0 and k["kernel"] == "diagonal block"), None)
    peak32 = cap.measure_fma_peak(device, False)
    # FP64 pipe roofline of the assembly: ops pinned by the oracle's operation
    # counter (248 per quad-ring interaction, 290 per horseshoe) / device time
    peak64 = cap.measure_fma_peak(device, True)
    peak_dmma = cap.measure_fma_peak(device, True, tensor=True)
    ops = 248.0 * N * N + 290.0 * 2 * w.nsheddings * N
    achieved = ops / (stg_d[0] * 1e-3) / 1e12
    d_launches, d_ms, d_flops, _ = ktime["fp64"]
    batched = batch_throughput(fp, device) if not args.no_batch else None
    post = surface_loads_timing(fp)
    wingbody = None if args.no_wingbody else wingbody_measure(fp, device, steps=2, warmup=1,
                                                              cpu=not args.no_cpu_baseline)
    cpu = None
    if not args.no_cpu_baseline:
        O = ge.load_oracle()
        ncores = os.cpu_count() or 1
        ms_cpu, x_cpu = cpu_reference_solve(fp, O, ncores)
        cpu = {"value": ms_cpu, "unit": "ms", "cores": ncores, "kind": "port",
               "sample": "one full 12k-panel solve (OpenMP assembly + LAPACK dgetrf/dgetrs)",
               "rel_diff_fp64_vs_cpu": float(np.linalg.norm(x_d - x_cpu) / np.linalg.norm(x_cpu))}
    line = {"metric": METRIC, "value": ms_mixed * 1.0 / ws if ws > 1 else ms_mixed, "unit": "ms",
            "value_definition": ("device ms per mixed solve" if ws == 1 else
                                 f"whole-job ms per mixed solve: the slowest rank's ms per step / {ws} ranks, "
                                 "each rank solving its own wing per step (replicas)"),
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic",
            "config": {"workload": f"swept wing NACA0012 {N_CHORD}x{N_SPAN}=12000 vortex-ring panels, "
                                   "rigid wake, AoA 4.2; mixed: FP64 assembly, FP32 LU, FP64 IR to 1e-12",
                       "n_panels": N, "l2": "inputs larger than L2 (AIC 1.15 GB FP64)",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
            "fp64_ms_per_solve": ms_fp64, "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed,
            "stages_ms": {"mixed": dict(zip(("assemble", "factor", "solve"), stg_m.tolist())),
                          "fp64": dict(zip(("assemble", "factor", "solve"), stg_d.tolist()))},
            "accuracy": {"CL_mixed": CLm, "CL_fp64": CLd, "abs_dCL": abs(CLm - CLd),
                         "rel_gamma_mixed_vs_fp64": rel_gamma, "ir_iters": st_m.ir_iters,
                         "used_gmres": st_m.used_gmres, "rel_residual_mixed": st_m.rel_residual,
                         "gepp_certified_fp64": bool(st_d.gepp_certified), "max_abs_L": st_d.max_abs_L},
            "adjoint_over_primal": (adj["mixed"][0] + adj["mixed"][1]) / ms_mixed,
            "adjoint": {"mixed": {"adjoint_solve_ms": adj["mixed"][0], "assembly_vjp_ms": adj["mixed"][1],
                                  "over_primal": (adj["mixed"][0] + adj["mixed"][1]) / ms_mixed},
                        "fp64": {"adjoint_solve_ms": adj["fp64"][0], "assembly_vjp_ms": adj["fp64"][1],
                                 "over_primal": (adj["fp64"][0] + adj["fp64"][1]) / ms_fp64}},
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 3 * 8 * N,
                    "d2h_bytes_per_step": 8 * N},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "k_tc_gemm_sub<2,RED,BF16,X3> (tcgen05 trailing update from BF16 "
                                                   "hi/lo pairs, three kind::f16 MMAs a 16-deep step, K = 128)",
                         "achieved": tc_gbs, "peak": peak_hbm, "unit": "GB/s", "frac": tc_gbs / peak_hbm,
                         "traffic": traffic, "launches": tc_launches, "ms_total": tc_ms,
                         "algorithmic_bytes": "8 B per updated C element (FP32 read + write; the operand "
                                              "panels add under 3 %)",
                         "peak_source": hbm_src,
                         "tensor_view": {"achieved_tflops": tc_tflops, "bf16_peak_tflops": peak_tc,
                                         "frac_of_bf16": tc_tflops / peak_tc,
                                         "frac_of_bf16_pair_ceiling": tc_tflops / (peak_tc / 3.0),
                                         "note": "2 m n k algorithmic flops; the BF16-pair update issues "
                                                 "3 BF16 MMAs per flop"}},
            "critical_path_roofline": None if diag is None else {
                "bound": "latency", "kernel": "k_pdiag (128 x 128 diagonal block, one CTA)",
                "avg_us_in_place": diag["avg_us"], "launches": diag["launches"],
                "achieved_gflops": (2.0 / 3.0) * 128 ** 3 / (diag["avg_us"] * 1e-6) / 1e9,
                "peak_gflops_one_sm": peak32 * 1e3 / 148.0,
                "frac": (2.0 / 3.0) * 128 ** 3 / (diag["avg_us"] * 1e-6) / 1e9 / (peak32 * 1e3 / 148.0),
                "chain_ms": timeline["stream0_busy_ms"], "span_ms": timeline["span_ms"],
                "peak_source": "measured FP32 FMA throughput (fp_measure_fma_peak) / 148 SMs",
                "note": "2/3 128^3 flops per launch on one SM: the kernel is a chain of dependent steps, "
                        "its frac says how far from compute-bound it is"},
            "assembly_roofline": {"bound": "fp64 pipe", "kernel": "k_asm_ring+k_asm_wake",
                                  "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                                  "frac": achieved / peak64,
                                  "peak_source": "measured FP64 FMA throughput (fp_measure_fma_peak)"},
            "fp64_trailing_update": {"kernel": "k_gemm_sub_dmma<512,4,2,32,2,64,2> (FP64 tensor path, mma.sync .f64, 128 x 64 tiles)",
                                     "launches": d_launches, "ms_total": d_ms,
                                     "tflops": d_flops / (d_ms * 1e-3) / 1e12 if d_ms else 0,
                                     "frac_of_fp64_fma_peak": (d_flops / (d_ms * 1e-3) / 1e12 / peak64) if d_ms else 0,
                                     "fp64_tensor_peak_tflops": peak_dmma,
                                     "frac_of_fp64_tensor_peak": (d_flops / (d_ms * 1e-3) / 1e12 / peak_dmma)
                                     if d_ms else 0},
            "mixed_factor_timeline": timeline,
            "cusolver_getrf": cusolver,
            "sphere_config1": sphere,
            "least_squares_f2": lsq,
            "potential_f3": pot,
            "aoa_sweep_config3a": aoa,
            "batched_wings": batched,
            "surface_loads": post,
            "wingbody_config5": wingbody,
            "clocks": clk.summary()}
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    solver.close()
    ctx.close()


def wingbody_measure(fp, device, steps=3, warmup=1, cpu=True, nprobes=1_000_000):
    """Config 5: prolate-ellipsoid fuselage (120 x 80) + swept NACA 2412 wing
    (150 x 180), 36,600 vortex-ring panels, rigid wake, AoA 3 deg, in the
    mixed form: FP32 static-order LU whose trailing update multiplies BF16
    hi/lo pairs, and FP64 refinement on the FP64 AIC to a relative residual of
    1e-10 (on this body 260 ms against 284 ms for the BF16 form, whose factors
    need GMRES-IR). Errors of strengths, surface Cp, CL and CD against the device FP64 form
    (the plain form, which matches the oracle to 1e-10 on the reduced wing-body
    test). Then velocity and Cp at 1,000,000 probes uniform in a 12 x 12 x 4 m
    box (default_rng(5)), none within 0.01 m of a panel, by the FP32 kernel,
    checked against the FP64 kernel on 20,000 of the probes. Returns a dict."""
    cap = fp._capi
    m = fp.meshes.wing_body()
    body = fp.RigidWakeBody(m)
    N = m.npanels
    normals = fp.calc_normals(body)
    cps = fp.calc_controlpoints(body, normals)
    a = np.deg2rad(3.0)
    V = np.array([np.cos(a), 0.0, np.sin(a)])
    U = np.tile(V, (N, 1))
    D = np.tile(V, (m.nsheddings, 1))
    ctx = cap.Context(device)
    ctx.set_geometry(m.nodes, m.panel_offsets, m.panel_nodes, cps, normals)
    ctx.set_wake(m.shedding, D, D)
    ctx.set_rhs(U)
    VR = cap.FP_ELEMENT_VORTEXRING
    opts = cap.make_opts("ludiv", "mixed", ir_tol=1e-10)

    def solve_step():
        ctx.assemble(VR, 1e-8, 1e-14, cap.FP_PREC_MIXED)
        ctx.factor(cap.FP_PREC_MIXED)
        return ctx.solve_device(1, opts)

    for _ in range(max(1, warmup)):
        solve_step()
    stg = np.zeros(3)
    with ClockSampler(device) as clk:
        for _ in range(steps):
            st = solve_step()
            stg += [st.ms_assemble, st.ms_factor, st.ms_solve]
        stg /= steps
        gamma, st = ctx.solve(1, opts)
        probes = fp.meshes.probe_box(m, nprobes)
        M = probes.shape[0]
        ctx.uind(VR, gamma, probes[:1000], np.tile(V, (1000, 1)), cap.FP_PREC_MIXED)   # warm-up
        field_ms = []
        for _ in range(steps):
            Uout = ctx.uind(VR, gamma, probes, np.tile(V, (M, 1)), cap.FP_PREC_MIXED)
            field_ms.append(ctx.last_kernel_ms(cap.FP_STAGE_UIND)[0])
        Cp = 1.0 - np.sum(Uout * Uout, axis=1)
    ns64 = min(20000, M)
    U64 = ctx.uind(VR, gamma, probes[:ns64], np.tile(V, (ns64, 1)), cap.FP_PREC_FP64)
    f64_ms_per_probe = ctx.last_kernel_ms(cap.FP_STAGE_UIND)[0] / ns64
    # the BF16 form (BF16-rounded AIC, BF16 tensor-core update, GMRES-IR with
    # FP64 residuals to 1e-10) on the same body, beside the mixed form
    opts16 = cap.make_opts("ludiv", "bf16", ir_tol=1e-10)
    stg16 = np.zeros(3)
    for i in range(1 + steps):
        ctx.assemble(VR, 1e-8, 1e-14, cap.FP_PREC_BF16)
        ctx.factor(cap.FP_PREC_BF16)
        st16 = ctx.solve_device(1, opts16)
        if i > 0:
            stg16 += [st16.ms_assemble, st16.ms_factor, st16.ms_solve]
    stg16 /= steps
    gamma16, st16 = ctx.solve(1, opts16)
    # the FP64 form on the same body, for the errors of both reduced forms
    x64, st64 = ctx.solve_body(VR, U, opts=cap.make_opts("ludiv", "fp64"))
    fms = float(np.mean(field_ms))
    nquad = int(np.sum(np.diff(m.panel_offsets) == 4))
    ntri = N - nquad
    ops = M * (248.0 * nquad + 186.0 * ntri + 2 * 290.0 * m.nsheddings)
    achieved = ops / (fms * 1e-3) / 1e12
    peak32 = cap.measure_fma_peak(device, False)
    abs_err = np.linalg.norm(Uout[:ns64] - U64, axis=1) / np.linalg.norm(V)   # in freestream-speed units
    rel = np.linalg.norm(Uout[:ns64] - U64, axis=1) / np.linalg.norm(U64, axis=1)
    dCp = np.abs(Cp[:ns64] - (1.0 - np.sum(U64 * U64, axis=1)))
    croot, taper, AR8 = 1.5, 0.4, 8.0
    cmean = croot * (1 + taper) / 2
    b = AR8 * cmean
    solver = fp.B200Solver("ludiv", "fp64", device=device)
    CLb, CDb, Cpb = lift_coefficient(fp, body, gamma, V, U, D, solver, chord=cmean, sref=b * cmean, with_drag=True)
    CLd, CDd, Cpd = lift_coefficient(fp, body, x64, V, U, D, solver, chord=cmean, sref=b * cmean, with_drag=True)
    solver.close()
    out = {"config": f"wing-body: fuselage 120x80 + NACA2412 wing 150x180 = {N} panels, AoA 3; "
                     f"{M} probes in 12x12x4 m box, none within 0.01 m",
           "form": "mixed: FP32 static-order LU, trailing update from BF16 hi/lo pairs (three kind::f16 "
                   "MMAs, FP32 accumulation), FP64 refinement to a relative residual of 1e-10",
           "solve_ms": {"assemble": stg[0], "factor": stg[1], "solve": stg[2], "total": float(stg.sum())},
           "refinement": {"ir_iters": st.ir_iters, "used_gmres": st.used_gmres, "gmres_iters": st.gmres_iters,
                          "rel_residual": st.rel_residual},
           "fp64_form_ms": {"assemble": st64.ms_assemble, "factor": st64.ms_factor, "solve": st64.ms_solve},
           "bf16_form": {"form": "BF16-rounded AIC, BF16 tensor-core update (kind::f16) with FP32 accumulation, "
                                 "static row order, GMRES-IR with FP64 residuals on the FP64 AIC to 1e-10",
                         "solve_ms": {"assemble": stg16[0], "factor": stg16[1], "solve": stg16[2],
                                      "total": float(stg16.sum())},
                         "refinement": {"ir_iters": st16.ir_iters, "used_gmres": st16.used_gmres,
                                        "gmres_iters": st16.gmres_iters, "rel_residual": st16.rel_residual},
                         "strength_rel_vs_fp64": float(np.linalg.norm(gamma16 - x64) / np.linalg.norm(x64))},
           "errors_vs_fp64": {"strength_rel": float(np.linalg.norm(gamma - x64) / np.linalg.norm(x64)),
                              "Cp_max_abs": float(np.abs(Cpb - Cpd).max()), "CL": CLb, "CL_fp64": CLd,
                              "abs_dCL": abs(CLb - CLd), "CD": CDb, "CD_fp64": CDd, "abs_dCD": abs(CDb - CDd)},
           "field_ms": fms, "field_probes_per_s": M / (fms * 1e-3),
           "field_fp64_ms_per_1M_probes": f64_ms_per_probe * 1e6,
           "field_err_vs_fp64_kernel_over_Vinf": {"max": float(abs_err.max()),
                                                  "p99_9": float(np.quantile(abs_err, 0.999)),
                                                  "median": float(np.median(abs_err)), "probes": int(ns64)},
           "field_rel_err_vs_fp64_kernel": {"max": float(rel.max()), "p99_9": float(np.quantile(rel, 0.999)),
                                            "median": float(np.median(rel)), "probes": int(ns64),
                                            "note": "relative to the local speed, which is near zero inside the bodies"},
           "Cp_abs_err_vs_fp64_kernel": {"max": float(dCp.max()), "p99_9": float(np.quantile(dCp, 0.999))},
           "Cp_range": [float(Cp.min()), float(Cp.max())],
           "field_roofline": {"bound": "fp32 pipe", "kernel": "k_uind_ring<float>",
                              "achieved": achieved, "peak": peak32, "unit": "TFLOP/s", "frac": achieved / peak32,
                              "peak_source": "measured FP32 FMA throughput (fp_measure_fma_peak)"},
           "clocks": clk.summary()}
    if cpu:
        O = ge.load_oracle()
        ncores = os.cpu_count() or 1
        ns = 2000
        t0 = time.perf_counter()
        ref = O.uind_vortexring(m, gamma, D, D, probes[:ns], nthreads=ncores)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        out["field_cpu_baseline"] = {"value": cpu_ms * M / ns, "unit": "ms (1M probes, extrapolated)",
                                     "cores": ncores, "kind": "port",
                                     "sample": f"{ns} probes with the oracle's threaded Uind, x {M // ns}"}
        out["field_rel_err_vs_oracle_max"] = float(np.max(
            np.linalg.norm(Uout[:ns] - (V + ref), axis=1) / np.linalg.norm(V + ref, axis=1)))
    ctx.close()
    return out


def run_wingbody(args, rank, ws, dist):
    """The config-5 line alone (bench.py --workload wingbody)."""
    if rank != 0:
        return
    fp = ge.load_package()
    device = int(os.environ.get("LOCAL_RANK", "0"))
    r = wingbody_measure(fp, device, args.steps, args.warmup, cpu=not args.no_cpu_baseline)
    line = {"metric": "wing-body 36.6k-panel mixed-form solve ms + 1M-probe velocity/Cp ms",
            "value": r["solve_ms"]["total"] + r["field_ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "data": "synthetic", "dtype": "bf16x2+f32+f64",
            "config": {"workload": r["config"]}, **{k: v for k, v in r.items() if k != "config"}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-wing batched throughput leg")
    ap.add_argument("--no-wingbody", action="store_true", help="skip the config-5 wing-body leg of the default line")
    ap.add_argument("--workload", default="wing12k", choices=["wing12k", "wingbody", "surface"],
                    help="wingbody: the 36.6k-panel wing-body solve and 1M-probe field evaluation; "
                         "surface: the post-processing (U, grad(mu), Cp, F, L/D/S) of a 12k-triangle wing")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="with --profile: which form to time")
    ap.add_argument("--profile", action="store_true",
                    help="timed device steps only (for ncu launch lists): no e2e, accuracy or CPU legs")
    ap.add_argument("--n-chord", type=int, default=N_CHORD, help="with --profile: smaller wings for ncu")
    ap.add_argument("--n-span", type=int, default=N_SPAN)
    args = ap.parse_args()
    rank, ws, dist = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, rank, ws, dist)
        elif args.workload == "wingbody":
            run_wingbody(args, rank, ws, dist)
        elif args.workload == "surface":
            if rank == 0:
                print(json.dumps({"workload": "surface", **surface_loads_timing(ge.load_package())}), flush=True)
        else:
            run_ours(args, rank, ws, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
