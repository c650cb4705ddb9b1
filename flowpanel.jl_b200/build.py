"""Build libflowpanel_b200.so in-tree (sm_100a only).

    python flowpanel.jl_b200/build.py [-v]

Each .cu file is compiled to an object in parallel with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` and linked into
``flowpanel.jl_b200/_build/libflowpanel_b200.so`` with the CUDA runtime
linked statically (the library then only needs the driver).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libflowpanel_b200.so")
SOURCES = ["fp_capi.cu", "fp_assembly.cu", "fp_lu.cu", "fp_field.cu", "fp_gmres.cu", "fp_tc.cu", "fp_peak.cu", "fp_vjp.cu", "fp_batch.cu", "fp_ls.cu", "fp_post.cu", "fp_lu_static.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", "-I" + os.path.join(HERE, "..", "include")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(HERE, "..", "include", "flowpanel_b200.h"))
    objs, procs = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OUT_DIR, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(f"--- {s}\n{out}")
        if p.returncode:
            failed.append(s)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    if force or _stale(LIB, objs):
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
               "-ccbin", "/usr/bin/g++", "-o", LIB, *objs]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
