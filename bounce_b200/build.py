"""Build libb3g.so in-tree with nvcc for sm_100a.

    python -m bounce_b200.build          (or build() from Python)

All kernels are compiled with -fmad=false: the element force and Jacobian
arithmetic then rounds exactly like the CPU reference.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libb3g.so")
SOURCES = ["cloth_kernels.cu", "cloth_api.cu", "mpcg_solve.cu", "batch_cg.cu", "batch_api.cu", "server.cu", "grid_cg.cu",
           "softbody.cu", "self_collision.cu", "bodies.cu", "topology.cpp", "softbody_prep.cpp", "broadphase_order.cpp"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(objs, srcs) -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "b3g.h"),
                                                                  os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(os.path.join(LIBDIR, "obj"), exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    objs = [os.path.join(LIBDIR, "obj", os.path.basename(s) + ".o") for s in SOURCES]
    if not force and not _stale(objs, srcs):
        return LIB
    nvcc = _nvcc()
    procs = []
    for s, o in zip(srcs, objs):
        cmd = [nvcc] + NVCC_FLAGS + ["-x", "cu" if s.endswith(".cu") else "c++", "-c", s, "-o", o]
        if s.endswith(".cpp"):
            cmd = [nvcc, "-O3", "-std=c++17", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   "-c", s, "-o", o]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
