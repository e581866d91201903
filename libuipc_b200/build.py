"""In-tree build of the native libraries.

    python -m libuipc_b200.build          # product + generator + oracle
    python -m libuipc_b200.build --only solve

Products (git-ignored, shipped with the tree):
  libuipc_b200/_lib/libb200solve.so   CUDA kernels for sm_100a behind include/b200solve.h
  libuipc_b200/_lib/libb200scene.so   synthetic Newton-system generator (host C++)
The CPU oracle (test infrastructure) is built by oracle/build_oracle.py.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_lib")
OBJ = os.path.join(ROOT, "_build", "obj")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-Wall",
]
SOLVE_SOURCES = [
    "b2s_assemble.cu",
    "b2s_spmv.cu",
    "b2s_mas.cu",
    "b2s_mas_invert.cu",
    "b2s_pcg.cu",
    "b2s_learned.cu",
    "b2s_generate.cu",
    "b2s_generate_shell.cu",
    "b2s_abi.cu",
    "b2s_noalloc.cu",
    "b2s_partition.cu",
    "b2s_trajectory.cu",
]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")
    if r.stdout.strip() and os.environ.get("B2S_BUILD_VERBOSE"):
        sys.stderr.write(r.stdout)


def _digest(paths: list[str], extra: str) -> str:
    h = hashlib.sha256(extra.encode())
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(CSRC, "scene", "elements.h"))
    return hs + [os.path.join(ROOT, "include", h) for h in ("b200solve.h", "b200gen.h")]


def build_solve(force: bool = False, extra_flags: list[str] | None = None) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    out = os.path.join(LIB, "libb200solve.so")
    flags = NVFLAGS + (extra_flags or [])
    stamp = out + ".stamp"
    srcs = [os.path.join(CSRC, f) for f in SOLVE_SOURCES]
    dig = _digest(srcs + _headers(), " ".join(flags))
    if not force and os.path.exists(out) and os.path.exists(stamp) and open(stamp).read() == dig:
        return out
    objs = []
    jobs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for src in srcs:
            obj = os.path.join(OBJ, os.path.basename(src) + ".o")
            objs.append(obj)
            jobs.append(ex.submit(_run, [NVCC, *flags, "-c", src, "-o", obj]))
        for j in jobs:
            j.result()
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart"])
    with open(stamp, "w") as f:
        f.write(dig)
    return out


def build_scene(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libb200scene.so")
    srcs = [os.path.join(CSRC, "scene", f) for f in ("scene_gen.cpp", "matrix_market.cpp")]
    hdrs = [os.path.join(CSRC, "scene", h) for h in ("scene_gen.h", "elements.h")] + [
        os.path.join(ROOT, "include", "b200io.h")]
    flags = ["-O3", "-fopenmp", "-shared", "-fPIC", "-std=c++17"]
    stamp = out + ".stamp"
    dig = _digest(srcs + hdrs, " ".join(flags))
    if not force and os.path.exists(out) and os.path.exists(stamp) and open(stamp).read() == dig:
        return out
    _run(["g++", *flags, *srcs, "-o", out])
    with open(stamp, "w") as f:
        f.write(dig)
    return out


def build_all(force: bool = False) -> None:
    build_scene(force)
    build_solve(force)
    sys.path.insert(0, ROOT)
    from oracle import build_oracle  # test infrastructure: the checker

    build_oracle.build(force)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["solve", "scene", "oracle"], default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    if a.only == "solve":
        print(build_solve(a.force))
    elif a.only == "scene":
        print(build_scene(a.force))
    elif a.only == "oracle":
        sys.path.insert(0, ROOT)
        from oracle import build_oracle

        build_oracle.build(a.force)
    else:
        build_all(a.force)


if __name__ == "__main__":
    main()
