"""Build recipe of the oracle (test infrastructure only).

  oracle/_build/liboracle.so   C++ restatement of the reference algorithm
  oracle/_ref/libmetis_ref.so  the reference's own vendored METIS, compiled
                               from its sources where they lie (only when the
                               reference tree is present; output git-ignored)
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
REFERENCE = os.environ.get("B2S_REFERENCE_TREE", "/root/reference")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError("oracle build failed")


def _stamp_ok(out, srcs, flags):
    h = hashlib.sha256(" ".join(flags).encode())
    for s in srcs:
        h.update(open(s, "rb").read())
    dig = h.hexdigest()
    st = out + ".stamp"
    ok = os.path.exists(out) and os.path.exists(st) and open(st).read() == dig
    return ok, dig


def build_oracle_lib(force=False):
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "liboracle.so")
    srcs = [os.path.join(HERE, "oracle.cpp"), os.path.join(HERE, "oracle.h")]
    flags = ["-O2", "-fopenmp", "-shared", "-fPIC", "-std=c++17"]
    ok, dig = _stamp_ok(out, srcs, flags)
    if ok and not force:
        return out
    _run(["g++", *flags, srcs[0], "-o", out])
    open(out + ".stamp", "w").write(dig)
    return out


def build_metis_ref(force=False):
    """Compile libuipc's vendored METIS 5.2.1 C++ port (src/geometry/metis)
    straight from the reference tree into oracle/_ref/libmetis_ref.so."""
    src_dir = os.path.join(REFERENCE, "src", "geometry", "metis")
    if not os.path.isdir(src_dir):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "libmetis_ref.so")
    srcs = sorted(glob.glob(os.path.join(src_dir, "*.cpp")))
    flags = ["-O2", "-std=c++20", "-shared", "-fPIC", "-w", "-I" + src_dir]
    ok, dig = _stamp_ok(out, srcs, flags)
    if ok and not force:
        return out
    _run(["g++", *flags, *srcs, "-o", out])
    open(out + ".stamp", "w").write(dig)
    return out


def build(force=False):
    build_oracle_lib(force)
    try:
        build_metis_ref(force)
    except RuntimeError:
        sys.stderr.write("note: the reference's METIS did not compile; partitions use RCB only\n")


if __name__ == "__main__":
    build("--force" in sys.argv)
