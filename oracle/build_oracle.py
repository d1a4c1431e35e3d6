"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/ref_lu.cpp into oracle/liboracle_lu.so, linked against the
OpenBLAS that ships inside the scipy wheel (exported with a ``scipy_``
prefix, LP64).  charmlu itself is not compiled: it needs the Charm++ runtime
(charmc, CkMulticast, SDAG, CrnStream) and cblas.h, none of which exist in
this image, so there is no oracle/_ref build.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "liboracle_lu.so")


def find_openblas():
    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas-*.so")))
    if not cands:
        raise RuntimeError("scipy's bundled OpenBLAS not found under " + libdir)
    return cands[0]


def build(force=False):
    src = os.path.join(HERE, "ref_lu.cpp")
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(src):
        return OUT
    blas = find_openblas()
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           src, "-o", OUT, blas, "-Wl,-rpath," + os.path.dirname(blas)]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
