"""Build recipe of the oracle's C restatement (test infrastructure).

    python oracle/build.py

Compiles oracle/qzref.c with gcc into oracle/_build/libqzref.so, linked
against the OpenBLAS build bundled with scipy (LAPACK/BLAS leaves,
symbols prefixed ``scipy_``).
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libqzref.so")


def openblas():
    import scipy
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    libs = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    if not libs:
        raise RuntimeError("scipy's OpenBLAS not found in " + d)
    return d, os.path.basename(libs[0])


def build(force=False):
    src = os.path.join(HERE, "qzref.c")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    os.makedirs(OUT, exist_ok=True)
    d, name = openblas()
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-o", LIB, src,
           "-L" + d, "-l:" + name, "-Wl,-rpath," + d, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
