"""The C-ABI library loads on a machine without a GPU and exports every
entry point include/b200qz.h declares (no compute calls here)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "b200qz.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z0-9_]+)\s*\(", src)) - {"if", "sizeof"})


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("pdhgeqz_", "kkqzconf_", "b200qz_create", "b200qz_solve_dev", "b200qz_solve_host"):
        assert s in syms


def test_library_exports_all_declared(pkg):
    lib = pkg.lib()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(pkg.EXPORTS) <= set(declared_symbols())


def test_kkqzconf_noop(pkg):
    pkg.kkqzconf(2.2e-16)


def test_pdhgeqz_argument_errors_need_no_gpu(pkg):
    import numpy as np
    n = 8
    H, T = pkg.pencils.random_ht(n, 0)
    Q = np.eye(n, order="F")
    Z = np.eye(n, order="F")
    # argument checks run before any device work (PDHGEQZ.f:383-405)
    assert pkg.pdhgeqz("X", "I", "I", H, T, Q, Z)[3] == -1
    assert pkg.pdhgeqz("S", "X", "I", H, T, Q, Z)[3] == -2
    assert pkg.pdhgeqz("S", "I", "X", H, T, Q, Z)[3] == -3
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, ilo=0)[3] == -5
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, ihi=n + 1)[3] == -6
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, nb=4)[3] == -7
    d = [pkg.descriptor(n, 16, n) for _ in range(4)]
    d[0][4] = 8  # MB != NB
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, descs=d)[3] == -8
    # workspace query (PDHGEQZ.f:409-430)
    dw, iw, _, info = pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, nb=16, ldwork=-1)
    assert info == 0 and dw == n * 16 and iw == 2 * n
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, nb=16, ldwork=5)[3] == -9
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, nb=16, liwork=3)[3] == -10
    # quick return: nothing touched
    H0 = H.copy()
    assert pkg.pdhgeqz("S", "I", "I", H, T, Q, Z, ilo=5, ihi=4)[3] == 0
    assert np.array_equal(H, H0)


def test_pdgghrd_argument_errors_need_no_gpu(pkg):
    """The PDGGHRD drop-in's quick return, workspace query and argument
    checks (src/ab2ht/PDGGHRD.f:198, 243-250, 278-296) run before any
    device work."""
    import ctypes
    import numpy as np
    n, nb = 6, 4
    A = np.array(np.arange(n * n, dtype=np.float64).reshape(n, n), order="F")
    A0 = A.copy()
    d = pkg.descriptor(n, nb, n)
    dp = d.ctypes.data_as(pkg._pi)
    work = np.zeros(nb)
    L = pkg.lib()

    def call(cq, cz, nn, ilo, ihi, desca, lwork):
        info = ctypes.c_int(99)
        L.pdgghrd_(cq, cz, pkg._ip(nn), pkg._ip(ilo), pkg._ip(ihi), pkg._vp(A.ctypes.data),
                   desca.ctypes.data_as(pkg._pi), pkg._vp(A.ctypes.data), dp, pkg._vp(A.ctypes.data), dp,
                   pkg._vp(A.ctypes.data), dp, pkg._p(work), ctypes.byref(ctypes.c_int(lwork)), ctypes.byref(info),
                   1, 1)
        return info.value

    # N <= 1: returns before any check
    assert call(b"X", b"X", 1, 1, 1, d, 0) == 0
    # workspace query: DESCA(MB_) in WORK(1)
    assert call(b"I", b"I", n, 1, n, d, -1) == 0 and work[0] == nb
    assert call(b"X", b"I", n, 1, n, d, nb) == -1
    assert call(b"I", b"X", n, 1, n, d, nb) == -2
    assert call(b"I", b"I", n, 0, n, d, nb) == -4
    assert call(b"I", b"I", n, 1, n + 1, d, nb) == -5
    assert call(b"I", b"I", n, 3, 1, d, nb) == -5
    bad = d.copy()
    bad[4] = nb + 1
    assert call(b"I", b"I", n, 1, n, bad, nb) == -6
    assert call(b"I", b"I", n, 1, n, d, nb - 1) == -7
    assert np.array_equal(A, A0)


def test_header_compiles_as_c99_and_links(tmp_path, pkg):
    """include/b200qz.h is plain C: a C99 program (pedantic, warnings as
    errors) includes it, links libb200qz.so and calls an entry point that
    needs no GPU."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "use_header.c"
    src.write_text('#include "b200qz.h"\n#include <stdio.h>\n'
                   'int main(void) { printf("%d\\n", b200qz_policy_nparams()); return 0; }\n')
    libdir = os.path.join(root, "gevp-pdhgeqz_b200")
    exe = str(tmp_path / "use_header")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(root, "include"),
                    str(src), "-L", libdir, "-lb200qz", "-Wl,-rpath," + libdir, "-o", exe], check=True,
                   capture_output=True, timeout=120)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=60)
    assert int(out.stdout.strip()) == pkg.learned.nparams()
