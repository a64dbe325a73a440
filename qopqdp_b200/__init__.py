"""B200-native asqtad/HISQ staggered Dslash and Krylov solvers behind the
QOPQDP C API.

The product is the C-ABI library lib/libqop_b200.so (sources in csrc/,
declarations in include/qop.h).  This package holds its build script, a
ctypes mirror of the API (qop.py) and the seeded input generator
(lattice.py).
"""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libqop_b200.so")


def library_path():
    return LIB_PATH
