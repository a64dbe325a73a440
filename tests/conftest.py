import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


_state = {"L": None}


def gpu_lattice(L, prec="D"):
    """Initialise the library for lattice L (re-initialising if needed)."""
    from qopqdp_b200.qop import Qop
    q = Qop(prec)
    L = tuple(L)
    if _state["L"] != L:
        if q.lib.QOP_is_initialized():
            q.finalize()
        st = q.init(L)
        assert st == 0, "QOP_init failed for %s" % (L,)
        _state["L"] = L
    return q
