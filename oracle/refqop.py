"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the reference's own asqtad
path, compiled from the unmodified QOPQDP 0.21.1 sources by oracle/ref
(against a single-process CPU implementation of the QDP/QLA/QMP calls it
makes) into oracle/_ref/libqopref.so.

It pins the oracle: tests compare the plain-C oracle (oracle.py) with the
reference's lib/asqtad_dslash_p.c, lib/asqtad_invert_p.c and
lib/invert_cg_p.c on the same inputs.  Only the test suite and bench.py's
reference arm use it.  The library exists only where the reference sources
were present when it was built; `available()` says whether it is.

The reference keeps per-lattice state in globals (shift tables, the
Dslash temporaries of lib/asqtad_dslash_p.c) that QOP_finalize does not
reset, so one loaded copy serves one lattice geometry: `RefLattice(L)`
loads a private copy of the library per geometry.
"""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np

from oracle import InvertArg, ResidArg, f64, _p, DP

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libqopref.so")
SRC = os.path.join(HERE, "ref")
F3, D3 = 0, 1


def build(ref_root="/root/reference"):
    """Compile the reference's path into LIB when its sources are present
    (a no-op, returning None, where they are not)."""
    if not os.path.isdir(os.path.join(ref_root, "lib")):
        return LIB if os.path.exists(LIB) else None
    subprocess.run(["make", "-C", SRC, "-s", "REF=" + ref_root], check=True)
    return LIB


def available():
    return os.path.exists(LIB)


_copies = {}
_tmpdir = None


def _load(L):
    global _tmpdir
    key = tuple(L)
    if key in _copies:
        return _copies[key]
    if not available():
        raise RuntimeError("reference library not built (oracle/_ref/libqopref.so)")
    if _tmpdir is None:
        _tmpdir = tempfile.mkdtemp(prefix="qopref_")
    path = os.path.join(_tmpdir, "libqopref_%s.so" % "x".join(map(str, key)))
    shutil.copyfile(LIB, path)
    l = C.CDLL(path, mode=os.RTLD_LOCAL)
    vp = C.c_void_p
    l.qr_init.argtypes = [C.POINTER(C.c_int)]
    l.qr_verbose.argtypes = [C.c_int]
    l.qr_set_opt.argtypes = [C.c_char_p, C.c_double]
    l.qr_fla_create.argtypes = [C.c_int, C.POINTER(DP), C.POINTER(DP)]
    l.qr_fla_create.restype = vp
    l.qr_fla_destroy.argtypes = [C.c_int, vp]
    l.qr_dslash.argtypes = [C.c_int, vp, C.c_double, DP, DP, C.c_int, C.c_int]
    l.qr_invert.argtypes = [C.c_int, vp, C.POINTER(InvertArg), C.POINTER(ResidArg), C.c_double, DP, DP,
                            C.POINTER(C.c_double)]
    l.qr_invert_multi.argtypes = [C.c_int, vp, C.POINTER(InvertArg), C.POINTER(C.POINTER(C.POINTER(ResidArg))),
                                  C.POINTER(DP), C.POINTER(C.c_int), C.POINTER(C.POINTER(DP)), C.POINTER(DP),
                                  C.c_int, C.POINTER(C.c_double)]
    l.qr_set_threads.argtypes = [C.c_int]
    l.qr_rephase_G.argtypes = [C.POINTER(DP), C.POINTER(C.c_int), DP, C.POINTER(C.c_int)]
    l.qr_asqtad_links_from_G.argtypes = [DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP)]
    l.qr_hisq_links.argtypes = [DP, C.c_int, DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP), C.POINTER(DP),
                                C.POINTER(DP), C.POINTER(DP)]
    l.qr_asqtad_deriv.argtypes = [DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP), C.POINTER(DP)]
    l.QOP_D3_u3_un_der_analytic.argtypes = [C.c_void_p, DP, DP, DP, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    l.QOP_hisq_force_set_opts.argtypes = [C.c_void_p, C.c_int]
    l.qr_asqtad_force.argtypes = [DP, C.POINTER(DP), C.POINTER(DP), DP, C.POINTER(DP), C.c_int, C.c_int]
    l.qr_hisq_force.argtypes = [DP, C.c_int, DP, C.POINTER(DP), C.POINTER(DP), DP, C.POINTER(DP),
                                C.POINTER(C.c_int), C.c_double]
    st = l.qr_init((C.c_int * 4)(*key))
    if st != 0:
        raise RuntimeError("QOP_init failed (%d)" % st)
    _copies[key] = l
    return l


def _p4(arrs):
    return (DP * 4)(*[_p(a) for a in arrs])


class RefFla:
    """The reference's QOP_{F3,D3}_FermionLinksAsqtad built from raw fat and
    long links (V x 3 x 3 complex as V x 18 doubles per direction; lng None
    for the no-Naik operator), with the oracle.Fla call surface."""

    def __init__(self, L, fat, lng, prec=D3):
        self.L = tuple(int(x) for x in L)
        self.prec = prec
        self.lib = _load(self.L)
        fat = [f64(a) for a in fat]
        lng = [f64(a) for a in lng] if lng is not None else None
        self.h = self.lib.qr_fla_create(prec, _p4(fat), _p4(lng) if lng is not None else None)
        if not self.h:
            raise RuntimeError("QOP_asqtad_create_L_from_qdp failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.qr_fla_destroy(self.prec, self.h)
            self.h = None

    def dslash(self, mass, inp, eo_out, eo_in, out=None):
        inp = f64(inp)
        out = np.zeros_like(inp) if out is None else f64(out).copy()
        st = self.lib.qr_dslash(self.prec, self.h, mass, _p(out), _p(inp), eo_out, eo_in)
        if st != 0:
            raise RuntimeError("QOP_asqtad_dslash_qdp status %d" % st)
        return out

    def invert(self, mass, inp, inv_arg, res_arg, out=None):
        inp = f64(inp)
        out = np.zeros_like(inp) if out is None else f64(out).copy()
        flop = C.c_double(0)
        self.lib.qr_invert(self.prec, self.h, C.byref(inv_arg), C.byref(res_arg), mass, _p(out), _p(inp),
                           C.byref(flop))
        return out, flop.value

    def invert_multi(self, masses, ins, inv_arg, res_args):
        nsrc = len(ins)
        ins = [f64(a) for a in ins]
        outs = [[np.zeros_like(ins[s]) for _ in masses[s]] for s in range(nsrc)]
        RA = C.POINTER(ResidArg)
        ra_rows = [(RA * len(r))(*[C.pointer(x) for x in r]) for r in res_args]
        ra = (C.POINTER(RA) * nsrc)(*[C.cast(r, C.POINTER(RA)) for r in ra_rows])
        m_rows = [(C.c_double * len(m))(*m) for m in masses]
        mp = (DP * nsrc)(*[C.cast(m, DP) for m in m_rows])
        nm = (C.c_int * nsrc)(*[len(m) for m in masses])
        o_rows = [(DP * len(o))(*[_p(a) for a in o]) for o in outs]
        op = (C.POINTER(DP) * nsrc)(*[C.cast(o, C.POINTER(DP)) for o in o_rows])
        ip_ = (DP * nsrc)(*[_p(a) for a in ins])
        flop = C.c_double(0)
        self.lib.qr_invert_multi(self.prec, self.h, C.byref(inv_arg), ra, mp, nm, op, ip_, nsrc, C.byref(flop))
        return outs, flop.value


def set_opt(L, tag, value):
    """QOP_asqtad_invert_set_opts({tag, value}) in the copy serving L."""
    return _load(tuple(L)).qr_set_opt(tag.encode(), float(value))


def rephase_G(L, links, r0=(0, 0, 0, 0), bc=(1, 1, 1, -1), signmask=(0, 1, 3, 7)):
    """QOP_D3_rephase_G_qdp on copies of raw links (oracle.Lattice.rephase_G
    call surface)."""
    links = [f64(a).copy() for a in links]
    bcr = np.array([[complex(z).real, complex(z).imag] for z in bc], dtype=np.float64).ravel()
    _load(tuple(L)).qr_rephase_G(_p4(links), (C.c_int * 4)(*r0), _p(bcr), (C.c_int * 4)(*signmask))
    return links


def asqtad_links(L, coeffs, gauge, naik=True):
    """Fat (and long) links of QOP_D3_asqtad_create_L_from_G, unscaled
    (oracle.Lattice.make_imp_links call surface)."""
    gauge = [f64(a) for a in gauge]
    fat = [np.zeros_like(gauge[0]) for _ in range(4)]
    lng = [np.zeros_like(gauge[0]) for _ in range(4)] if naik else None
    c = np.array(coeffs, dtype=np.float64)
    if not naik:
        c[5] = 0.0
    st = _load(tuple(L)).qr_asqtad_links_from_G(_p(c), _p4(gauge), _p4(fat), _p4(lng) if naik else None)
    if st != 0:
        raise RuntimeError("QOP_asqtad_create_L_from_G status %d" % st)
    return fat, lng


def hisq_links(L, hcoef, gauge, eps_naik=(0.0,), want_deps=False):
    """Link sets of QOP_D3_hisq_create_L_from_G (U(3), analytic projection):
    ([(fat, long)] * len(eps_naik), W, (deps_fat, deps_long) or None), all
    unscaled; hcoef holds the 13 coefficients in QOP_hisq_coeffs_t order
    (fat7 x5, asqtad x6, difference x2)."""
    gauge = [f64(a) for a in gauge]
    nk = len(eps_naik)
    z = lambda n: [np.zeros_like(gauge[0]) for _ in range(n)]
    fat, lng, W = z(4 * nk), z(4 * nk), z(4)
    dfat, dlng = (z(4), z(4)) if want_deps else (None, None)
    P = lambda arrs: (DP * len(arrs))(*[_p(a) for a in arrs])
    st = _load(tuple(L)).qr_hisq_links(_p(f64(np.asarray(hcoef)[:13])), nk, _p(f64(eps_naik)), P(gauge), P(fat),
                                       P(lng), P(W), P(dfat) if want_deps else None,
                                       P(dlng) if want_deps else None)
    if st != 0:
        raise RuntimeError("QOP_hisq_create_L_from_G status %d" % st)
    sets = [(fat[4 * k:4 * k + 4], lng[4 * k:4 * k + 4]) for k in range(nk)]
    return sets, W, ((dfat, dlng) if want_deps else None)


def set_threads(L, n):
    """OpenMP threads of the site loops in the copy serving L (n <= 0 keeps
    the current number); returns the number in effect."""
    return _load(tuple(L)).qr_set_threads(int(n))


def asqtad_force(L, coeffs, gauge, eps, xs, force=None, fnmat_src_min=2):
    """force_mu += the asqtad fermion force of QOP_D3_asqtad_force_multi_qdp
    for raw vectors xs with weights eps (oracle.Lattice.asqtad_force call
    surface); fnmat_src_min picks the reference's ASVEC (nsrc below it) or
    FNMAT algorithm."""
    gauge = [f64(a) for a in gauge]
    force = [np.zeros_like(gauge[0]) for _ in range(4)] if force is None else [f64(a).copy() for a in force]
    xs = [f64(x) for x in xs]
    P = lambda arrs: (DP * len(arrs))(*[_p(a) for a in arrs])
    st = _load(tuple(L)).qr_asqtad_force(_p(f64(coeffs)), P(gauge), P(force), _p(f64(eps)), P(xs), len(xs),
                                         int(fnmat_src_min))
    if st != 0:
        raise RuntimeError("QOP_asqtad_force_multi_qdp status %d" % st)
    return force


def hisq_force(L, hcoef, gauge, eps_naik, res, xs, n_orders, force=None):
    """force_mu += the HISQ fermion force of QOP_D3_hisq_force_multi_qdp on
    the links QOP_D3_hisq_create_L_from_G builds from gauge
    (oracle.Lattice.hisq_force call surface)."""
    gauge = [f64(a) for a in gauge]
    force = [np.zeros_like(gauge[0]) for _ in range(4)] if force is None else [f64(a).copy() for a in force]
    xs = [f64(x) for x in xs]
    P = lambda arrs: (DP * len(arrs))(*[_p(a) for a in arrs])
    hcoef = np.asarray(hcoef)
    ff = float(hcoef[17]) if len(hcoef) > 17 else 5e-5
    st = _load(tuple(L)).qr_hisq_force(_p(f64(hcoef[:13])), len(eps_naik), _p(f64(eps_naik)), P(gauge),
                                       P(force), _p(f64(res)), P(xs), (C.c_int * len(n_orders))(*n_orders), ff)
    if st != 0:
        raise RuntimeError("QOP_hisq_force_multi_qdp status %d" % st)
    return force


def asqtad_deriv(L, coeffs, gauge, midF, midN=None):
    """The reference's QOP_D3_asqtad_deriv (oracle.Lattice.asqtad_deriv call
    surface): its derivative field equals the oracle's up to terms U H, H
    Hermitian, that the force's projection TA(U D^+) removes."""
    gauge = [f64(a) for a in gauge]
    der = [np.zeros_like(gauge[0]) for _ in range(4)]
    st = _load(tuple(L)).qr_asqtad_deriv(_p(f64(coeffs)), _p4(gauge), _p4(der), _p4([f64(a) for a in midF]),
                                         _p4([f64(a) for a in midN]) if midN is not None else None)
    if st != 0:
        raise RuntimeError("QOP_asqtad_deriv status %d" % st)
    return der


class _Info(C.Structure):
    _fields_ = [("final_sec", C.c_double), ("final_flop", C.c_double), ("status", C.c_int), ("count1", C.c_int),
                ("count2", C.c_int)]


class _Opt(C.Structure):
    _fields_ = [("tag", C.c_char_p), ("value", C.c_double), ("extra", C.c_void_p)]


def u3_der(L, V, force_filter=5e-5):
    """The reference's QOP_D3_u3_un_der_analytic for one 3x3 complex matrix V:
    (dW/dV, dW^+/dV) as [i, j, m, n] = d(.)_ij / dV_mn, and whether the force
    filter was applied (QOP_hisq_force_set_opts force_filter)."""
    l = _load(tuple(L))
    o = _Opt(b"force_filter", float(force_filter), None)
    if l.QOP_hisq_force_set_opts(C.addressof(o), 1) != 0:
        raise RuntimeError("QOP_hisq_force_set_opts failed")
    v = np.ascontiguousarray(np.stack([np.real(V), np.imag(V)], -1), dtype=np.float64)
    dw, dwd = np.zeros((3, 3, 3, 3, 2)), np.zeros((3, 3, 3, 3, 2))
    svd, ff, info = C.c_int(0), C.c_int(0), _Info()
    l.QOP_D3_u3_un_der_analytic(C.addressof(info), _p(v), _p(dw), _p(dwd), C.byref(svd), C.byref(ff))
    cz = lambda a: np.einsum("imnj->ijmn", a[..., 0] + 1j * a[..., 1])
    return cz(dw), cz(dwd), bool(ff.value)
