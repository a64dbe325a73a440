"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU oracle (qop_oracle.c).

Only the test suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg
use this module, always as the checker or the timed CPU reference.  The
oracle is a plain-C FP64 restatement of the reference's asqtad/HISQ path,
pinned to the reference itself: refqop.py drives the reference's own
sources compiled by oracle/ref, and tests/test_ref_pin.py compares the two
(and this oracle with the reference's committed outputs under tests/golden).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

EVEN, ODD, EVENODD = 0, 1, 2


def build():
    src = os.path.join(HERE, "qop_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB


class InvertArg(C.Structure):
    _fields_ = [("mixed_rsq", C.c_double), ("max_iter", C.c_int), ("restart", C.c_int),
                ("max_restarts", C.c_int), ("evenodd", C.c_int)]


class ResidArg(C.Structure):
    _fields_ = [("rsqmin", C.c_double), ("final_rsq", C.c_double), ("relmin", C.c_double),
                ("final_rel", C.c_double), ("final_iter", C.c_int), ("final_restart", C.c_int)]


_lib = None
DP = C.POINTER(C.c_double)


def lib():
    global _lib
    if _lib is None:
        build()
        l = C.CDLL(LIB)
        vp = C.c_void_p
        l.or_lat_create.argtypes = [C.POINTER(C.c_int)]
        l.or_lat_create.restype = vp
        l.or_lat_destroy.argtypes = [vp]
        l.or_raw_index.argtypes = [vp, C.POINTER(C.c_int)]
        l.or_raw_index.restype = C.c_long
        l.or_rephase_G.argtypes = [vp, C.POINTER(DP), C.POINTER(C.c_int), DP, C.POINTER(C.c_int)]
        l.or_make_imp_links.argtypes = [vp, DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP), C.POINTER(DP)]
        l.or_u3_un_analytic.argtypes = [DP, DP, C.c_int, C.c_double, C.c_double]
        l.or_u3_un_analytic.restype = C.c_int
        l.or_hisq_links.argtypes = [vp, DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP), C.POINTER(DP)]
        l.or_hisq_links.restype = C.c_int
        l.or_fla_create.argtypes = [vp, C.POINTER(DP), C.POINTER(DP)]
        l.or_asqtad_deriv.argtypes = [vp, DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP), C.POINTER(DP), C.c_int]
        l.or_asqtad_force.argtypes = [vp, DP, C.POINTER(DP), C.POINTER(DP), DP, C.POINTER(DP), C.c_int, C.c_int]
        l.or_hisq_deriv.argtypes = [vp, DP, C.POINTER(DP), C.c_int, DP, C.POINTER(DP), C.POINTER(DP), C.POINTER(DP)]
        l.or_hisq_force.argtypes = [vp, DP, C.POINTER(DP), C.c_int, DP, C.POINTER(DP), DP, C.POINTER(DP),
                                    C.POINTER(C.c_int)]
        l.or_fla_create.restype = vp
        l.or_fla_destroy.argtypes = [vp]
        l.or_dslash.argtypes = [vp, C.c_double, DP, DP, C.c_int, C.c_int]
        l.or_dslash_dir.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, DP, DP, C.c_int]
        l.or_ddagd.argtypes = [vp, C.c_double, DP, DP, C.c_int]
        l.or_ddagd_norm2.argtypes = [vp, C.c_double, DP, DP, C.c_int]
        l.or_ddagd_norm2.restype = C.c_double
        l.or_check_op.argtypes = [vp, C.c_double, DP, C.POINTER(DP), C.POINTER(DP)]
        l.or_check_op.restype = C.c_double
        l.or_relnorm2.argtypes = [vp, DP, DP, C.c_int]
        l.or_relnorm2.restype = C.c_double
        l.or_invert.argtypes = [vp, C.POINTER(InvertArg), C.POINTER(ResidArg), C.c_double, DP, DP, DP]
        l.or_invert_multi.argtypes = [vp, C.POINTER(InvertArg), C.POINTER(C.POINTER(C.POINTER(ResidArg))),
                                      C.POINTER(DP), C.POINTER(C.c_int), C.POINTER(C.POINTER(DP)), C.POINTER(DP),
                                      C.c_int, DP]
        l.or_solve_multi.argtypes = [vp, C.POINTER(InvertArg), C.POINTER(C.POINTER(ResidArg)), DP, C.POINTER(DP),
                                     C.POINTER(DP), C.c_int, DP]
        l.or_set_threads.argtypes = [C.c_int]
        l.or_get_threads.restype = C.c_int
        _lib = l
    return _lib


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(DP)


def _p4(arrs):
    return (DP * 4)(*[_p(a) for a in arrs])


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Lattice:
    def __init__(self, L):
        self.L = tuple(int(x) for x in L)
        self.V = int(np.prod(self.L))
        self.h = lib().or_lat_create((C.c_int * 4)(*self.L))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_lat_destroy(self.h)
            self.h = None

    def rephase_G(self, links, r0=(0, 0, 0, 0), bc=(1, 1, 1, -1), signmask=(0, 1, 3, 7)):
        links = [f64(a).copy() for a in links]
        bcr = np.array([[complex(z).real, complex(z).imag] for z in bc], dtype=np.float64).ravel()
        lib().or_rephase_G(self.h, _p4(links), (C.c_int * 4)(*r0), _p(bcr), (C.c_int * 4)(*signmask))
        return links

    def make_imp_links(self, coeffs, gauge, naik=True):
        gauge = [f64(a) for a in gauge]
        fat = [np.zeros_like(gauge[0]) for _ in range(4)]
        lng = [np.zeros_like(gauge[0]) for _ in range(4)] if naik else None
        c = np.array(coeffs, dtype=np.float64)
        lib().or_make_imp_links(self.h, _p(c), _p4(gauge), _p4(gauge), _p4(fat), _p4(lng) if naik else None)
        return fat, lng

    def asqtad_deriv(self, coeffs, gauge, midF, midN=None, lepage_rep=False):
        """deriv_mu = dE/dU_mu for E = Re sum tr[midF^+ fat + midN^+ long];
        lepage_rep adds the reference's Lepage term of the form U H (H
        Hermitian), giving its QOP_asqtad_deriv field."""
        gauge = [f64(a) for a in gauge]
        midF = [f64(a) for a in midF]
        midN = [f64(a) for a in midN] if midN is not None else None
        der = [np.zeros_like(gauge[0]) for _ in range(4)]
        c = np.array(coeffs, dtype=np.float64)
        lib().or_asqtad_deriv(self.h, _p(c), _p4(gauge), _p4(midF), _p4(midN) if midN is not None else None, _p4(der),
                              int(bool(lepage_rep)))
        return der

    def asqtad_force(self, coeffs, gauge, eps, xs, force=None, fnmat_src_min=2):
        """force_mu += -2 TA(U_mu deriv_mu^+) for the outer products of xs
        (FNMAT); with fewer sources than fnmat_src_min (2, the reference's
        default) the reference's ASVEC result, force = TA(force) - TA(U deriv^+)."""
        gauge = [f64(a) for a in gauge]
        force = [np.zeros_like(gauge[0]) for _ in range(4)] if force is None else [f64(a).copy() for a in force]
        xs = [f64(x) for x in xs]
        xp = (DP * len(xs))(*[_p(x) for x in xs])
        e = np.array(eps, dtype=np.float64)
        c = np.array(coeffs, dtype=np.float64)
        lib().or_asqtad_force(self.h, _p(c), _p4(gauge), _p4(force), _p(e), xp, len(xs),
                              1 if len(xs) < fnmat_src_min else 0)
        return force

    def hisq_deriv(self, hcoef, gauge, eps_naik, midF, midN):
        """deriv = dE/dU for E = sum_k c_k Re sum tr[midF_k^+ fat_k(W) + midN_k^+ long_k(W)];
        midF / midN: lists of n_naiks lists of 4 fields."""
        gauge = [f64(a) for a in gauge]
        nk = len(midF)
        mf = [f64(a) for grp in midF for a in grp]
        mn = [f64(a) for grp in midN for a in grp]
        der = [np.zeros_like(gauge[0]) for _ in range(4)]
        lib().or_hisq_deriv(self.h, _p(f64(hcoef)), _p4(gauge), nk, _p(f64(eps_naik)),
                            (DP * len(mf))(*[_p(a) for a in mf]), (DP * len(mn))(*[_p(a) for a in mn]), _p4(der))
        return der

    def hisq_force(self, hcoef, gauge, eps_naik, res, xs, n_orders, force=None):
        gauge = [f64(a) for a in gauge]
        force = [np.zeros_like(gauge[0]) for _ in range(4)] if force is None else [f64(a).copy() for a in force]
        xs = [f64(x) for x in xs]
        lib().or_hisq_force(self.h, _p(f64(hcoef)), _p4(gauge), len(n_orders), _p(f64(eps_naik)), _p4(force),
                            _p(f64(res)), (DP * len(xs))(*[_p(x) for x in xs]), (C.c_int * len(n_orders))(*n_orders))
        return force

    def hisq_links(self, hcoef, gauge, want_W=False):
        gauge = [f64(a) for a in gauge]
        fat = [np.zeros_like(gauge[0]) for _ in range(4)]
        lng = [np.zeros_like(gauge[0]) for _ in range(4)]
        W = [np.zeros_like(gauge[0]) for _ in range(4)] if want_W else None
        n = lib().or_hisq_links(self.h, _p(f64(hcoef)), _p4(gauge), _p4(fat), _p4(lng), _p4(W) if want_W else None)
        return fat, lng, W, n


    def hisq_links_naik(self, hcoef, gauge, eps_naik):
        """All link sets of QOP_hisq_create_L_from_G with n_naiks = len(eps_naik)
        (lib/hisq_links_p.c:182-243): fn[0] = asqtad(acoeffs2, W) and, for
        k >= 1, fn[k] = eps_naik[k] asqtad(acoeffs3, W) + fn[0], where
        acoeffs3 keeps only difference_one_link and difference_naik
        (:107-112); deps = asqtad(acoeffs3, W), the links QOP keeps for the
        derivative with respect to epsilon (want_deps).  Returns
        ([(fat, long)] * n_naiks, (deps_fat, deps_long))."""
        fat, lng, W, _ = self.hisq_links(hcoef, gauge, want_W=True)
        h = f64(hcoef)
        dfat, dlng = self.make_imp_links([h[11], 0.0, 0.0, 0.0, 0.0, h[12]], W)
        sets = [(fat, lng)]
        for e in list(eps_naik)[1:]:
            sets.append(([e * a + b for a, b in zip(dfat, fat)], [e * a + b for a, b in zip(dlng, lng)]))
        return sets, (dfat, dlng)


class Fla:
    """Oracle asqtad operator (links x 1/2, double stored)."""

    def __init__(self, lat, fat, lng):
        self.lat = lat
        self.fat = [f64(a) for a in fat]
        self.lng = [f64(a) for a in lng] if lng is not None else None
        self.h = lib().or_fla_create(lat.h, _p4(self.fat), _p4(self.lng) if self.lng is not None else None)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_fla_destroy(self.h)
            self.h = None

    def dslash(self, mass, inp, eo_out, eo_in, out=None):
        inp = f64(inp)
        out = np.zeros_like(inp) if out is None else out
        lib().or_dslash(self.h, mass, _p(out), _p(inp), eo_out, eo_in)
        return out

    def dslash_dir(self, mu, fb, wtfat, wtlong, inp, eo_out, out):
        lib().or_dslash_dir(self.h, mu, fb, wtfat, wtlong, _p(out), _p(f64(inp)), eo_out)
        return out

    def ddagd(self, mass, inp, eo):
        inp = f64(inp)
        out = np.zeros_like(inp)
        lib().or_ddagd(self.h, mass, _p(out), _p(inp), eo)
        return out

    def ddagd_norm2(self, mass, inp, eo):
        inp = f64(inp)
        out = np.zeros_like(inp)
        n = lib().or_ddagd_norm2(self.h, mass, _p(out), _p(inp), eo)
        return out, n

    def check_op(self, mass, inp):
        return lib().or_check_op(self.h, mass, _p(f64(inp)), _p4(self.fat),
                                 _p4(self.lng) if self.lng is not None else None)

    def relnorm2(self, r, x, eo):
        return lib().or_relnorm2(self.lat.h, _p(f64(r)), _p(f64(x)), eo)

    def invert(self, mass, inp, inv_arg, res_arg, out=None):
        inp = f64(inp)
        out = np.zeros_like(inp) if out is None else f64(out).copy()
        flop = C.c_double(0)
        lib().or_invert(self.h, C.byref(inv_arg), C.byref(res_arg), mass, _p(out), _p(inp), C.byref(flop))
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
        lib().or_invert_multi(self.h, C.byref(inv_arg), ra, mp, nm, op, ip_, nsrc, C.byref(flop))
        return outs, flop.value


def set_threads(n):
    lib().or_set_threads(int(n))


def get_threads():
    return lib().or_get_threads()
