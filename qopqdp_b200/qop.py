"""ctypes mirror of the QOP C interface exported by libqop_b200.so.

The structs below are the reference's include/qop_int.h structs, member for
member.  `Qop(prec)` binds the F3 ('F', float32) or D3 ('D', float64) entry
points and accepts numpy arrays in the reference raw layout:

    vector : float array of shape (V, 3, 2)      (QLA_ColorVector per site)
    links  : 4 float arrays of shape (V, 3, 3, 2) (QLA_ColorMatrix per site)

in raw site order (even sites first, lib/layout_user.c:237-258).  The
library is loaded from the package directory; there is no fallback.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libqop_b200.so")

QOP_SUCCESS, QOP_FAIL, QOP_BC_ERROR, QOP_MEM_ERROR = 0, 1, 2, 3
QOP_EVEN, QOP_ODD, QOP_EVENODD = 0, 1, 2
QOP_UNITARIZE_U3, QOP_UNITARIZE_SU3 = 0, 1
QOP_UNITARIZE_NONE, QOP_UNITARIZE_RATIONAL, QOP_UNITARIZE_ANALYTIC = 0, 3, 5
QOP_MAX_NAIK = 20


class QOP_layout_t(C.Structure):
    _fields_ = [("node_number", C.c_void_p), ("node_index", C.c_void_p), ("latdim", C.c_int),
                ("latsize", C.POINTER(C.c_int)), ("machdim", C.c_int), ("machsize", C.POINTER(C.c_int)),
                ("this_node", C.c_int), ("sites_on_node", C.c_int)]


class QOP_Complex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class QOP_bc_t(C.Structure):
    _fields_ = [("phase", C.POINTER(QOP_Complex))]


class QOP_staggered_sign_t(C.Structure):
    _fields_ = [("signmask", C.POINTER(C.c_int))]


class QOP_opt_t(C.Structure):
    _fields_ = [("tag", C.c_char_p), ("value", C.c_double), ("extra", C.c_void_p)]


class QOPB_request_t(C.Structure):
    """One request of the solve service (include/qop_b200.h)."""
    _fields_ = [("links", C.c_void_p), ("lattice", C.c_int), ("evenodd", C.c_int), ("mass", C.c_double),
                ("rsqmin", C.c_double), ("max_iter", C.c_int), ("nrhs", C.c_int),
                ("src", C.POINTER(C.POINTER(C.c_double))), ("dst", C.POINTER(C.POINTER(C.c_double)))]


class QOPB_result_t(C.Structure):
    _fields_ = [("status", C.c_int), ("iters_max", C.c_int), ("final_rsq_max", C.c_double),
                ("queue_ms", C.c_double), ("solve_ms", C.c_double), ("total_ms", C.c_double),
                ("batch_systems", C.c_int)]


class QOP_info_t(C.Structure):
    _fields_ = [("final_sec", C.c_double), ("final_flop", C.c_double), ("status", C.c_int),
                ("count1", C.c_int), ("count2", C.c_int)]


class QOP_invert_arg_t(C.Structure):
    _fields_ = [("mixed_rsq", C.c_double), ("max_iter", C.c_int), ("restart", C.c_int),
                ("max_restarts", C.c_int), ("evenodd", C.c_int)]

    @classmethod
    def default(cls):
        # QOP_INVERT_ARG_DEFAULT (include/qop_int.h:126)
        return cls(1e9, 2000, 1000, 5, QOP_EVENODD)


class QOP_resid_arg_t(C.Structure):
    _fields_ = [("rsqmin", C.c_double), ("final_rsq", C.c_double), ("relmin", C.c_double),
                ("final_rel", C.c_double), ("final_iter", C.c_int), ("final_restart", C.c_int)]

    @classmethod
    def default(cls):
        # QOP_RESID_ARG_DEFAULT (include/qop_int.h:137)
        return cls(1e-6, 0, 0, 0, 0, 0)


class QOP_asqtad_coeffs_t(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("one_link", "three_staple", "five_staple", "seven_staple", "lepage", "naik")]


class QOP_hisq_coeffs_t(C.Structure):
    _fields_ = [("n_naiks", C.c_int), ("eps_naik", C.c_double * QOP_MAX_NAIK), ("ugroup", C.c_int),
                ("umethod", C.c_int)] + [(n, C.c_double) for n in (
                    "fat7_one_link", "fat7_three_staple", "fat7_five_staple", "fat7_seven_staple", "fat7_lepage",
                    "asqtad_one_link", "asqtad_three_staple", "asqtad_five_staple", "asqtad_seven_staple",
                    "asqtad_lepage", "asqtad_naik", "difference_one_link", "difference_naik")]


_lib = None


def load_library(path=None):
    """Load libqop_b200.so once; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError("libqop_b200.so not built (%s); run python -m qopqdp_b200.build" % path)
    lib = C.CDLL(path)
    vp, ip = C.c_void_p, C.c_int
    lib.QOP_init.argtypes = [C.POINTER(QOP_layout_t)]
    lib.QOP_init.restype = ip
    lib.QOP_finalize.restype = ip
    lib.QOP_is_initialized.restype = ip
    lib.QOP_version_str.restype = C.c_char_p
    lib.QOP_version_int.restype = ip
    lib.QOP_verbose.argtypes = [ip]
    lib.QOP_verbose.restype = ip
    lib.QOP_node_index_raw_V.argtypes = [C.POINTER(C.c_int), ip]
    lib.QOP_node_index_raw_V.restype = ip
    lib.QOP_sites_on_node_raw_V.argtypes = [ip]
    lib.QOP_sites_on_node_raw_V.restype = ip
    lib.QOPB_comm_unique_id.argtypes = [C.POINTER(C.c_ubyte)]
    lib.QOPB_comm_init.argtypes = [C.POINTER(C.c_ubyte), ip, ip]
    lib.QOPB_dd_info.argtypes = [C.POINTER(C.c_int)] * 3 + [C.POINTER(C.c_int)]
    lib.QOPB_layout_hyper.argtypes = [C.POINTER(C.c_int), ip, C.POINTER(C.c_int)]
    lib.QOPB_layout_node_number.argtypes = [C.POINTER(C.c_int)] * 3
    lib.QOPB_layout_node_index.argtypes = [C.POINTER(C.c_int)] * 3
    lib.QOPB_layout_node_index.restype = C.c_long
    lib.QOPB_layout_neighbors.argtypes = [C.POINTER(C.c_int), ip, C.POINTER(C.c_int)]
    lib.QOPB_dd_pack_site.argtypes = [C.POINTER(C.c_int), ip, ip, ip, ip, ip, C.POINTER(C.c_int)]
    lib.QOPB_dd_halo_ref.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), ip, ip, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]
    lib.QOPB_lattice_create.argtypes = [C.POINTER(C.c_int)]
    lib.QOPB_lattice_create.restype = ip
    lib.QOPB_lattice_use.argtypes = [ip]
    lib.QOPB_lattice_use.restype = ip
    lib.QOPB_lattice_current.restype = ip
    lib.QOPB_serve_start.restype = ip
    lib.QOPB_serve_stop.restype = ip
    lib.QOPB_serve_submit.argtypes = [C.POINTER(QOPB_request_t)]
    lib.QOPB_serve_submit.restype = C.c_longlong
    lib.QOPB_serve_wait.argtypes = [C.c_longlong, C.c_double, C.POINTER(QOPB_result_t)]
    lib.QOPB_serve_wait.restype = ip
    for f in ("QOP_asqtad_invert_set_opts", "QOP_hisq_links_set_opts", "QOP_hisq_invert_set_opts",
              "QOP_asqtad_force_set_opts"):
        getattr(lib, f).argtypes = [C.POINTER(QOP_opt_t), ip]
        getattr(lib, f).restype = ip
    for pc, real in (("F3", C.c_float), ("D3", C.c_double)):
        rp = C.POINTER(real)
        rpp = C.POINTER(rp)
        info = C.POINTER(QOP_info_t)

        def sig(name, args, res=None):
            fn = getattr(lib, "QOP_%s_%s" % (pc, name))
            fn.argtypes = args
            fn.restype = res

        sig("create_V_from_raw", [rp, ip], vp)
        sig("extract_V_to_raw", [rp, vp, ip])
        sig("destroy_V", [vp])
        sig("create_G_from_raw", [rpp, ip], vp)
        sig("create_F_from_raw", [rpp, ip], vp)
        sig("extract_F_to_raw", [rpp, vp, ip])
        sig("destroy_F", [vp])
        sig("asqtad_force_multi", [info, vp, vp, C.POINTER(QOP_asqtad_coeffs_t), rp, C.POINTER(vp), ip])
        sig("hisq_force_multi", [info, vp, vp, C.POINTER(QOP_hisq_coeffs_t), rp, C.POINTER(vp), C.POINTER(ip)])
        sig("extract_G_to_raw", [rpp, vp, ip])
        sig("destroy_G", [vp])
        sig("rephase_G", [vp, C.POINTER(C.c_int), C.POINTER(QOP_bc_t), C.POINTER(QOP_staggered_sign_t)])
        sig("asqtad_create_L_from_raw", [rpp, rpp, ip], vp)
        sig("asqtad_create_L_from_G", [info, C.POINTER(QOP_asqtad_coeffs_t), vp], vp)
        sig("asqtad_create_L_from_G2", [info, C.POINTER(QOP_asqtad_coeffs_t), vp, vp], vp)
        sig("asqtad_load_L_from_raw", [vp, rpp, rpp, ip])
        sig("asqtad_extract_L_to_raw", [rpp, rpp, vp, ip])
        sig("asqtad_destroy_L", [vp])
        sig("asqtad_rephase_L", [vp, C.POINTER(C.c_int), C.POINTER(QOP_bc_t), C.POINTER(QOP_staggered_sign_t)])
        sig("asqtad_dslash", [info, vp, real, vp, vp, ip, ip])
        sig("asqtad_dslash_dir", [info, vp, ip, ip, C.c_double, C.c_double, vp, vp, ip])
        sig("asqtad_diaginv", [info, vp, real, vp, vp, ip])
        sig("asqtad_ddagd", [info, vp, real, vp, vp, ip])
        sig("asqtad_ddagd_norm2", [info, vp, real, vp, vp, ip], real)
        sig("asqtad_invert", [info, vp, C.POINTER(QOP_invert_arg_t), C.POINTER(QOP_resid_arg_t), real, vp, vp])
        sig("asqtad_invert_multi", [info, vp, C.POINTER(QOP_invert_arg_t),
                                    C.POINTER(C.POINTER(C.POINTER(QOP_resid_arg_t))), C.POINTER(rp),
                                    C.POINTER(C.c_int), C.POINTER(C.POINTER(vp)), C.POINTER(vp), ip])
        sig("hisq_create_L_from_G", [info, C.POINTER(QOP_hisq_coeffs_t), vp], vp)
        sig("hisq_destroy_L", [vp])
        sig("get_asqtad_links_from_hisq", [vp], C.POINTER(vp))
        sig("get_asqtad_deps_links_from_hisq", [vp], vp)
    lib.QOP_FD3_asqtad_create_L_from_L.argtypes = [vp]
    lib.QOP_FD3_asqtad_create_L_from_L.restype = vp
    dp = C.POINTER(C.c_double)
    lib.QOPB_D3_sloppy_ddagd.argtypes = [C.POINTER(QOP_info_t), vp, C.c_double, vp, vp, vp, ip, ip, ip, dp]
    lib.QOPB_D3_sloppy_ddagd.restype = ip
    lib.QOPB_D3_sloppy_ddagd_batch.argtypes = [C.POINTER(QOP_info_t), vp, ip, dp, C.POINTER(vp), C.POINTER(vp),
                                               C.POINTER(vp), ip, ip, dp]
    lib.QOPB_D3_sloppy_ddagd_batch.restype = ip
    _lib = lib
    return lib


def exported_symbols(header=None):
    """Function names declared in include/qop.h (and qop_b200.h)."""
    import re
    root = os.path.dirname(_HERE)
    names = []
    for h in ("qop.h", "qop_b200.h"):
        p = os.path.join(root, "include", h)
        if not os.path.exists(p):
            continue
        txt = open(p).read()
        if h == "qop.h":
            body = txt.split("QOPB_DECLARE_PC(PC, REAL)")[1].split("QOPB_DECLARE_PC(F3")[0]
            pcs = re.findall(r"QOP_##PC##_(\w+)\(", body)
            for pc in ("F3", "D3"):
                names += ["QOP_%s_%s" % (pc, n) for n in pcs]
            txt = txt.replace(body, "")
        names += re.findall(r"^\s*[\w\s\*]+?\b(QOPB?_\w+)\s*\(", txt, re.M)
    return sorted(set(n for n in names if not n.startswith("QOPB_DECLARE") and n != "QOPB_GEN"))


def _c_opts(opts):
    arr = (QOP_opt_t * len(opts))()
    keep = []
    for i, (k, v) in enumerate(opts.items()):
        b = k.encode()
        keep.append(b)
        arr[i].tag = b
        arr[i].value = float(v)
    return arr, keep


class Qop:
    """Bindings for one precision: prec 'F' (QOP_F3_*) or 'D' (QOP_D3_*)."""

    def __init__(self, prec="D"):
        self.lib = load_library()
        self.prec = prec
        self.pc = "F3" if prec == "F" else "D3"
        self.real = C.c_float if prec == "F" else C.c_double
        self.dtype = np.float32 if prec == "F" else np.float64

    def f(self, name):
        return getattr(self.lib, "QOP_%s_%s" % (self.pc, name))

    # ------------------------------------------------------------ library
    def init(self, L, machsize=None):
        """QOP_init; machsize (4 ints) decomposes the lattice over the
        processes of the communicator made by comm_init."""
        ls = (C.c_int * 4)(*L)
        lay = QOP_layout_t()
        lay.latdim = 4
        lay.latsize = ls
        lay.machdim = -1
        if machsize is not None:
            ms = (C.c_int * 4)(*machsize)
            lay.machdim = 4
            lay.machsize = ms
        st = self.lib.QOP_init(C.byref(lay))
        return st

    # ------------------------------------------------------------ decomposition
    def comm_unique_id(self):
        buf = (C.c_ubyte * 128)()
        if self.lib.QOPB_comm_unique_id(buf) != 0:
            raise RuntimeError("QOPB_comm_unique_id failed")
        return bytes(buf)

    def comm_init(self, uid, nranks, rank):
        buf = (C.c_ubyte * 128).from_buffer_copy(uid)
        return self.lib.QOPB_comm_init(buf, nranks, rank)

    def comm_finalize(self):
        return self.lib.QOPB_comm_finalize()

    def dd_self_split(self, mask):
        return self.lib.QOPB_dd_self_split(mask)

    def dd_info(self):
        P, m, loc, mask = (C.c_int * 4)(), (C.c_int * 4)(), (C.c_int * 4)(), C.c_int()
        r = self.lib.QOPB_dd_info(P, m, loc, C.byref(mask))
        return dict(rank=r, nsquares=tuple(P), coords=tuple(m), local=tuple(loc), mask=mask.value)

    def finalize(self):
        return self.lib.QOP_finalize()

    def set_opts(self, **opts):
        arr, _keep = _c_opts(opts)
        return self.lib.QOP_asqtad_invert_set_opts(arr, len(opts))

    def set_hisq_opts(self, **opts):
        arr, _keep = _c_opts(opts)
        return self.lib.QOP_hisq_links_set_opts(arr, len(opts))

    # ------------------------------------------------------------ arrays
    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        return a, a.ctypes.data_as(C.POINTER(self.real))

    def _arr4(self, links):
        keep, ptrs = [], (C.POINTER(self.real) * 4)()
        for i in range(4):
            a, p = self._arr(links[i])
            keep.append(a)
            ptrs[i] = p
        return keep, ptrs

    # ------------------------------------------------------------ fields
    def create_V(self, raw, eo=QOP_EVENODD):
        a, p = self._arr(raw)
        h = self.f("create_V_from_raw")(p, eo)
        if not h:
            raise RuntimeError("create_V_from_raw failed")
        return h

    def extract_V(self, h, V, eo=QOP_EVENODD, into=None):
        out = into if into is not None else np.zeros((V, 3, 2), dtype=self.dtype)
        assert out.dtype == self.dtype and out.flags.c_contiguous
        self.f("extract_V_to_raw")(out.ctypes.data_as(C.POINTER(self.real)), h, eo)
        return out

    def destroy_V(self, h):
        self.f("destroy_V")(h)

    def create_G(self, links, eo=QOP_EVENODD):
        keep, ptrs = self._arr4(links)
        h = self.f("create_G_from_raw")(ptrs, eo)
        if not h:
            raise RuntimeError("create_G_from_raw failed")
        return h

    def extract_G(self, h, V, eo=QOP_EVENODD):
        outs = [np.zeros((V, 3, 3, 2), dtype=self.dtype) for _ in range(4)]
        ptrs = (C.POINTER(self.real) * 4)(*[o.ctypes.data_as(C.POINTER(self.real)) for o in outs])
        self.f("extract_G_to_raw")(ptrs, h, eo)
        return outs

    def create_F(self, fields, eo=QOP_EVENODD):
        keep, ptrs = self._arr4(fields)
        h = self.f("create_F_from_raw")(ptrs, eo)
        if not h:
            raise RuntimeError("create_F_from_raw failed")
        return h

    def extract_F(self, h, V, eo=QOP_EVENODD):
        outs = [np.zeros((V, 3, 3, 2), dtype=self.dtype) for _ in range(4)]
        ptrs = (C.POINTER(self.real) * 4)(*[o.ctypes.data_as(C.POINTER(self.real)) for o in outs])
        self.f("extract_F_to_raw")(ptrs, h, eo)
        return outs

    def destroy_F(self, h):
        self.f("destroy_F")(h)

    def asqtad_force(self, gauge, force, coeffs, eps, vecs, info=None):
        """QOP_*_asqtad_force_multi: force += -2 TA(U deriv^+) for the sources vecs."""
        info = info or QOP_info_t()
        c = QOP_asqtad_coeffs_t(*coeffs)
        e = (self.real * len(eps))(*eps)
        v = (C.c_void_p * len(vecs))(*vecs)
        self.f("asqtad_force_multi")(C.byref(info), gauge, force, C.byref(c), e, v, len(vecs))
        return info

    def hisq_force(self, hisq, force, hcoef, eps, vecs, n_orders, info=None):
        """QOP_*_hisq_force_multi: force += TA(U (2 deriv)^+)."""
        info = info or QOP_info_t()
        e = (self.real * len(eps))(*eps)
        v = (C.c_void_p * len(vecs))(*vecs)
        no = (C.c_int * len(n_orders))(*n_orders)
        self.f("hisq_force_multi")(C.byref(info), hisq, force, C.byref(hcoef), e, v, no)
        return info

    def destroy_G(self, h):
        self.f("destroy_G")(h)

    @staticmethod
    def _phases(r0, bc, signmask):
        r0c = (C.c_int * 4)(*r0)
        ph = (QOP_Complex * 4)(*[QOP_Complex(complex(z).real, complex(z).imag) for z in bc])
        bct = QOP_bc_t(ph)
        sm = (C.c_int * 4)(*signmask)
        sgn = QOP_staggered_sign_t(sm)
        return r0c, ph, bct, sm, sgn

    def rephase_G(self, h, r0=(0, 0, 0, 0), bc=(1, 1, 1, -1), signmask=(0, 1, 3, 7)):
        r0c, ph, bct, sm, sgn = self._phases(r0, bc, signmask)
        self.f("rephase_G")(h, r0c, C.byref(bct), C.byref(sgn))

    # ------------------------------------------------------------ links
    def create_L_from_raw(self, fat, lng, eo=QOP_EVENODD):
        kf, pf = self._arr4(fat)
        if lng is not None:
            kl, pl = self._arr4(lng)
        else:
            pl = None
        h = self.f("asqtad_create_L_from_raw")(pf, pl, eo)
        if not h:
            raise RuntimeError("asqtad_create_L_from_raw failed")
        return h

    def create_L_from_G(self, coeffs, gauge, info=None):
        info = info or QOP_info_t()
        c = QOP_asqtad_coeffs_t(*coeffs)
        h = self.f("asqtad_create_L_from_G")(C.byref(info), C.byref(c), gauge)
        if not h:
            raise RuntimeError("asqtad_create_L_from_G failed (status %d)" % info.status)
        return h

    def extract_L(self, h, V, naik=True, eo=QOP_EVENODD):
        fat = [np.zeros((V, 3, 3, 2), dtype=self.dtype) for _ in range(4)]
        lng = [np.zeros((V, 3, 3, 2), dtype=self.dtype) for _ in range(4)] if naik else None
        pf = (C.POINTER(self.real) * 4)(*[o.ctypes.data_as(C.POINTER(self.real)) for o in fat])
        pl = (C.POINTER(self.real) * 4)(*[o.ctypes.data_as(C.POINTER(self.real)) for o in lng]) if naik else None
        self.f("asqtad_extract_L_to_raw")(pf, pl, h, eo)
        return fat, lng

    def load_L_from_raw(self, h, fat, lng, eo=QOP_EVENODD):
        kf, pf = self._arr4(fat)
        pl = self._arr4(lng)[1] if lng is not None else None
        self.f("asqtad_load_L_from_raw")(h, pf, pl, eo)

    def destroy_L(self, h):
        self.f("asqtad_destroy_L")(h)

    def rephase_L(self, h, r0=(0, 0, 0, 0), bc=(1, 1, 1, -1), signmask=(0, 1, 3, 7)):
        r0c, ph, bct, sm, sgn = self._phases(r0, bc, signmask)
        self.f("asqtad_rephase_L")(h, r0c, C.byref(bct), C.byref(sgn))

    def hisq_create_L_from_G(self, hc, gauge, info=None):
        info = info or QOP_info_t()
        h = self.f("hisq_create_L_from_G")(C.byref(info), C.byref(hc), gauge)
        if not h:
            raise RuntimeError("hisq_create_L_from_G failed (status %d)" % info.status)
        return h

    def hisq_asqtad_links(self, hh, k=0):
        return self.f("get_asqtad_links_from_hisq")(hh)[k]

    def hisq_destroy_L(self, hh):
        self.f("hisq_destroy_L")(hh)

    # ------------------------------------------------------------ operators
    def dslash(self, fla, mass, out, inp, eo_out, eo_in, info=None):
        info = info or QOP_info_t()
        self.f("asqtad_dslash")(C.byref(info), fla, self.real(mass), out, inp, eo_out, eo_in)
        return info

    def dslash_dir(self, fla, mu, fb, wtfat, wtlong, out, inp, eo_out, info=None):
        info = info or QOP_info_t()
        self.f("asqtad_dslash_dir")(C.byref(info), fla, mu, fb, wtfat, wtlong, out, inp, eo_out)
        return info

    def diaginv(self, fla, mass, out, inp, eo, info=None):
        info = info or QOP_info_t()
        self.f("asqtad_diaginv")(C.byref(info), fla, self.real(mass), out, inp, eo)
        return info

    def ddagd(self, fla, mass, out, inp, eo, info=None):
        info = info or QOP_info_t()
        self.f("asqtad_ddagd")(C.byref(info), fla, self.real(mass), out, inp, eo)
        return info

    def ddagd_norm2(self, fla, mass, out, inp, eo, info=None):
        info = info or QOP_info_t()
        return self.f("asqtad_ddagd_norm2")(C.byref(info), fla, self.real(mass), out, inp, eo)

    def sloppy_ddagd(self, fla, mass, t_out, ap_out, inp, eo, variant=25, kind2=3):
        """int16 operator of the mixed solver: returns (status, [|t|^2, |p|^2, <p,Ap>, |Ap|^2])."""
        info = QOP_info_t()
        sums = (C.c_double * 4)()
        self.lib.QOPB_D3_sloppy_ddagd(C.byref(info), fla, mass, t_out, ap_out, inp, eo, variant, kind2, sums)
        return info.status, list(sums)

    def sloppy_ddagd_batch(self, fla, masses, t_outs, ap_outs, ins, eo, variant=-1):
        """batched int16 operator: returns (status, [(|t_j|^2, <p_j, A_j p_j>)])."""
        n = len(ins)
        info = QOP_info_t()
        sums = (C.c_double * (2 * n))()
        arr = lambda hs: (C.c_void_p * n)(*hs)
        self.lib.QOPB_D3_sloppy_ddagd_batch(C.byref(info), fla, n, (C.c_double * n)(*masses), arr(t_outs),
                                            arr(ap_outs), arr(ins), eo, variant, sums)
        return info.status, [(sums[2 * j], sums[2 * j + 1]) for j in range(n)]

    def invert(self, fla, mass, out, inp, inv_arg, res_arg, info=None):
        info = info or QOP_info_t()
        self.f("asqtad_invert")(C.byref(info), fla, C.byref(inv_arg), C.byref(res_arg), self.real(mass), out, inp)
        return info

    def invert_multi(self, fla, masses, outs, ins, inv_arg, res_args, info=None):
        """masses[s][j], outs[s][j] (handles), ins[s] (handles), res_args[s][j]."""
        info = info or QOP_info_t()
        nsrc = len(ins)
        RA = C.POINTER(QOP_resid_arg_t)
        ra_rows = [(RA * len(r))(*[C.pointer(x) for x in r]) for r in res_args]
        ra = (C.POINTER(RA) * nsrc)(*[C.cast(r, C.POINTER(RA)) for r in ra_rows])
        m_rows = [(self.real * len(m))(*m) for m in masses]
        mp = (C.POINTER(self.real) * nsrc)(*[C.cast(m, C.POINTER(self.real)) for m in m_rows])
        nm = (C.c_int * nsrc)(*[len(m) for m in masses])
        o_rows = [(C.c_void_p * len(o))(*o) for o in outs]
        op = (C.POINTER(C.c_void_p) * nsrc)(*[C.cast(o, C.POINTER(C.c_void_p)) for o in o_rows])
        ip_ = (C.c_void_p * nsrc)(*ins)
        self.f("asqtad_invert_multi")(C.byref(info), fla, C.byref(inv_arg), ra, mp, nm, op, ip_, nsrc)
        return info

    def eigcg_values(self, fla, eo, max_values=1024):
        """Stored eigCG eigenvalues for solve parity eo (ascending)."""
        buf = (C.c_double * max_values)()
        fn = getattr(self.lib, "QOPB_%s_eigcg_values" % self.pc)
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int]
        n = fn(fla, eo, buf, max_values)
        if n < 0:
            raise RuntimeError("QOPB_%s_eigcg_values failed" % self.pc)
        return np.array(buf[:min(n, max_values)])

    # ------------------------------------------------------------ lattices and the solve service
    def lattice_create(self, L):
        return self.lib.QOPB_lattice_create((C.c_int * 4)(*L))

    def lattice_use(self, lat):
        return self.lib.QOPB_lattice_use(lat)

    def serve_start(self):
        self._pending = {}
        return self.lib.QOPB_serve_start()

    def serve_stop(self):
        return self.lib.QOPB_serve_stop()

    def serve_submit(self, fla, lattice, eo, mass, rsqmin, srcs, dsts, max_iter=0):
        """srcs: raw float64 arrays (kept alive here); dsts: preallocated raw
        float64 arrays written by the service.  Returns the ticket (< 0 on error)."""
        n = len(srcs)
        src = [np.ascontiguousarray(a, dtype=np.float64) for a in srcs]
        pp = C.POINTER(C.c_double)
        sp = (pp * n)(*[a.ctypes.data_as(pp) for a in src])
        dp = (pp * n)(*[a.ctypes.data_as(pp) for a in dsts])
        rq = QOPB_request_t(fla, lattice, eo, mass, rsqmin, max_iter, n, sp, dp)
        t = self.lib.QOPB_serve_submit(C.byref(rq))
        if t >= 0:
            self._pending[t] = (src, dsts, sp, dp)
        return t

    def serve_wait(self, ticket, timeout=0.0):
        res = QOPB_result_t()
        rc = self.lib.QOPB_serve_wait(ticket, timeout, C.byref(res))
        if rc == 0:
            self._pending.pop(ticket, None)
        return rc, res


# ---------------------------------------------------------------- layout (host only)
def layout_hyper(L, nranks):
    """The reference's split of lattice L over nranks processes."""
    P = (C.c_int * 4)()
    if load_library().QOPB_layout_hyper((C.c_int * 4)(*L), nranks, P) != 0:
        raise ValueError("bad layout arguments")
    return tuple(P)


def layout_node_number(L, P, x):
    return load_library().QOPB_layout_node_number((C.c_int * 4)(*L), (C.c_int * 4)(*P), (C.c_int * 4)(*x))


def layout_node_index(L, P, x):
    return load_library().QOPB_layout_node_index((C.c_int * 4)(*L), (C.c_int * 4)(*P), (C.c_int * 4)(*x))


def layout_neighbors(P, rank):
    """[(-mu rank, +mu rank) for mu in 0..3]."""
    nb = (C.c_int * 8)()
    load_library().QOPB_layout_neighbors((C.c_int * 4)(*P), rank, nb)
    return [(nb[2 * i], nb[2 * i + 1]) for i in range(4)]


def dd_pack_site(local, mu, nlinks, parity, slab, face):
    """(local site x, link slot or -1) packed at (slab, face) of direction
    mu's halo, from the library's halo plan."""
    x = (C.c_int * 4)()
    slot = load_library().QOPB_dd_pack_site((C.c_int * 4)(*local), mu, nlinks, parity, slab, face, x)
    if slot < -1:
        raise ValueError("bad halo plan arguments")
    return tuple(x), slot


def dd_halo_ref(local, x, mu, disp):
    """Where the hop term (mu, disp) of local site x reads its neighbour:
    None inside the block, else ('up' | 'dn', slab, face)."""
    sl, fc = C.c_int(), C.c_int()
    r = load_library().QOPB_dd_halo_ref((C.c_int * 4)(*local), (C.c_int * 4)(*x), mu, disp, C.byref(sl), C.byref(fc))
    if r < 0:
        raise ValueError("bad halo plan arguments")
    return None if r == 0 else ("up" if r == 1 else "dn", sl.value, fc.value)
