"""FP64 reference for the int16 sloppy operator (test infrastructure).

The mixed solvers store links and site vectors as 16-bit fixed point with a
per-site / per-link scale (component q = round(32767 x / s), s the largest
|re|, |im|; Naik links whose products are |c| x unitary keep rows 0-1 over
the lattice-wide |c| and rebuild row 2 from the phase of the determinant).
This module reproduces that quantisation on the host, so that the device's
int16 hop can be compared with the exact operator applied to exactly the
values the device stores: the remaining difference is the FP32 arithmetic
and the rounding of the output to int16.

Links follow the reference's double-stored order (lib/asqtad_dslash_p.c:79-133):
slot 4 mu + {fat fwd, long fwd, fat bck, long bck} with displacements
{+1, +3, -1, -3} along mu, every link times 1/2 (:201-206), a backward link
bck(x) = -fwd(x - d mu)^+.  Vectors are raw arrays (V, 3, 2) in the
reference's raw site order (lib/layout_user.c:237-258).
"""
import numpy as np

from qopqdp_b200 import lattice as LT

F32 = np.float32


def cplx(a):
    return np.asarray(a, dtype=np.float64)[..., 0] + 1j * np.asarray(a, dtype=np.float64)[..., 1]


class Geometry:
    """Neighbour tables in raw site order."""

    def __init__(self, L):
        self.L = tuple(L)
        self.V = LT.volume(L)
        self.x = LT.raw_coords(L)
        self.nbr = {}
        for mu in range(4):
            for d in (1, 3, -1, -3):
                y = self.x.copy()
                y[:, mu] = (y[:, mu] + d) % L[mu]
                self.nbr[(mu, d)] = LT.raw_index(L, y)

    def slots(self):
        """(mu, displacement) of the 16 double-stored slots."""
        return [(k // 4, (1, 3, -1, -3)[k % 4]) for k in range(16)]


def dbl_links(geo, fat, lng):
    """16 complex (V, 3, 3) arrays: the double-stored links times 1/2."""
    out = []
    for mu in range(4):
        f = 0.5 * cplx(fat[mu])
        l = 0.5 * cplx(lng[mu])
        out += [f, l,
                -np.conj(np.swapaxes(f[geo.nbr[(mu, -1)]], 1, 2)),
                -np.conj(np.swapaxes(l[geo.nbr[(mu, -3)]], 1, 2))]
    return out


def _q16(x, inv):
    """round-to-nearest-even of x * inv in float32, clamped to +-32767."""
    q = np.rint((x.astype(F32) * inv).astype(F32))
    return np.clip(q, -32767, 32767)


def quantize_vector(v):
    """int16 site vectors as stored and decoded (in float32, as the device
    decodes them): (V, 3) complex -> (V, 3) complex."""
    re, im = v.real.astype(F32), v.imag.astype(F32)
    m = np.maximum(np.abs(re).max(axis=1), np.abs(im).max(axis=1)).astype(F32)
    inv = np.where(m > 0, F32(32767.0) / np.where(m > 0, m, F32(1)), F32(0)).astype(F32)[:, None]
    c = (m * (F32(1.0) / F32(32767.0))).astype(F32)[:, None]
    dec = lambda q: (q.astype(F32) * c).astype(F32).astype(np.float64)
    return dec(_q16(re, inv)) + 1j * dec(_q16(im, inv))


def _bf16(x):
    """float32 -> bfloat16 (round to nearest even), returned as float32"""
    b = np.asarray(x, dtype=F32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(F32)


def split_vector(v):
    """site vectors as the tensor-core batched solver stores them: float32
    values split into bf16 hi + lo (hi + lo is exact in float32)."""
    def one(x):
        x = x.astype(F32)
        hi = _bf16(x)
        lo = _bf16((x - hi).astype(F32))
        return hi.astype(np.float64) + lo.astype(np.float64)
    return one(v.real) + 1j * one(v.imag)


def _recon_ok(longs):
    """the device's test for rebuilding row 2: unitarity defect and |c| spread below 1e-7."""
    c2 = np.concatenate([(np.abs(u[:, 0, :]) ** 2).sum(axis=1) for u in longs])
    d = 0.0
    for u in longs:
        g = np.einsum("vaj,vbj->vab", u, np.conj(u)) / ((np.abs(u[:, 0, :]) ** 2).sum(axis=1))[:, None, None]
        d = max(d, float(np.abs(g.real - np.eye(3)).max()), float(np.abs(g.imag).max()))
    c = np.sqrt(c2)
    return d < 1e-7 and (c.max() - c.min()) <= 1e-7 * c.max(), float(c.max())


def quantize_links(dbl):
    """the int16 link copy as decoded by the hop: 16 complex (V, 3, 3) arrays."""
    longs = [dbl[k] for k in range(1, 16, 2)]
    recon, c_long = _recon_ok(longs)
    out = []
    for k, u in enumerate(dbl):
        if recon and k % 2 == 1:
            inv = F32(32767.0 / c_long)
            rows = _q16(u[:, :2, :].real, inv) + 1j * _q16(u[:, :2, :].imag, inv)   # integer units
            det = np.linalg.det(u)
            ph = np.angle(det).astype(F32).astype(np.float64)
            r0, r1 = rows[:, 0, :] / 32767.0, rows[:, 1, :] / 32767.0
            r2 = np.exp(1j * ph)[:, None] * np.conj(np.cross(r0, r1))
            out.append(c_long * np.stack([r0, r1, r2], axis=1))
        else:
            re, im = u.real.astype(F32), u.imag.astype(F32)
            m = np.maximum(np.abs(re).reshape(len(u), -1).max(axis=1), np.abs(im).reshape(len(u), -1).max(axis=1))
            m = m.astype(F32)
            inv = np.where(m > 0, F32(32767.0) / np.where(m > 0, m, F32(1)), F32(0)).astype(F32)[:, None, None]
            c = (m.astype(np.float64) * float(F32(1.0) / F32(32767.0)))[:, None, None]
            out.append(_q16(re, inv) * c + 1j * _q16(im, inv) * c)
    return out, recon


def hop(geo, links, v, sites):
    """(sum_k U_k(x) v(x + d_k mu_k), sum_k |U_k(x)|_F |v(x + d_k mu_k)|) for raw sites `sites`."""
    acc = np.zeros((len(sites), 3), dtype=np.complex128)
    mag = np.zeros(len(sites))
    for k, (mu, d) in enumerate(geo.slots()):
        w = v[geo.nbr[(mu, d)][sites]]
        u = links[k][sites]
        acc += np.einsum("vab,vb->va", u, w)
        mag += np.sqrt((np.abs(u) ** 2).sum(axis=(1, 2))) * np.sqrt((np.abs(w) ** 2).sum(axis=1))
    return acc, mag


def parity_sites(V, eo):
    return np.arange(0, V // 2) if eo == 0 else np.arange(V // 2, V)


def site_err(got, ref, mag, out_scale=4e-5, acc_scale=1e-6):
    """max over sites of |got - ref| / (out_scale |ref| + acc_scale mag): <= 1 passes.

    out_scale covers the int16 rounding of the stored output (half a unit of
    15 bits on each of 6 components: sqrt(6)/2/32767 = 3.7e-5 of the site
    norm), acc_scale the FP32 products and sums over 16 terms."""
    e = np.sqrt((np.abs(got - ref) ** 2).sum(axis=1))
    r = np.sqrt((np.abs(ref) ** 2).sum(axis=1))
    return float((e / (out_scale * r + acc_scale * mag + 1e-300)).max())
