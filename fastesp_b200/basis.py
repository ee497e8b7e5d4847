"""Cartesian Gaussian basis and Cartesian density matrix (host side).

Conventions follow fastesp (fastesp/basis.py), because a MOLDEN file written by
ORCA only reproduces its density under exactly these:

* Cartesian component order of a shell: ``x`` fastest-decreasing,
  (l,0,0), (l-1,1,0), (l-1,0,1), ... (fastesp/basis.py:27-39).
* MOLDEN contraction coefficients already carry the radial factor
  ``N_s(a,l) = (2a/pi)^{3/4} (4a)^{l/2}`` and no angular factor, so every
  Cartesian component of a shell shares the file's coefficients
  (fastesp/basis.py:53-66, 221-233).
* Spherical functions are real solid harmonics in MOLDEN order
  m = 0, +1, -1, +2, -2, ... with the f-shell m = +-3 functions carrying the
  opposite sign to the textbook form (fastesp/basis.py:119-142), each row
  normalised in the Cartesian overlap metric so that ``T S T^T = 1``
  (fastesp/basis.py:145-163).

The solid harmonics are generated here from the closed-form expansion of real
solid harmonics (Helgaker, Jorgensen, Olsen, *Molecular Electronic-Structure
Theory*, eqs. 6.4.48-6.4.50) rather than tabulated, so any l works.
"""
from __future__ import annotations

from functools import lru_cache
from math import comb, pi

import numpy as np

from .molden import Shell, Wavefunction


@lru_cache(maxsize=None)
def cart_order(l: int) -> tuple:
    """Cartesian exponent triples of an l-shell in the MOLDEN/fastesp order."""
    return tuple((lx, ly, l - lx - ly)
                 for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1))


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def primitive_norm(alpha, lx: int, ly: int, lz: int):
    """Radial prefactor ``(2a/pi)^{3/4} (4a)^{l/2}`` already in MOLDEN coefficients."""
    l = lx + ly + lz
    return (2.0 * alpha / pi) ** 0.75 * (4.0 * alpha) ** (0.5 * l)


def _dfact(n: int) -> float:
    """n!! with (-1)!! = 0!! = 1."""
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


@lru_cache(maxsize=None)
def cartesian_overlap_block(l: int) -> np.ndarray:
    """Overlap of same-centre, same-exponent MOLDEN-normalised components of an l-shell.

    With g_i = N_s(a,l) x^i y^j z^k exp(-a r^2) the block does not depend on a;
    each 1-D factor is int x^n exp(-2a x^2) dx = (n-1)!! / (4a)^{n/2} sqrt(pi/(2a)).
    """
    comps = cart_order(l)
    a = 1.0
    pref = primitive_norm(a, l, 0, 0) ** 2 * (pi / (2.0 * a)) ** 1.5
    s = np.zeros((len(comps), len(comps)))
    for i, ci in enumerate(comps):
        for j, cj in enumerate(comps):
            v = pref
            for k in range(3):
                n = ci[k] + cj[k]
                if n % 2:
                    v = 0.0
                    break
                v *= _dfact(n - 1) / (4.0 * a) ** (n // 2)
            s[i, j] = v
    return s


# Sign convention of the stored spherical functions relative to the textbook
# real solid harmonics: ORCA's f functions with |m| = 3 are negated
# (fastesp/basis.py:130-131).  Every other (l, m) keeps the textbook sign.
_MOLDEN_PHASE = {(3, 3): -1.0, (3, -3): -1.0}


@lru_cache(maxsize=None)
def solid_harmonic(l: int, m: int) -> dict:
    """Unnormalised real solid harmonic S_lm as {(lx,ly,lz): coefficient}.

    Closed form (Helgaker-Jorgensen-Olsen eq. 6.4.48-6.4.50): with v_m = 0 for
    m >= 0 and 1/2 for m < 0,
    S_lm ~ sum_{t,u,v} (-1)^{t+v-v_m} 4^{-t} C(l,t) C(l-t,|m|+t) C(t,u) C(|m|,2v)
           x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|}.
    v is carried as the integer w = 2v.
    """
    am = abs(m)
    wm = 0 if m >= 0 else 1
    out: dict = {}
    for t in range((l - am) // 2 + 1):
        for u in range(t + 1):
            for w in range(wm, am + 1, 2):
                c = ((-1.0) ** (t + (w - wm) // 2) * 0.25 ** t * comb(l, t)
                     * comb(l - t, am + t) * comb(t, u) * comb(am, w))
                key = (2 * t + am - 2 * u - w, 2 * u + w, l - 2 * t - am)
                out[key] = out.get(key, 0.0) + c
    ph = _MOLDEN_PHASE.get((l, m), 1.0)
    return {k: ph * v for k, v in out.items() if v != 0.0}


def molden_m_order(l: int) -> list:
    """m values of the stored spherical functions: 0, +1, -1, +2, -2, ..."""
    out = [0]
    for k in range(1, l + 1):
        out += [k, -k]
    return out


@lru_cache(maxsize=None)
def pure_to_cartesian(l: int) -> np.ndarray:
    """T (2l+1, ncart): rows are S-orthonormal MOLDEN solid harmonics (identity for l<=1)."""
    comps = cart_order(l)
    if l <= 1:
        return np.eye(len(comps))
    col = {c: i for i, c in enumerate(comps)}
    v = np.zeros((2 * l + 1, len(comps)))
    for r, m in enumerate(molden_m_order(l)):
        for key, c in solid_harmonic(l, m).items():
            v[r, col[key]] = c
    s = cartesian_overlap_block(l)
    nrm = np.sqrt(np.einsum("ri,ij,rj->r", v, s, v))
    return v / nrm[:, None]


class Basis:
    """Cartesian basis built from a wavefunction's shells (fastesp/basis.py:207-238).

    Attributes mirror the reference: per Cartesian function ``centers``,
    ``atoms``, ``ang`` / ``ang_arr``, ``exps``, ``coefs``, ``shell_of``; plus the
    wavefunction's ``shells`` and ``n`` (number of Cartesian functions).
    """

    def __init__(self, wfn: Wavefunction, use_primitive_norm: bool = True):
        self.wfn = wfn
        self.use_primitive_norm = use_primitive_norm
        centers, atoms, ang, exps, coefs, shell_of = [], [], [], [], [], []
        for s_idx, sh in enumerate(wfn.shells):
            for comp in cart_order(sh.l):
                centers.append(wfn.coords[sh.atom])
                atoms.append(sh.atom)
                ang.append(comp)
                exps.append(np.asarray(sh.exps, dtype=np.float64))
                coefs.append(np.asarray(sh.coeffs, dtype=np.float64))
                shell_of.append(s_idx)
        self.shells = list(wfn.shells)
        self.n = len(centers)
        self.centers = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
        self.atoms = np.asarray(atoms, dtype=np.int32)
        self.ang = ang
        self.ang_arr = np.asarray(ang, dtype=np.int32).reshape(-1, 3)
        self.exps = exps
        self.coefs = coefs
        self.shell_of = shell_of

    def shell_offsets(self) -> np.ndarray:
        """First Cartesian function index of every shell."""
        n = [ncart(sh.l) for sh in self.shells]
        return np.concatenate([[0], np.cumsum(n)[:-1]]).astype(np.int64)

    def block_transform(self) -> np.ndarray:
        """(n_cart, n_spherical) map from stored coefficients to Cartesian ones."""
        nsph = sum(2 * sh.l + 1 for sh in self.shells)
        t = np.zeros((self.n, nsph))
        oc = os_ = 0
        for sh in self.shells:
            nc, ns = ncart(sh.l), 2 * sh.l + 1
            t[oc:oc + nc, os_:os_ + ns] = pure_to_cartesian(sh.l).T
            oc += nc
            os_ += ns
        return t

    def density_matrix_cartesian(self, min_occ: float = 1e-10, device=None):
        """P_cart = T (C_occ n C_occ^T) T^T (fastesp/basis.py:264-270).

        With ``device`` (a CUDA device) the two products run there as FP64
        GEMMs and the result is a CUDA tensor; otherwise NumPy."""
        w = self.wfn
        occ = w.mo_occ > min_occ
        c = w.mo_coeff[:, occ] * np.sqrt(w.mo_occ[occ])[None, :]
        t = self.block_transform()
        if device is not None:
            import torch
            tc = torch.as_tensor(t, device=device) @ torch.as_tensor(c, device=device)
            return tc @ tc.T
        tc = t @ c
        return tc @ tc.T


def _hermite_e0(la: int, lb: int, p, xpa, xpb):
    """E^{ij}_0 for all i<=la, j<=lb of a batch of 1-D Gaussian products.

    Returns (B, la+1, lb+1).  Standard McMurchie-Davidson recurrence
    E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}.
    """
    b = p.shape[0]
    tm = la + lb
    e = np.zeros((b, la + 1, lb + 1, tm + 2))
    e[:, 0, 0, 0] = 1.0
    ip = 0.5 / p
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                src, x = e[:, i - 1, j], xpa
            else:
                src, x = e[:, i, j - 1], xpb
            dst = e[:, i, j]
            dst[:, 1:tm + 1] += src[:, 0:tm] * ip[:, None]
            dst[:, 0:tm + 1] += x[:, None] * src[:, 0:tm + 1]
            dst[:, 0:tm + 1] += np.arange(1, tm + 2)[None, :] * src[:, 1:tm + 2]
    return e[:, :, :, 0]


def overlap_matrix(b: Basis) -> np.ndarray:
    """Full Cartesian overlap matrix, vectorised over shell pairs of equal (la, lb)."""
    shells = b.shells
    coords = b.wfn.coords
    off = b.shell_offsets()
    s = np.zeros((b.n, b.n))
    by_l: dict = {}
    for i, sh in enumerate(shells):
        by_l.setdefault(sh.l, []).append(i)
    for la, ia in by_l.items():
        for lb, ib in by_l.items():
            rows = []
            for i in ia:
                for j in ib:
                    si, sj = shells[i], shells[j]
                    for a, (ea, ca) in enumerate(zip(si.exps, si.coeffs)):
                        for bb, (eb, cb) in enumerate(zip(sj.exps, sj.coeffs)):
                            rows.append((i, j, ea, ca, eb, cb))
            if not rows:
                continue
            arr = np.array([(r[2], r[3], r[4], r[5]) for r in rows])
            si_idx = np.array([r[0] for r in rows])
            sj_idx = np.array([r[1] for r in rows])
            ea, ca, eb, cb = arr.T
            A = coords[[shells[i].atom for i in si_idx]]
            B = coords[[shells[j].atom for j in sj_idx]]
            p = ea + eb
            P = (ea[:, None] * A + eb[:, None] * B) / p[:, None]
            ab2 = ((A - B) ** 2).sum(1)
            kab = np.exp(-ea * eb / p * ab2) * (pi / p) ** 1.5 * ca * cb
            ex = [_hermite_e0(la, lb, p, P[:, k] - A[:, k], P[:, k] - B[:, k])
                  for k in range(3)]
            ca_ = cart_order(la)
            cb_ = cart_order(lb)
            vals = np.empty((len(rows), len(ca_), len(cb_)))
            for u, (ax, ay, az) in enumerate(ca_):
                for v, (bx, by, bz) in enumerate(cb_):
                    vals[:, u, v] = (kab * ex[0][:, ax, bx] * ex[1][:, ay, by]
                                     * ex[2][:, az, bz])
            # accumulate primitive pairs into their shell pair block
            key = si_idx * len(shells) + sj_idx
            uniq, inv = np.unique(key, return_inverse=True)
            acc = np.zeros((len(uniq), len(ca_), len(cb_)))
            np.add.at(acc, inv, vals)
            for q, k in enumerate(uniq):
                i, j = divmod(int(k), len(shells))
                s[off[i]:off[i] + len(ca_), off[j]:off[j] + len(cb_)] = acc[q]
    return s


def build_basis(path, use_primitive_norm: bool = True):
    from .molden import read_molden
    wfn = read_molden(path)
    return wfn, Basis(wfn, use_primitive_norm=use_primitive_norm)


__all__ = ["Basis", "Shell", "cart_order", "ncart", "primitive_norm",
           "cartesian_overlap_block", "pure_to_cartesian", "solid_harmonic",
           "overlap_matrix", "build_basis"]
