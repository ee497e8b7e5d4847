"""CPU oracle for fastesp's exact-ESP path -- TEST INFRASTRUCTURE ONLY.

This module restates, in NumPy, the reference algorithm that the CUDA kernels
of ``fastesp_b200`` must reproduce.  It is the checker, never the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path (``fastesp_b200``) never imports
or calls anything here and fails loudly when its CUDA library is missing.

Every function cites the reference file:line it follows (paths are inside the
ZidongS/fastesp project).  The restatement is pinned against fixtures generated
by running the reference itself (``tests/golden/make_golden.py``), see
``tests/test_oracle_pins.py``.

Third-party arithmetic used by the reference and kept here: the Boys function
through ``scipy.special.hyp1f1`` (fastesp/ints.py:30,39) and NumPy
``einsum``/``matmul`` for the density-weighted contraction (fastesp/esp.py:247-248).
"""
from __future__ import annotations

import struct
from functools import lru_cache
from math import pi

import numpy as np
from scipy.special import hyp1f1

# M_n = int |He_n(x)| exp(-x^2/2) dx; screening-bound moments (fastesp/esp.py:25-28)
M_ABS = np.array([2.5066282746310002, 2.0, 1.5957691216057308, 4.0,
                  10.212920779565312, 33.63284766793385, 136.5963625280984,
                  665.1416330443616, 3768.863619586618, 25506.330595911374,
                  202331.81842358326, 1872154.2572862155])


@lru_cache(maxsize=None)
def cart_order(l: int) -> tuple:
    """Cartesian component order (fastesp/basis.py:27-39)."""
    return tuple((lx, ly, l - lx - ly)
                 for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1))


def boys(m, T):
    """F_m(T) = 1F1(m+1/2; m+3/2; -T)/(2m+1) (fastesp/ints.py:35-40)."""
    m = np.asarray(m)
    T = np.asarray(T, dtype=np.float64)
    out = hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1)
    return out if out.ndim else float(out)


@lru_cache(maxsize=None)
def a_table(lmax: int) -> np.ndarray:
    """a[t+1,j] = -a[t,j] + (t-2j+2) a[t,j-1] (fastesp/esp.py:31-41, ints.py:46-59)."""
    a = np.zeros((lmax + 1, lmax // 2 + 2))
    a[0, 0] = 1.0
    for t in range(lmax):
        for j in range(a.shape[1]):
            v = -a[t, j]
            if j >= 1:
                v += (t - 2 * j + 2) * a[t, j - 1]
            a[t + 1, j] = v
    return a


@lru_cache(maxsize=None)
def pair_type(L: int):
    """Per-L map etab[t] -> G[(alpha, m)] (fastesp/esp.py:54-105).

    Returns (M0, w, abs_t, mono, mvals, npow): M0 is (nterm, T^3) with T=L+1,
    keys sorted lexicographically by (ax, ay, az, m); w the |He| moment
    products and abs_t = |t| over flat (tx,ty,tz); mono (nterm,3) alphas,
    mvals = npow = m.
    """
    T = L + 1
    tab = a_table(L)
    terms: dict = {}
    for ax in range(T):
        for ay in range(T):
            for az in range(T):
                lt = ax + ay + az
                if lt > L:
                    continue
                col = ax * T * T + ay * T + az
                sgn = (-1.0) ** lt
                for jx in range(ax // 2 + 1):
                    a1 = tab[ax, jx]
                    if a1 == 0:
                        continue
                    for jy in range(ay // 2 + 1):
                        a2 = tab[ay, jy]
                        if a2 == 0:
                            continue
                        for jz in range(az // 2 + 1):
                            a3 = tab[az, jz]
                            if a3 == 0:
                                continue
                            key = (ax - 2 * jx, ay - 2 * jy, az - 2 * jz, lt - (jx + jy + jz))
                            arr = terms.setdefault(key, np.zeros(T ** 3))
                            arr[col] += sgn * a1 * a2 * a3
    keys = sorted(terms)
    M0 = np.array([terms[k] for k in keys])
    mono = np.array([k[:3] for k in keys], dtype=np.int64)
    mvals = np.array([k[3] for k in keys], dtype=np.int64)
    tt = np.arange(T)
    abs_t = (tt[:, None, None] + tt[None, :, None] + tt[None, None, :]).ravel()
    w = (M_ABS[:T, None, None] * M_ABS[None, :T, None] * M_ABS[None, None, :T]).ravel()
    return M0, w, abs_t, mono, mvals, mvals.copy()


def e1d_all(i: int, j: int, p, xa, xb) -> np.ndarray:
    """Batched 1-D Hermite coefficients E[b, i', j', t] (fastesp/esp.py:108-147)."""
    tmax = i + j
    b = np.shape(p)[0]
    e = np.zeros((b, i + 1, j + 1, tmax + 1))
    xa = np.asarray(xa)[:, None]
    xb = np.asarray(xb)[:, None]
    ip = (1.0 / (2.0 * np.asarray(p)))[:, None]
    e[:, 0, 0, 0] = 1.0
    tap = np.arange(1, tmax + 1) if tmax else np.zeros(0)
    for ii in range(i + 1):
        for jj in range(j + 1):
            if ii == 0 and jj == 0:
                continue
            src = (ii - 1, jj) if ii > 0 else (ii, jj - 1)
            x = xa if ii > 0 else xb
            prev = e[:, src[0], src[1]]
            cur = e[:, ii, jj]
            cur[:, 1:] += prev[:, :-1] * ip
            cur += x * prev
            cur[:, :-1] += tap * prev[:, 1:]
    return e


def _layout(shells):
    off, out = 0, []
    for sh in shells:
        nc = len(cart_order(sh.l))
        out.append((off, nc))
        off += nc
    return out


def primitive_pairs(shells, coords, density) -> dict:
    """Contract every primitive pair into (p, P, K, G, bound, reff, L).

    Pairs come out in the reference's order: shell pairs (si <= sj) in shell
    order, then primitive pairs with the primitive of shell si outer
    (fastesp/esp.py:194-200, 233-238).

    Follows ESPEngine._build/_make_pair (fastesp/esp.py:168-257); the NumPy
    work is batched over all shell pairs with the same (la, lb), which changes
    only the batch size of each array operation, not the per-pair arithmetic.
    """
    coords = np.asarray(coords, dtype=np.float64)
    lay = _layout(shells)
    groups: dict = {}
    for si, (oi, ni) in enumerate(lay):
        for sj in range(si, len(shells)):
            oj, nj = lay[sj]
            blk = density[oi:oi + ni, oj:oj + nj].copy()
            if si != sj:
                blk += density[oj:oj + nj, oi:oi + ni].T
            if np.abs(blk).max() < 1e-15:
                continue
            groups.setdefault((shells[si].l, shells[sj].l), []).append((si, sj, blk))

    out = {k: [] for k in ("p", "P", "K", "G", "bound", "reff", "L", "order", "etab0")}
    for (la, lb), items in groups.items():
        L = la + lb
        M0, wvec, abs_t, _, _, npow = pair_type(L)
        ci, cj = cart_order(la), cart_order(lb)
        kx = np.array([[a[0], b[0]] for a in ci for b in cj])
        ky = np.array([[a[1], b[1]] for a in ci for b in cj])
        kz = np.array([[a[2], b[2]] for a in ci for b in cj])
        rows = []
        for si, sj, blk in items:
            shi, shj = shells[si], shells[sj]
            A, B = coords[shi.atom], coords[shj.atom]
            na, nb = len(shi.exps), len(shj.exps)
            al = np.repeat(np.asarray(shi.exps, float), nb)
            be = np.tile(np.asarray(shj.exps, float), na)
            ca = np.repeat(np.asarray(shi.coeffs, float), nb)
            cb = np.tile(np.asarray(shj.coeffs, float), na)
            ii = np.repeat(np.arange(na), nb)
            jj = np.tile(np.arange(nb), na)
            rows.append((si, sj, blk.ravel(), A, B, al, be, ca, cb, ii, jj))
        si_a = np.concatenate([np.full(len(r[5]), r[0]) for r in rows])
        sj_a = np.concatenate([np.full(len(r[5]), r[1]) for r in rows])
        wgt0 = np.concatenate([np.broadcast_to(r[2], (len(r[5]), len(r[2]))) for r in rows])
        A = np.concatenate([np.broadcast_to(r[3], (len(r[5]), 3)) for r in rows])
        B = np.concatenate([np.broadcast_to(r[4], (len(r[5]), 3)) for r in rows])
        al, be, ca, cb, ii, jj = (np.concatenate([r[k] for r in rows]) for k in range(5, 11))
        ab = A - B
        ab2 = np.einsum("ij,ij->i", ab, ab)
        p = al + be
        P = (al[:, None] * A + be[:, None] * B) / p[:, None]
        XPA, XPB = P - A, P - B
        K = np.exp(-(al * be) / p * ab2)
        sel = K >= 1e-30
        if not sel.any():
            continue
        p, P, XPA, XPB, K = p[sel], P[sel], XPA[sel], XPB[sel], K[sel]
        wgt0, ca, cb = wgt0[sel], ca[sel], cb[sel]
        si_a, sj_a, ii, jj = si_a[sel], sj_a[sel], ii[sel], jj[sel]
        nb_ = p.size
        ex = e1d_all(la, lb, p, XPA[:, 0], XPB[:, 0])
        ey = e1d_all(la, lb, p, XPA[:, 1], XPB[:, 1])
        ez = e1d_all(la, lb, p, XPA[:, 2], XPB[:, 2])
        cw = ca * cb
        wgt = wgt0 * cw[:, None]
        Ax = ex[:, kx[:, 0], kx[:, 1]]
        Ay = ey[:, ky[:, 0], ky[:, 1]]
        Az = ez[:, kz[:, 0], kz[:, 1]]
        etab = np.einsum("qk,qka,qkb,qkc->qabc", wgt, Ax, Ay, Az)
        contrib = etab.reshape(nb_, -1) @ M0.T
        cf = 2.0 * pi / p
        G = cf[:, None] * (2.0 * p)[:, None] ** npow[None, :] * contrib
        powt = (2.0 * p)[:, None] ** (abs_t / 2.0)
        bound = (2.0 * p) ** -1.5 * (np.abs(etab).reshape(nb_, -1) * wvec[None, :] * powt).sum(1)
        reff = 1.6 * np.sqrt((L + 2.0) / p)
        out["p"].append(p)
        out["P"].append(P)
        out["K"].append(K)
        out["G"].extend(list(G))
        out["bound"].append(bound)
        out["reff"].append(reff)
        out["L"].append(np.full(nb_, L))
        out["etab0"].append(etab.reshape(nb_, -1)[:, 0])
        out["order"].append(np.stack([si_a, sj_a, ii, jj], axis=1))
    if not out["p"]:
        return {"n": 0}
    order = np.concatenate(out["order"])
    perm = np.lexsort((order[:, 3], order[:, 2], order[:, 1], order[:, 0]))
    res = {k: np.concatenate(out[k])[perm] for k in ("p", "K", "bound", "reff", "L", "etab0")}
    res["P"] = np.concatenate(out["P"])[perm]
    res["G"] = [out["G"][i] for i in perm]
    res["n"] = len(perm)
    return res


def sum_rule(pp) -> float:
    """Tr(P S) = sum over pairs of K (pi/p)^{3/2} etab[0] (build_pairs.cpp:294-296)."""
    if pp["n"] == 0:
        return 0.0
    return float(np.sum(pp["K"] * (pi / pp["p"]) ** 1.5 * pp["etab0"]))


@lru_cache(maxsize=None)
def mono_schedule(L: int):
    """Monomial closure of the alpha set of class L (fastesp/table.py:198-221).

    Returns (parent, axis, aidx): monomials sorted lexicographically, each
    built as mono[j] = mono[parent[j]] * R[axis[j]] from its first decrementable
    axis; aidx maps every term of ``pair_type(L)`` to its monomial.
    """
    _, _, _, mono, _, _ = pair_type(L)
    grown = set(tuple(map(int, a)) for a in mono)
    changed = True
    while changed:
        changed = False
        for a in list(grown):
            for k in range(3):
                if a[k] > 0:
                    q = a[:k] + (a[k] - 1,) + a[k + 1:]
                    if q not in grown:
                        grown.add(q)
                        changed = True
    order = sorted(grown)
    idx = {a: i for i, a in enumerate(order)}
    parent = np.zeros(len(order), np.int32)
    axis = np.zeros(len(order), np.int32)
    for i, a in enumerate(order):
        for k in range(3):
            if a[k] > 0:
                parent[i] = idx[a[:k] + (a[k] - 1,) + a[k + 1:]]
                axis[i] = k
                break
    aidx = np.array([idx[tuple(map(int, a))] for a in mono], np.int32)
    return parent, axis, aidx


class OracleTable:
    """Flat pair table in the reference's ``pairs.bin`` layout (fastesp/table.py:11-23, 40-62)."""

    FIELDS_F = ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K")
    FIELDS_I = ("pp_nt", "pp_off", "pp_nmono", "pp_monooff")

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def n_pairs(self) -> int:
        return len(self.pp_exp)

    @property
    def n_terms(self) -> int:
        return len(self.tm_g)

    def electron(self, points=None, pair_mask=None) -> np.ndarray:
        """-int rho/|r-C| contribution (fastesp/table.py:73-93), batched over pairs of one class."""
        pts = self.pts if points is None else np.asarray(points, float)
        out = np.zeros(len(pts))
        nt = self.pp_nt
        idx_all = np.arange(self.n_pairs)
        if pair_mask is not None:
            idx_all = idx_all[pair_mask]
        for n in np.unique(nt[idx_all]):
            sel = idx_all[nt[idx_all] == n]
            off0 = self.pp_off[sel]
            mo0 = self.pp_monooff[sel]
            nm = int(self.pp_nmono[sel[0]])
            # all pairs of a class share one schedule and term layout
            par = self.mo_parent[mo0[0]:mo0[0] + nm]
            axs = self.mo_axis[mo0[0]:mo0[0] + nm]
            aidx = self.tm_aidx[off0[0]:off0[0] + n]
            mm = self.tm_m[off0[0]:off0[0] + n]
            g = self.tm_g[off0[:, None] + np.arange(n)[None, :]]          # (np, n)
            for c0 in range(0, len(sel), 2048):
                cs = slice(c0, c0 + 2048)
                P = np.stack([self.pp_cx[sel[cs]], self.pp_cy[sel[cs]], self.pp_cz[sel[cs]]], 1)
                R = pts[None, :, :] - P[:, None, :]                       # (c, N, 3)
                T = self.pp_exp[sel[cs]][:, None] * np.einsum("cij,cij->ci", R, R)
                F = [boys(k, T) for k in range(int(mm.max()) + 1)]
                mono = [np.ones_like(T)]
                for j in range(1, nm):
                    mono.append(mono[par[j]] * R[:, :, axs[j]])
                acc = np.zeros_like(T)
                for k in range(n):
                    acc += g[cs, k][:, None] * mono[aidx[k]] * F[mm[k]]
                out += (self.pp_K[sel[cs]][:, None] * acc).sum(0)
        return out

    def electron_gradient(self, points=None) -> np.ndarray:
        """d/dC of electron(C), (N, 3): the derivative of the sum in electron()
        term by term, d/dC_c [R^a F_m(pR^2)] = a_c R^(a-e_c) F_m - 2p R_c R^a F_(m+1)
        (R = C - P, dF_m/dT = -F_(m+1)); R^(a-e_c) is in the class's monomial
        closure."""
        pts = self.pts if points is None else np.asarray(points, float)
        out = np.zeros((len(pts), 3))
        nt = self.pp_nt
        for n in np.unique(nt):
            sel = np.nonzero(nt == n)[0]
            off0 = self.pp_off[sel]
            mo0 = self.pp_monooff[sel]
            nm = int(self.pp_nmono[sel[0]])
            par = self.mo_parent[mo0[0]:mo0[0] + nm]
            axs = self.mo_axis[mo0[0]:mo0[0] + nm]
            aidx = self.tm_aidx[off0[0]:off0[0] + n]
            mm = self.tm_m[off0[0]:off0[0] + n]
            exps = [(0, 0, 0)]
            for j in range(1, nm):
                e = list(exps[par[j]])
                e[axs[j]] += 1
                exps.append(tuple(e))
            where = {e: j for j, e in enumerate(exps)}
            g = self.tm_g[off0[:, None] + np.arange(n)[None, :]]
            for c0 in range(0, len(sel), 2048):
                cs = slice(c0, c0 + 2048)
                P = np.stack([self.pp_cx[sel[cs]], self.pp_cy[sel[cs]], self.pp_cz[sel[cs]]], 1)
                R = pts[None, :, :] - P[:, None, :]
                pe = self.pp_exp[sel[cs]][:, None]
                T = pe * np.einsum("cij,cij->ci", R, R)
                F = [boys(k, T) for k in range(int(mm.max()) + 2)]
                mono = [np.ones_like(T)]
                for j in range(1, nm):
                    mono.append(mono[par[j]] * R[:, :, axs[j]])
                K = self.pp_K[sel[cs]][:, None]
                for c in range(3):
                    acc = np.zeros_like(T)
                    for k in range(n):
                        e = exps[aidx[k]]
                        term = -2.0 * pe * R[:, :, c] * mono[aidx[k]] * F[mm[k] + 1]
                        if e[c] > 0:
                            d = list(e)
                            d[c] -= 1
                            term = term + e[c] * mono[where[tuple(d)]] * F[mm[k]]
                        acc += g[cs, k][:, None] * term
                    out[:, c] += (K * acc).sum(0)
        return out

    def esp_gradient(self, points=None) -> np.ndarray:
        """dV/dC (N, 3) = d nuclear/dC - d electron/dC; minus the electric field."""
        pts = self.pts if points is None else np.asarray(points, float)
        g = -self.electron_gradient(pts)
        for z, c in zip(self.Z, self.xyz):
            d = pts - c
            r = np.linalg.norm(d, axis=1)
            g -= (z / r ** 3)[:, None] * d
        return g

    def nuclear(self, points=None) -> np.ndarray:
        """sum_A Z_A/|C-R_A| (fastesp/table.py:95-100)."""
        pts = self.pts if points is None else np.asarray(points, float)
        nuc = np.zeros(len(pts))
        for z, c in zip(self.Z, self.xyz):
            nuc += z / np.linalg.norm(pts - c, axis=1)
        return nuc

    def esp(self, points=None) -> np.ndarray:
        """nuclear - electron (fastesp/table.py:102-104)."""
        return self.nuclear(points) - self.electron(points)

    def write(self, path) -> None:
        """Binary layout of fastesp/table.py:119-141."""
        with open(path, "wb") as f:
            f.write(struct.pack("<8i", self.n_pairs, self.n_terms, len(self.pts),
                                len(self.Z), int(self.max_mono), 0, 0, 0))
            for k in self.FIELDS_F:
                f.write(np.ascontiguousarray(getattr(self, k), np.float64).tobytes())
            for k in self.FIELDS_I + ("mo_parent", "mo_axis", "tm_aidx", "tm_m"):
                f.write(np.ascontiguousarray(getattr(self, k), np.int32).tobytes())
            for k in ("tm_g", "pts", "Z", "xyz"):
                f.write(np.ascontiguousarray(getattr(self, k), np.float64).tobytes())

    @classmethod
    def read(cls, path) -> "OracleTable":
        """Binary layout of fastesp/table.py:143-170."""
        d = open(path, "rb").read()
        n, nt, npt, nat, maxmono = struct.unpack_from("<8i", d, 0)[:5]
        o = 32
        kw = {}

        def rd(dt, count):
            nonlocal o
            a = np.frombuffer(d, dtype=dt, count=count, offset=o)
            o += np.dtype(dt).itemsize * count
            return a

        for k in cls.FIELDS_F:
            kw[k] = rd(np.float64, n)
        for k in cls.FIELDS_I:
            kw[k] = rd(np.int32, n)
        n_mono = int(kw["pp_monooff"][-1]) + int(kw["pp_nmono"][-1]) if n else 0
        kw["mo_parent"] = rd(np.int32, n_mono)
        kw["mo_axis"] = rd(np.int32, n_mono)
        kw["tm_aidx"] = rd(np.int32, nt)
        kw["tm_m"] = rd(np.int32, nt)
        kw["tm_g"] = rd(np.float64, nt)
        kw["pts"] = rd(np.float64, 3 * npt).reshape(npt, 3)
        kw["Z"] = rd(np.float64, nat)
        kw["xyz"] = rd(np.float64, 3 * nat).reshape(nat, 3)
        return cls(max_mono=maxmono, **kw)


def screen_mask(pp, points, tol, rule="numpy"):
    """Pairs kept by the point screen.

    rule="numpy":  keep unless K*bound/max(dmin, 0.05) < tol       (fastesp/table.py:190-194)
    rule="native": drop if K*bound/max(dmin - reff, 0.05) < tol    (build_pairs.cpp:318-328)
    """
    pts = np.asarray(points, float)
    n = pp["n"]
    if n == 0:
        return np.zeros(0, bool)
    dmin = np.empty(n)
    for c0 in range(0, n, 4096):
        P = pp["P"][c0:c0 + 4096]
        d2 = ((pts[None, :, :] - P[:, None, :]) ** 2).sum(-1)
        dmin[c0:c0 + 4096] = np.sqrt(d2.min(axis=1))
    if rule == "numpy":
        den = np.maximum(dmin, 0.05)
    elif rule == "native":
        den = np.maximum(dmin - pp["reff"], 0.05)
    else:
        raise ValueError(rule)
    return ~(pp["K"] * pp["bound"] / den < tol)


def table_from_pairs(pp, keep, points, Z, xyz) -> OracleTable:
    """Flatten kept pairs into the pairs.bin layout (fastesp/table.py:223-259)."""
    idx = np.nonzero(keep)[0]
    nts, offs, nmonos, monooffs, par_l, ax_l, aidx_l, m_l, g_l = ([] for _ in range(9))
    toff = moff = 0
    for i in idx:
        L = int(pp["L"][i])
        _, _, _, _, mvals, _ = pair_type(L)
        parent, axis, aidx = mono_schedule(L)
        n = len(mvals)
        nts.append(n)
        offs.append(toff)
        nmonos.append(len(parent))
        monooffs.append(moff)
        par_l.append(parent)
        ax_l.append(axis)
        aidx_l.append(aidx)
        m_l.append(mvals.astype(np.int32))
        g_l.append(pp["G"][i])
        toff += n
        moff += len(parent)
    cat = (lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt))
    P = pp["P"][idx] if len(idx) else np.zeros((0, 3))
    return OracleTable(
        pp_exp=pp["p"][idx] if len(idx) else np.zeros(0), pp_cx=P[:, 0].copy(),
        pp_cy=P[:, 1].copy(), pp_cz=P[:, 2].copy(),
        pp_K=pp["K"][idx] if len(idx) else np.zeros(0),
        pp_nt=np.array(nts, np.int32), pp_off=np.array(offs, np.int32),
        pp_nmono=np.array(nmonos, np.int32), pp_monooff=np.array(monooffs, np.int32),
        mo_parent=cat(par_l, np.int32), mo_axis=cat(ax_l, np.int32),
        tm_aidx=cat(aidx_l, np.int32), tm_m=cat(m_l, np.int32), tm_g=cat(g_l, np.float64),
        pts=np.asarray(points, float), Z=np.asarray(Z, float), xyz=np.asarray(xyz, float),
        max_mono=int(max(nmonos)) if nmonos else 0)


def build_table(shells, coords, Z, density, points, tol=1e-12, rule="numpy") -> OracleTable:
    """build_table (fastesp/table.py:176-259) on plain inputs.

    ``shells``: objects with ``atom``, ``l``, ``exps``, ``coeffs``; ``density`` the
    Cartesian density in shell/cart_order layout; ``points`` (N, 3) Bohr.
    """
    pp = primitive_pairs(shells, coords, np.asarray(density, float))
    keep = screen_mask(pp, points, tol, rule) if pp["n"] else np.zeros(0, bool)
    return table_from_pairs(pp, keep, points, Z, coords)


# ---------------------------------------------------------------------------
# Single primitive-pair integral by direct Hermite expansion (fastesp/ints.py)
# ---------------------------------------------------------------------------
def _e1d(i, j, p, xa, xb, tmax):
    """E[t] of (u+xa)^i (u+xb)^j e^{-p u^2} (fastesp/ints.py:62-81)."""
    e = np.zeros((i + 1, j + 1, tmax + 1))
    e[0, 0, 0] = 1.0
    for ii in range(i + 1):
        for jj in range(j + 1):
            if ii == 0 and jj == 0:
                continue
            src = (ii - 1, jj) if ii > 0 else (ii, jj - 1)
            x = xa if ii > 0 else xb
            prev = e[src[0], src[1]]
            for t in range(tmax + 1):
                v = 0.0
                if t >= 1:
                    v += prev[t - 1] / (2.0 * p)
                v += x * prev[t]
                if t + 1 <= tmax:
                    v += (t + 1) * prev[t + 1]
                e[ii, jj, t] = v
    return e[i, j, :tmax + 1]


def primitive_pair_integral(alpha, A, la, beta, B, lb, C):
    """<g_A^a|1/|r-C||g_B^b> for bare primitives (fastesp/ints.py:84-158)."""
    A, B, C = (np.asarray(x, float) for x in (A, B, C))
    p = alpha + beta
    P = (alpha * A + beta * B) / p
    K = float(np.exp(-alpha * beta / p * float((A - B) @ (A - B))))
    R = C - P
    ex = [_e1d(la[k], lb[k], p, P[k] - A[k], P[k] - B[k], la[k] + lb[k]) for k in range(3)]
    tab = a_table(sum(la) + sum(lb))
    RR = float(R @ R)
    tot = 0.0
    for tx, cx in enumerate(ex[0]):
        for ty, cy in enumerate(ex[1]):
            for tz, cz in enumerate(ex[2]):
                et = cx * cy * cz
                if et == 0.0:
                    continue
                t = (tx, ty, tz)
                lt = tx + ty + tz
                d = 0.0
                for jx in range(tx // 2 + 1):
                    for jy in range(ty // 2 + 1):
                        for jz in range(tz // 2 + 1):
                            a3 = tab[tx, jx] * tab[ty, jy] * tab[tz, jz]
                            if a3 == 0.0:
                                continue
                            jj = jx + jy + jz
                            d += (a3 * (2.0 * p) ** (lt - jj) * R[0] ** (t[0] - 2 * jx)
                                  * R[1] ** (t[1] - 2 * jy) * R[2] ** (t[2] - 2 * jz)
                                  * boys(lt - jj, p * RR))
                tot += et * (-1.0) ** lt * (2.0 * pi / p) * d
    return K * tot
