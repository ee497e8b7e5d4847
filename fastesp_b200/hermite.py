"""Point-independent Hermite bookkeeping of one angular class L = la + lb.

For a primitive pair with Hermite expansion coefficients etab[t] (t = (tx,ty,tz),
|t| <= L) the electron potential at R = C - P is

    I(C) = K (2 pi/p) sum_t (-1)^|t| etab[t] d^t/dR^t F_0(p R^2)

and each 1-D derivative expands through the a-table recurrence
a[t+1,j] = -a[t,j] + (t-2j+2) a[t,j-1] (fastesp/ints.py:18-21, 46-59) into
(2p)^(t-j) R^(t-2j) F_(t-j).  Collecting equal (alpha = t - 2j, m = |t| - |j|)
gives, per class, a fixed sparse map etab -> G[alpha, m] with

    I(C) = K sum_k G_k R^alpha_k F_m_k(p R^2),   G_k = (2 pi/p)(2p)^m_k sum_t M0[k,t] etab[t]

(fastesp/esp.py:54-105, fastesp/table.py:3-9).  Terms are kept in the order the
reference stores them: keys (ax, ay, az, m) sorted lexicographically.  The
monomial schedule (closure of the alpha set under decrement, sorted; each
monomial built from its first decrementable axis) is the reference's
(fastesp/table.py:198-221) and only matters for the ``pairs.bin`` export: the
CUDA kernels evaluate the same polynomial in nested Horner form instead.

Everything here depends on L only; ``csrc/gen_classes.py`` turns it into
compile-time tables and unrolled device code.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

LMAX_SHELL = 4                 # s..g shells
NCLASS = 2 * LMAX_SHELL + 1    # L = 0..8


@lru_cache(maxsize=None)
def a_table(lmax: int) -> np.ndarray:
    """a[t, j] with d^t/dx^t F_0(p x^2) = sum_j a[t,j] (2p)^(t-j) x^(t-2j) F_(t-j)."""
    a = np.zeros((lmax + 1, lmax // 2 + 2))
    a[0, 0] = 1.0
    for t in range(lmax):
        for j in range(lmax // 2 + 2):
            a[t + 1, j] = -a[t, j] + ((t - 2 * j + 2) * a[t, j - 1] if j else 0.0)
    return a


# Screening-bound moment table of the reference (fastesp/esp.py:25-28,
# build_pairs.cpp:98-102).  Its comment defines M_n = int |He_n(x)| e^{-x^2/2} dx,
# which holds for n = 0, 1 only (e.g. M_2 here is 4/sqrt(2 pi), the integral is
# 4/sqrt(e)); the values are kept verbatim because the screening decision
# K * bound / d < tol must select the same pairs as the reference.
SCREEN_MOMENTS = (2.5066282746310002, 2.0, 1.5957691216057308, 4.0,
                  10.212920779565312, 33.63284766793385, 136.5963625280984,
                  665.1416330443616, 3768.863619586618, 25506.330595911374,
                  202331.81842358326, 1872154.2572862155)


def t_index(L: int) -> dict:
    """Compact index of Hermite triples t with |t| <= L (x-major, then y, then z)."""
    out = {}
    for tx in range(L + 1):
        for ty in range(L + 1 - tx):
            for tz in range(L + 1 - tx - ty):
                out[(tx, ty, tz)] = len(out)
    return out


@lru_cache(maxsize=None)
def class_terms(L: int):
    """(keys, rows) of class L.

    keys: sorted list of (ax, ay, az, m); rows[k]: list of (t, coef) with t a
    Hermite triple and coef the integer-valued M0[k, t] = (-1)^|t| a a a.
    """
    tab = a_table(max(L, 1))
    terms: dict = {}
    for tx in range(L + 1):
        for ty in range(L + 1 - tx):
            for tz in range(L + 1 - tx - ty):
                lt = tx + ty + tz
                sgn = -1.0 if lt % 2 else 1.0
                for jx in range(tx // 2 + 1):
                    for jy in range(ty // 2 + 1):
                        for jz in range(tz // 2 + 1):
                            c = tab[tx, jx] * tab[ty, jy] * tab[tz, jz]
                            if c == 0.0:
                                continue
                            key = (tx - 2 * jx, ty - 2 * jy, tz - 2 * jz, lt - jx - jy - jz)
                            row = terms.setdefault(key, {})
                            row[(tx, ty, tz)] = row.get((tx, ty, tz), 0.0) + sgn * c
    keys = sorted(terms)
    rows = [sorted((t, v) for t, v in terms[k].items() if v != 0.0) for k in keys]
    return keys, rows


def n_terms(L: int) -> int:
    return len(class_terms(L)[0])


def record_stride(L: int) -> int:
    """FP64 words per pair record [p, Px, Py, Pz, K, K*bound, G_0..G_nt-1], padded to 16 bytes."""
    n = 6 + n_terms(L)
    return n + (n & 1)


def record_stride_f32(L: int) -> int:
    """FP32 words per mixed-precision record, padded to 16 bytes.

    The pair's scalars (the centre as float pairs hi = float(v), lo =
    float(v - hi)), then every coefficient twice (a {c, c} operand pair of the
    packed FP32x2 code), then the L + 1 coefficients of the routing bound
    sum_n b_n / |R|^(n+1): [p, sqrt(p), Px_hi, Py_hi, Pz_hi, Px_lo, Py_lo,
    Pz_lo, rfar^2, p^-1/2, 0, 0, c_0, c_0, c_1, c_1, ..., b_0, .., b_L] with
    c_k = K G_k s_m p^-(m+1/2) (csrc/table.cuh).
    """
    n = 12 + 2 * n_terms(L) + L + 1
    return (n + 3) // 4 * 4


@lru_cache(maxsize=None)
def mono_schedule(L: int):
    """(parent, axis, aidx) of the reference's monomial schedule for class L."""
    keys, _ = class_terms(L)
    grown = {k[:3] for k in keys}
    stack = list(grown)
    while stack:
        a = stack.pop()
        for ax in range(3):
            if a[ax] > 0:
                q = a[:ax] + (a[ax] - 1,) + a[ax + 1:]
                if q not in grown:
                    grown.add(q)
                    stack.append(q)
    order = sorted(grown)
    idx = {a: i for i, a in enumerate(order)}
    parent = np.zeros(len(order), np.int32)
    axis = np.zeros(len(order), np.int32)
    for i, a in enumerate(order):
        for ax in range(3):
            if a[ax] > 0:
                parent[i] = idx[a[:ax] + (a[ax] - 1,) + a[ax + 1:]]
                axis[i] = ax
                break
    aidx = np.array([idx[k[:3]] for k in keys], np.int32)
    return parent, axis, aidx


def term_m(L: int) -> np.ndarray:
    return np.array([k[3] for k in class_terms(L)[0]], np.int32)


def eval_flops(L: int) -> int:
    """Algorithmic floating-point operations of one (pair, point) evaluation.

    2 nt (a multiply and an add per term) + (nmono - 1) monomial products
    + 14 for R, T, K*s and the accumulation (exp/erf counted as one each)
    + 3 mmax for the Boys recursion, mmax = L: the count of the reference
    formulation (fastesp/table.py:82-92, fastesp/native/esp_gpu.cu:182-206).
    The kernels' nested-Horner form needs fewer operations; this count is the
    fixed yardstick of the achieved-throughput figure.
    """
    nt = n_terms(L)
    nm = len(mono_schedule(L)[0])
    return 2 * nt + (nm - 1) + 14 + 3 * L


def build_flops(la: int, lb: int) -> int:
    """Algorithmic floating-point operations of building one primitive pair of
    shells with angular momenta (la, lb), without the point screen:
    3 (la+1)(lb+1)(L+1) * 4 for the three axes' E-coefficients, ncart(la)
    ncart(lb) (L+1)^3 * 2 for the density-weighted Hermite table and
    2 nnz(M0) for the G contraction -- the steps of the reference's pair
    construction (fastesp/esp.py:108-257, fastesp/native/build_pairs.cpp:237-316).
    """
    L = la + lb
    nc = lambda l: (l + 1) * (l + 2) // 2  # noqa: E731
    nnz = sum(len(r) for r in class_terms(L)[1])
    return 3 * (la + 1) * (lb + 1) * (L + 1) * 4 + nc(la) * nc(lb) * (L + 1) ** 3 * 2 + 2 * nnz


def field_flops(L: int) -> int:
    """Algorithmic FLOPs of one (pair, point) of the potential-and-gradient
    (field) evaluation: the potential's eval_flops, the companion sum
    sum_k G_k R^a F_(m+1) (2 nt), the three monomial-derivative sums (6 nt),
    the order L+1 of the Boys recursion (3), and d/dC = dS/dR - 2pR u plus
    the three extra accumulations (18)."""
    return eval_flops(L) + 8 * n_terms(L) + 21
