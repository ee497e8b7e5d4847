"""Generate ``classes_gen.cuh``: compile-time data and unrolled code per class L.

    python fastesp_b200/csrc/gen_classes.py        (run by the build; output committed)

For every angular class L = la + lb (0..8) this emits

* the term count, FP64/FP32 record strides and Boys order;
* ``fe_poly_L<L>``: s = sum_k G_k R^alpha_k F_m_k for NP points per thread in
  nested Horner form -- per Boys order m the polynomial sum_k G_k R^alpha_k is
  evaluated x-outer / y / z-inner with fused multiply-adds, every coefficient
  is read once and reused for the NP points;
* ``fe_grad_L<L>``: the same sum and its gradient with respect to R (field);
* ``fe_mom_L<L>_c<c>``: the adjoint moments acc_k += w F_m_k R^alpha_k of one
  chunk of the class's terms (terms in reference order, split at monomial
  boundaries into chunks of at most MOM_CHUNK terms so the accumulators of a
  chunk stay in registers);
* the sparse contraction rows M0[k, t] (etab -> G) used by the table builder,
  with t in the compact order of ``hermite.t_index``, and for the small
  classes the same contraction as straight-line code (``fe_m0_rows_L``,
  ``fe_g_store_L``);
* ``fe_f32_terms_L``: the coefficient pairs and routing-bound sums of one
  mixed-precision record, straight-line;
* the Boys Taylor grid F_n(i h), n = 0..NTAB-1, computed here in 40-digit
  arithmetic (mpmath), and the per-order asymptotic thresholds.
"""
from __future__ import annotations

import math
import sys
from functools import lru_cache
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from fastesp_b200 import hermite as H  # noqa: E402

LMAX = 2 * H.LMAX_SHELL        # largest class
MMAX = LMAX + 1                # largest Boys order needed (adjoint needs L+1)
TAYLOR_K = 8                   # Taylor terms of the tabulated branch
GRID_H = 1.0 / 16.0            # grid spacing of the tabulated branch
GRID_TMAX = 20.0               # tabulated branch covers 0 <= T < GRID_TMAX
NTAB = MMAX + TAYLOR_K         # orders stored per grid row
TAYLOR_K32 = 6                 # FP32 grid: Taylor terms
GRID_H32 = 1.0 / 4.0           # FP32 grid spacing (truncation < 6e-9 relative)
GRID_TMAX32 = 32.0             # FP32 grid covers 0 <= T < 32 (the FP32 asymptotic
                               # thresholds of orders <= 6 lie below it)
NTAB32 = MMAX + TAYLOR_K32
VARS = ("x", "y", "z")
MOM_CHUNK = 48                 # adjoint moment accumulators per thread
M0_UNROLL_LMAX = 2             # classes whose G contraction is emitted straight-line


# --------------------------------------------------------------------------
# Horner emission
# --------------------------------------------------------------------------
class Emitter:
    def __init__(self, real="Real"):
        self.lines = []
        self.nops = 0
        self.real = real

    def w(self, s):
        self.lines.append("  " + s)

    def horner(self, terms, depth, acc, coef):
        """Emit acc[depth][j] = sum_terms coef(k) * v^e ... over VARS[depth:].

        ``terms``: {exponent tuple over VARS[depth:]: k}.  ``coef(k)`` returns
        (setup_line or None, scalar expression).
        """
        v = VARS[depth]
        groups = {}
        for e, k in terms.items():
            groups.setdefault(e[0], {})[e[1:]] = k
        emax = max(groups)
        dst = acc[depth]
        first = True
        for e in range(emax, -1, -1):
            if e in groups:
                if depth == len(VARS) - 1:
                    (k,) = groups[e].values()
                    setup, sub = coef(k)
                    if setup:
                        self.w(setup)
                    sub_j = sub
                else:
                    self.horner(groups[e], depth + 1, acc, coef)
                    sub_j = f"{acc[depth + 1]}[j]"
                if first:
                    self.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) {dst}[j] = {sub_j};")
                    first = False
                else:
                    self.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) "
                           f"{dst}[j] = fe_fma({dst}[j], {v}[j], {sub_j});")
                    self.nops += 1
            elif not first:
                self.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) {dst}[j] *= {v}[j];")
                self.nops += 1


class CoefLoader:
    """Hands out coefficient expressions in first-use (consumption) order.

    The record stores class-L coefficients in this order, so the generated
    code reads them front to back: ``vec`` > 0 emits one 16-byte vector load
    per ``vec`` consecutive coefficients (float4 / double2), 0 scalar loads.
    """

    def __init__(self, em, order=None, vec=0, vtype="", dup=None):
        self.em = em
        self.pos = {} if order is None else {k: i for i, k in enumerate(order)}
        self.fixed = order is not None
        self.vec = vec
        self.vtype = vtype
        self.dup = dup          # None, "scalar" or "packed": FP32 {g, g} pairs
        self.loaded = set()

    def expr(self, k):
        if k not in self.pos:
            assert not self.fixed
            self.pos[k] = len(self.pos)
        p = self.pos[k]
        if self.dup:
            # coefficient p occupies floats 2p, 2p+1 (the same value twice), so one
            # float4 holds two coefficients, each already a float2 pair
            c, half = divmod(p, 2)
            if c not in self.loaded:
                self.loaded.add(c)
                self.em.w(f"const float4 gv{c} = *reinterpret_cast<const float4*>(g + {4 * c});")
            a, b = ("x", "y") if half == 0 else ("z", "w")
            return f"make_float2(gv{c}.{a}, gv{c}.{b})" if self.dup == "packed" else f"gv{c}.{a}"
        if not self.vec:
            return f"g[{p}]"
        c, lane = divmod(p, self.vec)
        if c not in self.loaded:
            self.loaded.add(c)
            self.em.w(f"const {self.vtype} gv{c} = *reinterpret_cast<const {self.vtype}*>(g + {c * self.vec});")
        return f"gv{c}.{'xyzw'[lane]}"

    def order(self):
        return [k for k, _ in sorted(self.pos.items(), key=lambda kv: kv[1])]


def poly_m_major(L, order=None, vec=0, vtype="", dup=None, asym=False):
    """s = sum_m F_m h_m(R), h_m the Horner polynomial of the order-m terms,
    orders taken from the highest down (the coefficient consumption order).

    ``asym``: the form for points where every F_m is asymptotic and the
    coefficients carry p^-(m+1/2), so F_m is 1/|R|^(2m+1): s = sum_m ir2^m
    h_m, in Horner form in ir2 = 1/|R|^2 (the caller multiplies by 1/|R|)."""
    keys, _ = H.class_terms(L)
    em = Emitter()
    ld = CoefLoader(em, order, vec, vtype, dup)
    by_m = {}
    for k, (ax, ay, az, m) in enumerate(keys):
        by_m.setdefault(m, {})[(ax, ay, az)] = k
    acc = ("ha", "hb", "hc")
    prev = None
    for m in sorted(by_m, reverse=True):
        em.horner(by_m[m], 0, acc, lambda k: (None, ld.expr(k)))
        if asym:
            if prev is None:
                em.w("FE_UNROLL for (int j = 0; j < NP; ++j) s[j] = ha[j];")
            else:
                for _ in range(prev - m - 1):
                    em.w("FE_UNROLL for (int j = 0; j < NP; ++j) s[j] *= ir2[j];")
                    em.nops += 1
                em.w("FE_UNROLL for (int j = 0; j < NP; ++j) s[j] = fe_fma(s[j], ir2[j], ha[j]);")
                em.nops += 1
        elif prev is None:
            em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) s[j] = F[j][{m}] * ha[j];")
            em.nops += 1
        else:
            em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) s[j] = fe_fma(F[j][{m}], ha[j], s[j]);")
            em.nops += 1
        prev = m
    if asym:
        for _ in range(prev):
            em.w("FE_UNROLL for (int j = 0; j < NP; ++j) s[j] *= ir2[j];")
            em.nops += 1
    return em, ld


def poly_alpha_major(L, order=None, vec=0, vtype="", dup=None):
    keys, _ = H.class_terms(L)
    em = Emitter()
    ld = CoefLoader(em, order, vec, vtype, dup)
    by_a = {}
    for k, (ax, ay, az, m) in enumerate(keys):
        by_a.setdefault((ax, ay, az), []).append((k, m))
    acc = ("ha", "hb", "hc")

    def coef(a):
        ks = by_a[a]
        k0, m0 = ks[0]
        em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) hd[j] = {ld.expr(k0)} * F[j][{m0}];")
        em.nops += 1
        for k, m in ks[1:]:
            em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) hd[j] = fe_fma({ld.expr(k)}, F[j][{m}], hd[j]);")
            em.nops += 1
        return None, "hd[j]"

    em.horner({a: a for a in by_a}, 0, acc, coef)
    em.w("FE_UNROLL for (int j = 0; j < NP; ++j) s[j] = ha[j];")
    return em, ld


def poly_variant(L):
    """(builder, tag) of the cheaper of the two nested-Horner orders for class L."""
    a, _ = poly_m_major(L)
    b, _ = poly_alpha_major(L)
    return (poly_m_major, "m-major", a.nops) if a.nops <= b.nops else \
        (poly_alpha_major, "alpha-major", b.nops)


@lru_cache(maxsize=None)
def consumption_order(L):
    """Term indices k in the order the class-L code reads them = record order."""
    build, _, _ = poly_variant(L)
    return build(L)[1].order()


def route_constants(L):
    """Routing-bound constants of the mixed path, per record position of class L.

    Returns [(n, m, c)] with |G R^a F_m(p R^2)| <= |G| c p^-(m + 1/2) / |R|^(n + 1),
    n = 2m - |a|: from F_m(T) <= Gamma(m + 1/2) / (2 T^(m + 1/2)) and
    |R^a| <= |R|^|a| max_{|u|=1} |u^a|, the maximum of ux^ax uy^ay uz^az on the
    unit sphere being sqrt(ax^ax ay^ay az^az / |a|^|a|) (at u_i^2 = a_i / |a|).
    """
    keys, _ = H.class_terms(L)
    out = []
    for k in consumption_order(L):
        ax, ay, az, m = keys[k]
        deg = ax + ay + az
        num = 1.0
        for v in (ax, ay, az):
            num *= float(v) ** v if v else 1.0
        mf = (num / float(deg) ** deg) ** 0.5 if deg else 1.0
        n = 2 * m - deg
        assert 0 <= n <= L and m < 16
        out.append((n, m, math.gamma(m + 0.5) / 2.0 * mf))
    return out


def f32_terms_function(L):
    """Straight-line FP32-record terms of class L (one thread per record).

    For record position j with routing constants (n, m, c): the coefficient
    pair o[2j] = o[2j+1] = K G_j s_m v_m and the bound sum b_n += |G_j| c v_m,
    with v_m = p^-(m+1/2).  Every index is a constant, so s, v and b stay in
    registers; the operation order is that of a loop over j.
    """
    out = [f"// class L={L}: FP32 coefficient pairs and routing-bound sums, record order",
           f"__device__ __forceinline__ void fe_f32_terms_L{L}(const double* __restrict__ g, double K,",
           f"    const double (&s)[{L + 1}], const double (&v)[{L + 1}], float* __restrict__ o,",
           f"    double (&b)[{L + 1}]) {{"]
    for j, (n, m, c) in enumerate(route_constants(L)):
        out.append(f"  {{ const double t = g[{j}]; o[{2 * j}] = o[{2 * j + 1}] = float(K * t * s[{m}] * v[{m}]);"
                   f" b[{n}] += fabs(t) * {c!r} * v[{m}]; }}")
    out.append("}")
    return out


def m0_functions(L):
    """Straight-line G contraction of class L for the table builder.

    ``fe_m0_rows_L``: s_k = sum_t M0[k, t] etab[t] for every term k, as fused
    multiply-adds in the order of the sparse rows; ``fe_g_store_L``: record
    position j of the term k it holds gets cf (2p)^m_k s_k.  With constant
    indices the builder keeps etab and s in registers.
    """
    keys, rows = H.class_terms(L)
    tix = H.t_index(L)
    nt, ntri = len(keys), len(tix)
    out = [f"// class L={L}: contraction sums s_k = sum_t M0[k, t] etab[t], term order",
           f"__device__ __forceinline__ void fe_m0_rows_L{L}(const double (&e)[{ntri}], double (&s)[{nt}]) {{"]
    for k, r in enumerate(rows):
        (t0, c0), rest = r[0], r[1:]
        expr = f"{float(c0)!r} * e[{tix[t0]}]"
        for t, c in rest:
            expr = f"fma({float(c)!r}, e[{tix[t]}], {expr})"
        out.append(f"  s[{k}] = {expr};")
    out.append("}")
    out.append(f"// class L={L}: G at record position j = cf (2p)^m s_k for the term k stored there")
    out.append(f"__device__ __forceinline__ void fe_g_store_L{L}(const double (&s)[{nt}],"
               f" const double (&pw)[{L + 1}], double cf, double* __restrict__ g) {{")
    for j, k in enumerate(consumption_order(L)):
        out.append(f"  g[{j}] = cf * pw[{keys[k][3]}] * s[{k}];")
    out.append("}")
    return out


def poly_functions(L):
    """FP32 (coefficients stored as {g, g} pairs), packed FP32x2 (two points per
    float2, the same pairs as operands) and FP64 (double2 loads) evaluators."""
    build, tag, nops = poly_variant(L)
    order = consumption_order(L)
    out = []
    for real, vtype, vec, suffix, dup in (("float", "float4", 4, "32", "scalar"),
                                          ("float2", "float4", 4, "32x2", "packed"),
                                          ("double", "double2", 2, "64", None)):
        em, _ = build(L, order, vec, vtype, dup)
        lay = ("coefficients g[2k] = g[2k+1] = c_k in consumption order" if dup else
               "coefficients g[k] in consumption order")
        out += [f"// class L={L}: {H.n_terms(L)} terms, {nops} fused ops per point ({tag}),",
                f"// {lay}, 16-byte aligned"
                + ("; two points per float2 lane" if dup == "packed" else ""),
                "template <int NP>",
                f"__device__ __forceinline__ void fe_poly{suffix}_L{L}(const {'float' if dup else real}* __restrict__ g,",
                f"    const {real} (&x)[NP], const {real} (&y)[NP], const {real} (&z)[NP],",
                f"    const {real} (&F)[NP][{L + 1}], {real} (&s)[NP]) {{",
                "  using Real = " + real + ";",
                "  Real ha[NP], hb[NP], hc[NP], hd[NP];",
                "  (void)hb; (void)hc; (void)hd;"]
        out += em.lines
        out.append("}")
        out.append("")
    if tag == "m-major":
        # the asymptotic form of the packed FP32 code (see poly_m_major)
        em, _ = poly_m_major(L, order, 4, "float4", "packed", asym=True)
        out += [f"// class L={L}: the packed form for points whose Boys vectors are all",
                "// asymptotic: s = sum_m ir2^m h_m (Horner in ir2 = 1/|R|^2); the caller",
                "// multiplies by 1/|R|; coefficients as fe_poly32x2_L" + str(L),
                "template <int NP>",
                f"__device__ __forceinline__ void fe_poly32x2a_L{L}(const float* __restrict__ g,",
                "    const float2 (&x)[NP], const float2 (&y)[NP], const float2 (&z)[NP],",
                "    const float2 (&ir2)[NP], float2 (&s)[NP]) {",
                "  using Real = float2;",
                "  Real ha[NP], hb[NP], hc[NP], hd[NP];",
                "  (void)hb; (void)hc; (void)hd; (void)ir2;"]
        out += em.lines
        out.append("}")
        out.append("")
    return out, nops


def grad_function(L):
    """s = sum_k G_k R^a F_m and dS/dR_c = sum_k G_k (a_c R^(a-e_c) F_m - 2p R_c R^a F_(m+1)).

    Written as s, u = sum_k G_k R^a F_(m+1) and the three partial derivatives
    of the monomials, each again in Horner form over exponents; F carries
    orders 0..L+1.  Coefficients are read from the record's consumption order.
    """
    keys, _ = H.class_terms(L)
    pos = {k: i for i, k in enumerate(consumption_order(L))}
    em = Emitter()
    acc = ("ha", "hb", "hc")
    for name, shift in (("s", 0), ("u", 1)):
        by_m = {}
        for k, (ax, ay, az, m) in enumerate(keys):
            by_m.setdefault(m + shift, {})[(ax, ay, az)] = k
        first = True
        for m in sorted(by_m):
            em.horner(by_m[m], 0, acc, lambda k: (None, f"g[{pos[k]}]"))
            op = (f"{name}[j] = F[j][{m}] * ha[j];" if first else
                  f"{name}[j] = fe_fma(F[j][{m}], ha[j], {name}[j]);")
            em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) {op}")
            first = False
    for c, cname in enumerate(("dx", "dy", "dz")):
        by_m = {}
        for k, key in enumerate(keys):
            a = list(key[:3])
            m = key[3]
            if a[c] == 0:
                continue
            fac = a[c]
            a[c] -= 1
            by_m.setdefault(m, {})[tuple(a)] = (k, fac)
        first = True
        for m in sorted(by_m):
            em.horner(by_m[m], 0, acc,
                      lambda kf: (None, f"(Real({kf[1]}) * g[{pos[kf[0]]}])"))
            op = (f"{cname}[j] = F[j][{m}] * ha[j];" if first else
                  f"{cname}[j] = fe_fma(F[j][{m}], ha[j], {cname}[j]);")
            em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) {op}")
            first = False
        if first:
            em.w(f"FE_UNROLL for (int j = 0; j < NP; ++j) {cname}[j] = Real(0);")
    out = [f"// class L={L}: value, F_(m+1) companion sum and monomial derivatives",
           "template <typename Real, int NP>",
           f"__device__ __forceinline__ void fe_grad_L{L}(const Real* __restrict__ g,",
           "    const Real (&x)[NP], const Real (&y)[NP], const Real (&z)[NP],",
           f"    const Real (&F)[NP][{L + 2}], Real (&s)[NP], Real (&u)[NP],",
           "    Real (&dx)[NP], Real (&dy)[NP], Real (&dz)[NP]) {",
           "  Real ha[NP], hb[NP], hc[NP];",
           "  (void)hb; (void)hc;"]
    out += em.lines
    out.append("}")
    return out


def mom_chunks(L):
    """Contiguous term ranges [k0, k1) of class L (reference order), cut only
    between monomials, as even as possible with at most MOM_CHUNK terms."""
    keys, _ = H.class_terms(L)
    bounds = [0]
    for k in range(1, len(keys)):
        if keys[k][:3] != keys[k - 1][:3]:
            bounds.append(k)
    nt = len(keys)
    n = -(-nt // MOM_CHUNK)
    while True:
        cuts, last = [0], 0
        for c in range(1, n):
            want = nt * c / n
            b = min((x for x in bounds if x > last), key=lambda x: abs(x - want), default=nt)
            cuts.append(b)
            last = b
        cuts.append(nt)
        spans = list(zip(cuts[:-1], cuts[1:]))
        if all(0 < b - a <= MOM_CHUNK for a, b in spans):
            return spans
        n += 1


def mom_function(L, c, k0, k1):
    """acc[j] += R^alpha F_m w for the terms k0 + j of class L (wF[m] = w F_m)."""
    keys, _ = H.class_terms(L)
    sub = keys[k0:k1]
    lines = [f"// class L={L} chunk {c}: terms [{k0}, {k1}) in reference order",
             "template <typename Real>",
             f"__device__ __forceinline__ void fe_mom_L{L}_c{c}(Real x, Real y, Real z,",
             f"    const Real (&wF)[{L + 1}], Real (&acc)[{k1 - k0}]) {{"]
    for ax, v in enumerate(VARS):
        top = max(k[ax] for k in sub)
        if top >= 1:
            lines.append(f"  const Real {v}1 = {v};")
        for e in range(2, top + 1):
            lines.append(f"  const Real {v}{e} = {v}{e - 1} * {v};")
    have_xy = set()
    prev = None
    fac, name = [], ""
    for j, (a, b, cz, m) in enumerate(sub):
        if (a, b, cz) != prev:
            if a and b and (a, b) not in have_xy:
                lines.append(f"  const Real x{a}y{b} = x{a} * y{b};")
                have_xy.add((a, b))
            fac = ([f"x{a}y{b}"] if a and b else ([f"x{a}"] if a else []) + ([f"y{b}"] if b else []))
            fac += [f"z{cz}"] if cz else []
            name = f"m{a}_{b}_{cz}"
            if fac:
                lines.append(f"  const Real {name} = {' * '.join(fac)};")
            prev = (a, b, cz)
        if fac:
            lines.append(f"  acc[{j}] = fe_fma({name}, wF[{m}], acc[{j}]);")
        else:
            lines.append(f"  acc[{j}] += wF[{m}];")
    lines.append("}")
    lines.append("")
    return lines


# --------------------------------------------------------------------------
# Boys grid and thresholds (40-digit reference values)
# --------------------------------------------------------------------------
def boys_mp(m, T):
    import mpmath as mp
    if T == 0:
        return mp.mpf(1) / (2 * m + 1)
    a = mp.mpf(m) + mp.mpf(1) / 2
    return mp.gammainc(a, 0, T) / (2 * mp.power(T, a))


def boys_grid():
    import mpmath as mp
    mp.mp.dps = 40
    nrow = int(round(GRID_TMAX / GRID_H)) + 2
    rows = []
    for i in range(nrow):
        T = mp.mpf(i) * mp.mpf(GRID_H)
        rows.append([float(boys_mp(n, T)) for n in range(NTAB)])
    return rows


def boys_grid32():
    import mpmath as mp
    mp.mp.dps = 30
    nrow = int(round(GRID_TMAX32 / GRID_H32)) + 2
    return [[float(boys_mp(n, mp.mpf(i) * mp.mpf(GRID_H32))) for n in range(NTAB32)]
            for i in range(nrow)]


def boys_scale(m):
    """s_m = (sqrt(pi)/2) (2m-1)!!/2^m, the large-T limit of F_m(T) T^(m+1/2).

    The packed FP32 evaluator works with F^_m = F_m / s_m: its asymptotic form
    is T^-(m+1/2) and its recursions have exactly representable constants, so
    no FP32 rounding of a constant biases every pair alike; the table build
    folds s_m into the FP32 coefficients in FP64."""
    import mpmath as mp
    mp.mp.dps = 30
    s = mp.sqrt(mp.pi) / 2
    for j in range(1, m + 1):
        s *= mp.mpf(2 * j - 1) / 2
    return s


def boys_grid32_scaled(M):
    """Rows F_(M+k)(i h)/(k! s_M), k < TAYLOR_K32, of the FP32 grid (30 digits):
    the Taylor polynomial of F^_M = F_M / s_M in d directly."""
    import mpmath as mp
    mp.mp.dps = 30
    nrow = int(round(GRID_TMAX32 / GRID_H32)) + 2
    sM = boys_scale(M)
    return [[float(boys_mp(M + k, mp.mpf(i) * mp.mpf(GRID_H32)) / (mp.factorial(k) * sM))
             for k in range(TAYLOR_K32)] for i in range(nrow)]


def split_f32(v):
    """(hi, lo) floats with hi + lo = v to about 48 bits."""
    import numpy as np
    hi = float(np.float32(float(v)))
    lo = float(np.float32(float(v - hi)))
    return hi, lo


def asym_thresholds(rel=1e-16):
    """Smallest T (on a 0.25 grid) from which the asymptotic Boys vector
    F_m = (2m-1)!!/2^(m+1) sqrt(pi/T^(2m+1)) is within ``rel`` of F_m for all
    m <= M, for every M <= MMAX."""
    import mpmath as mp
    mp.mp.dps = 40
    out = []
    for M in range(MMAX + 1):
        T = 120.0
        while T > 1.0:
            Tm = mp.mpf(T - 0.25)
            ok = True
            for m in range(M + 1):
                ex = boys_mp(m, Tm)
                df = mp.mpf(1)
                for q in range(1, 2 * m, 2):
                    df *= q
                asy = df / mp.power(2, m + 1) * mp.sqrt(mp.pi / mp.power(Tm, 2 * m + 1))
                if abs(asy - ex) / ex > rel:
                    ok = False
                    break
            if not ok:
                break
            T -= 0.25
        out.append(T)
    return out


def main() -> int:
    out = ["// Generated by gen_classes.py -- do not edit.",
           "#pragma once",
           "#ifndef FE_UNROLL",
           "#define FE_UNROLL _Pragma(\"unroll\")",
           "#endif",
           "",
           f"#define FE_NCLASS {LMAX + 1}",
           f"#define FE_MMAX {MMAX}",
           f"#define FE_BOYS_NTAB {NTAB}",
           f"#define FE_BOYS_TAYLOR_K {TAYLOR_K}",
           f"#define FE_BOYS_GRID_INV_H {1.0 / GRID_H!r}",
           f"#define FE_BOYS_GRID_H {GRID_H!r}",
           f"#define FE_BOYS_GRID_TMAX {GRID_TMAX!r}",
           ""]
    nts = [H.n_terms(L) for L in range(LMAX + 1)]
    out.append("static constexpr int fe_class_nterm[FE_NCLASS] = {"
               + ", ".join(map(str, nts)) + "};")
    out.append("static constexpr int fe_class_rec64[FE_NCLASS] = {"
               + ", ".join(str(H.record_stride(L)) for L in range(LMAX + 1)) + "};")
    out.append("static constexpr int fe_class_rec32[FE_NCLASS] = {"
               + ", ".join(str(H.record_stride_f32(L)) for L in range(LMAX + 1)) + "};")
    out.append("static constexpr int fe_class_ntri[FE_NCLASS] = {"
               + ", ".join(str(len(H.t_index(L))) for L in range(LMAX + 1)) + "};")
    out.append("")
    ths = asym_thresholds()
    out.append("// T above which the Boys vector F_0..F_M is its asymptotic form to 1e-16")
    out.append("static constexpr double fe_boys_asym_T[FE_MMAX + 1] = {"
               + ", ".join(repr(t) for t in ths) + "};")
    th32 = asym_thresholds(rel=2e-8)
    out.append("// the same for FP32 (2e-8 relative)")
    out.append("static constexpr float fe_boys32_asym_T[FE_MMAX + 1] = {"
               + ", ".join(repr(t) + "f" for t in th32) + "};")
    out.append("")
    rows32 = boys_grid32()
    out.append(f"#define FE_BOYS32_NTAB {NTAB32}")
    out.append(f"#define FE_BOYS32_TAYLOR_K {TAYLOR_K32}")
    out.append(f"#define FE_BOYS32_GRID_INV_H {1.0 / GRID_H32!r}f")
    out.append(f"#define FE_BOYS32_GRID_H {GRID_H32!r}f")
    out.append(f"#define FE_BOYS32_GRID_TMAX {GRID_TMAX32!r}f")
    out.append(f"#define FE_BOYS32_NROW {len(rows32)}")
    out.append("__device__ const float fe_boys_grid32[FE_BOYS32_NROW * FE_BOYS32_NTAB] = {")
    for r in rows32:
        out.append("  " + ", ".join(repr(float(v)) + "f" if v > 1e-37 else "0.0f" for v in r) + ",")
    out.append("};")
    out.append("")
    # per-order scaled FP32 rows for the packed evaluator: F_(M+k)(i h) / k!
    ms = 6
    out.append(f"#define FE_BOYS32S_MMAX {ms}")
    # kappa_m = 1 / (2 s_m) and 1 / s_m as float hi/lo pairs (FP32 Boys recursions)
    kap = [split_f32(1 / (2 * boys_scale(m))) for m in range(MMAX + 1)]
    sinv = [split_f32(1 / boys_scale(m)) for m in range(MMAX + 1)]
    for name, vals, k in (("fe_boys32_kappa_hi", kap, 0), ("fe_boys32_kappa_lo", kap, 1),
                          ("fe_boys32_sinv_hi", sinv, 0), ("fe_boys32_sinv_lo", sinv, 1)):
        out.append(f"static constexpr float {name}[FE_MMAX + 1] = {{"
                   + ", ".join(repr(v[k]) + "f" for v in vals) + "};")
    out.append("// F_(M+k)(i h)/(k! s_M), M = 0..FE_BOYS32S_MMAX, k < FE_BOYS32_TAYLOR_K: row (M, i) at")
    out.append("// (M * FE_BOYS32_NROW + i) * FE_BOYS32_TAYLOR_K (Taylor polynomial in d directly)")
    out.append("__device__ const float fe_boys_grid32s[(FE_BOYS32S_MMAX + 1) * FE_BOYS32_NROW"
               " * FE_BOYS32_TAYLOR_K] = {")
    for M in range(ms + 1):
        for i, r in enumerate(boys_grid32_scaled(M)):
            out.append("  " + ", ".join(repr(float(v)) + "f" if abs(v) > 1e-37 else "0.0f" for v in r) + ",")
    out.append("};")
    out.append("")
    # Boys grid
    # e^(-i h) on the Boys grid's spacing up to T = 64, beyond every FP64
    # asymptotic threshold (40-digit values): e^-T = e^(-i h) e^d, |d| <= h/2
    import mpmath as mp
    mp.mp.dps = 40
    nexp = int(64.0 / GRID_H) + 1
    out.append(f"#define FE_EXP_NROW {nexp}")
    out.append("// e^(-i h), h = FE_BOYS_GRID_H, i = 0..FE_EXP_NROW-1")
    out.append("__device__ const double fe_exp_grid[FE_EXP_NROW] = {")
    vals = [float(mp.exp(-mp.mpf(i) * mp.mpf(GRID_H))) for i in range(nexp)]
    for i in range(0, nexp, 6):
        out.append("  " + ", ".join(repr(v) for v in vals[i:i + 6]) + ",")
    out.append("};")
    out.append("")
    rows = boys_grid()
    out.append(f"// F_n(i*h), i = 0..{len(rows) - 1}, n = 0..FE_BOYS_NTAB-1")
    out.append(f"#define FE_BOYS_NROW {len(rows)}")
    out.append("__device__ const double fe_boys_grid[FE_BOYS_NROW * FE_BOYS_NTAB] = {")
    for r in rows:
        out.append("  " + ", ".join(repr(v) for v in r) + ",")
    out.append("};")
    out.append("")
    # contraction rows
    for L in range(LMAX + 1):
        keys, rows_ = H.class_terms(L)
        tix = H.t_index(L)
        ptr, col, val = [0], [], []
        for r in rows_:
            for t, c in r:
                col.append(tix[t])
                val.append(c)
            ptr.append(len(col))
        out.append(f"// class L={L}: M0 rows (etab compact index -> G term), nnz={len(col)}")
        out.append(f"__constant__ short fe_m0_ptr_L{L}[{len(ptr)}] = {{" + ", ".join(map(str, ptr)) + "};")
        out.append(f"__constant__ short fe_m0_col_L{L}[{len(col)}] = {{" + ", ".join(map(str, col)) + "};")
        out.append(f"__constant__ signed char fe_m0_m_L{L}[{len(keys)}] = {{"
                   + ", ".join(str(k[3]) for k in keys) + "};")
        vals = ", ".join(repr(float(v)) for v in val)
        out.append(f"__constant__ float fe_m0_val_L{L}[{len(val)}] = {{{vals}}};")
        assert all(abs(v) < 2 ** 24 and float(int(v)) == v for v in val)
    out.append("")
    # polynomial evaluators
    nops = []
    for L in range(LMAX + 1):
        lines, n = poly_functions(L)
        nops.append(n)
        out += lines
    # record position of every term (the builder writes G_k at fe_gpos_L[k])
    for L in range(LMAX + 1):
        pos = {k: i for i, k in enumerate(consumption_order(L))}
        out.append(f"__constant__ short fe_gpos_L{L}[{H.n_terms(L)}] = {{"
                   + ", ".join(str(pos[k]) for k in range(H.n_terms(L))) + "};")
    out.append("")
    out.append("static constexpr int fe_class_polyops[FE_NCLASS] = {"
               + ", ".join(map(str, nops)) + "};")
    out.append("")
    for L in range(LMAX + 1):
        out += f32_terms_function(L)
    out.append("template <int L>")
    out.append("__device__ __forceinline__ void fe_f32_terms(const double* __restrict__ g, double K,")
    out.append("    const double (&s)[L + 1], const double (&v)[L + 1], float* __restrict__ o,")
    out.append("    double (&b)[L + 1]) {")
    for L in range(LMAX + 1):
        kw = "if" if L == 0 else "else if"
        out.append(f"  {kw} constexpr (L == {L}) fe_f32_terms_L{L}(g, K, s, v, o, b);")
    out.append("}")
    out.append("")
    out.append(f"#define FE_M0_UNROLL_LMAX {M0_UNROLL_LMAX}")
    for L in range(M0_UNROLL_LMAX + 1):
        out += m0_functions(L)
    for name, args, call in (
            ("fe_m0_rows", "const double (&e)[fe_class_ntri[L]], double (&s)[fe_class_nterm[L]]",
             "(e, s)"),
            ("fe_g_store", "const double (&s)[fe_class_nterm[L]], const double (&pw)[L + 1], "
             "double cf, double* __restrict__ g", "(s, pw, cf, g)")):
        out.append("template <int L>")
        out.append(f"__device__ __forceinline__ void {name}({args}) {{")
        out.append("  static_assert(L <= FE_M0_UNROLL_LMAX, \"straight-line contraction not generated\");")
        for L in range(M0_UNROLL_LMAX + 1):
            kw = "if" if L == 0 else "else if"
            out.append(f"  {kw} constexpr (L == {L}) {name}_L{L}{call};")
        out.append("}")
    out.append("")
    for L in range(LMAX + 1):
        out += grad_function(L)
        out.append("")
    # compile-time dispatch on the class
    out.append("// s = sum_k G_k R^a F_m for class L; g: the record's coefficients (consumption order)")
    out.append("template <int L, typename Real, int NP>")
    out.append("__device__ __forceinline__ void fe_poly(const Real* __restrict__ g,")
    out.append("    const Real (&x)[NP], const Real (&y)[NP], const Real (&z)[NP],")
    out.append("    const Real (&F)[NP][L + 1], Real (&s)[NP]) {")
    for L in range(LMAX + 1):
        kw = "if" if L == 0 else "else if"
        out.append(f"  {kw} constexpr (L == {L}) {{")
        out.append(f"    if constexpr (sizeof(Real) == 4) fe_poly32_L{L}<NP>(g, x, y, z, F, s);")
        out.append(f"    else fe_poly64_L{L}<NP>(g, x, y, z, F, s);")
        out.append("  }")
    out.append("}")
    out.append("")
    out.append("// the same for two points per float2 lane (FP32 records, {g, g} coefficient pairs)")
    out.append("template <int L, int NP>")
    out.append("__device__ __forceinline__ void fe_poly32x2(const float* __restrict__ g,")
    out.append("    const float2 (&x)[NP], const float2 (&y)[NP], const float2 (&z)[NP],")
    out.append("    const float2 (&F)[NP][L + 1], float2 (&s)[NP]) {")
    for L in range(LMAX + 1):
        kw = "if" if L == 0 else "else if"
        out.append(f"  {kw} constexpr (L == {L}) fe_poly32x2_L{L}<NP>(g, x, y, z, F, s);")
    out.append("}")
    out.append("")
    out.append("// the asymptotic packed form (m-major classes only)")
    out.append("template <int L, int NP>")
    out.append("__device__ __forceinline__ void fe_poly32x2a(const float* __restrict__ g,")
    out.append("    const float2 (&x)[NP], const float2 (&y)[NP], const float2 (&z)[NP],")
    out.append("    const float2 (&ir2)[NP], float2 (&s)[NP]) {")
    for L in range(LMAX + 1):
        if poly_variant(L)[1] != "m-major":
            continue
        kw = "if" if L == 0 else "else if"
        out.append(f"  {kw} constexpr (L == {L}) fe_poly32x2a_L{L}<NP>(g, x, y, z, ir2, s);")
    out.append("}")
    out.append("")
    out.append("template <int L, typename Real, int NP>")
    out.append("__device__ __forceinline__ void fe_grad(const Real* __restrict__ g,")
    out.append("    const Real (&x)[NP], const Real (&y)[NP], const Real (&z)[NP],")
    out.append("    const Real (&F)[NP][L + 2], Real (&s)[NP], Real (&u)[NP],")
    out.append("    Real (&dx)[NP], Real (&dy)[NP], Real (&dz)[NP]) {")
    for L in range(LMAX + 1):
        kw = "if" if L == 0 else "else if"
        out.append(f"  {kw} constexpr (L == {L}) fe_grad_L{L}<Real, NP>(g, x, y, z, F, s, u, dx, dy, dz);")
    out.append("}")
    out.append("")
    # adjoint moment chunks
    chunks = [mom_chunks(L) for L in range(LMAX + 1)]
    nck = max(len(c) for c in chunks)
    out.append(f"#define FE_MOM_MAXCHUNK {nck}")
    out.append("static constexpr int fe_mom_nchunk[FE_NCLASS] = {"
               + ", ".join(str(len(c)) for c in chunks) + "};")
    for nm, idx in (("k0", 0), ("k1", 1)):
        rows = ["{" + ", ".join(str(c[i][idx]) if i < len(c) else "0" for i in range(nck)) + "}"
                for c in chunks]
        out.append(f"static constexpr int fe_mom_{nm}[FE_NCLASS][FE_MOM_MAXCHUNK] = {{"
                   + ", ".join(rows) + "};")
    out.append("")
    for L in range(LMAX + 1):
        for c, (k0, k1) in enumerate(chunks[L]):
            out += mom_function(L, c, k0, k1)
    out.append("template <int L, int C, typename Real>")
    out.append("__device__ __forceinline__ void fe_mom(Real x, Real y, Real z, const Real (&wF)[L + 1],")
    out.append("    Real (&acc)[fe_mom_k1[L][C] - fe_mom_k0[L][C]]) {")
    first = True
    for L in range(LMAX + 1):
        for c in range(len(chunks[L])):
            kw = "if" if first else "else if"
            first = False
            out.append(f"  {kw} constexpr (L == {L} && C == {c}) fe_mom_L{L}_c{c}<Real>(x, y, z, wF, acc);")
    out.append("}")
    out.append("")
    out.append("__constant__ int fe_c_rec64[FE_NCLASS] = {"
               + ", ".join(str(H.record_stride(L)) for L in range(LMAX + 1)) + "};")
    out.append("__constant__ int fe_c_rec32[FE_NCLASS] = {"
               + ", ".join(str(H.record_stride_f32(L)) for L in range(LMAX + 1)) + "};")
    out.append("__constant__ int fe_c_nterm[FE_NCLASS] = {"
               + ", ".join(map(str, nts)) + "};")
    (HERE / "classes_gen.cuh").write_text("\n".join(out) + "\n")
    print("classes_gen.cuh:", len(out), "lines; poly ops", nops, "terms", nts,
          "asym T", ths, "fp32 asym T", th32)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
