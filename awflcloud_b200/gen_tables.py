"""Derive the constant transform tables of the ADER/WENO scheme from first principles
and write them as a C header of exact hex-float literals (``csrc/awfl_tables.h``).

The tables are the ones the reference ships precomputed in TransformMatrices.h
(generated there by sage/generate_transform_source.sage); the definitions followed are
sage/transformation_matrices.sage and sage/poly_utils.sage:

* polynomial basis  p(x) = sum_j a_j x^j  on the unit cell [-1/2, 1/2];
* ``get_gll_points/weights(N)``: Gauss-Lobatto-Legendre nodes/weights mapped to
  [-1/2, 1/2] (weights sum to 1) -- sage/quadrature_utils.sage:15-50;
* ``gll_to_coefs(N)`` / ``coefs_to_gll(N)``: inverse / Vandermonde at the GLL nodes
  (transformation_matrices.sage:8-16);
* ``coefs_to_deriv(N)``: d/dx on coefficients (transformation_matrices.sage:178-185);
* ``sten_to_coefs(N)``: N unit-width cell averages centred on 0 -> coefficients
  (transformation_matrices.sage:43-51);
* ``coefs_to_gll_lower(N, M)``: N coefficients -> M GLL point values (M=1: x=0)
  (transformation_matrices.sage:210-228);
* ``weno_sten_to_coefs(N)``: hs+1 candidate polynomials of hs+1 coefficients on the
  sub-stencils j..j+hs, plus the full N-coefficient polynomial
  (transformation_matrices.sage:231-254);
* ``coefs_to_tv(N)``: sum_{d=1}^{N-1} integral over the cell of (p^(d))^2, where -- as in
  the reference's integrate_poly (poly_utils.sage:21-26) -- the integrand is TRUNCATED to
  its first N Taylor coefficients before integration.

Every matrix is stored in the reference's (col,row) convention (sage/c_utils.sage:38-51):
``out[row] = sum_col M[col][row] * in[col]``, C-order with the column index first.

Values are computed in mpmath at 256 bits and rounded to double the way the reference's
literals are: to the x87 64-bit-mantissa long double (its ``_fp`` literal operator,
const.h:31-33) and then to double, both round-to-nearest-even.

Run:  python -m awflcloud_b200.gen_tables   (rewrites csrc/awfl_tables.h)
"""
from __future__ import annotations

import os
import struct

from fractions import Fraction

import mpmath as mp

mp.mp.prec = 256
HALF = mp.mpf(1) / 2


# ----------------------------------------------------------------------------- rounding
def _round_mant(x: mp.mpf, bits: int) -> mp.mpf:
    """Round x to ``bits`` significant bits, nearest-even (no exponent range limits)."""
    if x == 0:
        return mp.mpf(0)
    m, e = mp.frexp(x)  # x = m * 2^e, 0.5 <= |m| < 1
    scaled = m * mp.mpf(2) ** bits
    fl = mp.floor(scaled)
    rem = scaled - fl
    if rem > HALF or (rem == HALF and int(fl) % 2 == 1):
        fl += 1
    return mp.ldexp(fl, int(e) - bits)


def to_double(x) -> float:
    """long-double (64-bit mantissa) rounding followed by double rounding."""
    x = mp.mpf(x)
    y = _round_mant(_round_mant(x, 64), 53)
    return float(y)  # exact: y has <= 53 significant bits


def hexlit(v: float) -> str:
    if v == 0.0:
        return "0.0" if struct.pack(">d", v)[0] == 0 else "-0.0"
    return float.hex(v)


# ----------------------------------------------------------------------------- math
def gll_nodes_weights(n: int):
    """GLL nodes/weights on [-1,1]: endpoints plus the roots of P'_{n-1}."""
    if n == 1:
        return [mp.mpf(0)], [mp.mpf(2)]
    N = n - 1
    # Legendre P_N coefficients via the three-term recurrence (highest degree last)
    P = [[mp.mpf(1)], [mp.mpf(0), mp.mpf(1)]]
    for k in range(1, N):
        a = [mp.mpf(0)] + [(2 * k + 1) * c for c in P[k]]  # (2k+1) x P_k
        b = P[k - 1] + [mp.mpf(0)] * 2
        P.append([(a[i] - k * b[i]) / (k + 1) for i in range(k + 2)])
    PN = P[N]
    dPN = [i * PN[i] for i in range(1, len(PN))]
    interior = []
    if len(dPN) > 1:
        roots = mp.polyroots(list(reversed(dPN)), maxsteps=500, extraprec=600)
        interior = sorted(mp.re(r) for r in roots)
    x = [mp.mpf(-1)] + interior + [mp.mpf(1)]

    def pn(t):
        return sum(PN[i] * t ** i for i in range(len(PN)))

    w = [mp.mpf(2) / (N * n * pn(t) ** 2) for t in x]
    return x, w


def gll_points(n):
    x, _ = gll_nodes_weights(n)
    return [t / 2 for t in x]


def gll_weights(n):
    _, w = gll_nodes_weights(n)
    return [t / 2 for t in w]


def cell_avg_monomial(j: int, lo, hi):
    """Average of x^j over [lo, hi]."""
    return (hi ** (j + 1) - lo ** (j + 1)) / ((j + 1) * (hi - lo))


def minv(rows):
    return mp.matrix(rows) ** -1


def qinv(rows):
    """Exact inverse of a rational matrix (Gauss-Jordan over Fractions); returns mpf."""
    n = len(rows)
    a = [[Fraction(v) for v in r] + [Fraction(int(i == j)) for j in range(n)] for i, r in enumerate(rows)]
    for c in range(n):
        p = next(r for r in range(c, n) if a[r][c] != 0)
        a[c], a[p] = a[p], a[c]
        piv = a[c][c]
        a[c] = [v / piv for v in a[c]]
        for r in range(n):
            if r != c and a[r][c] != 0:
                f = a[r][c]
                a[r] = [vr - f * vc for vr, vc in zip(a[r], a[c])]
    return mp.matrix([[mp.mpf(v.numerator) / v.denominator for v in r[n:]] for r in a])


def qcell_avg_monomial(j: int, lo: Fraction, hi: Fraction) -> Fraction:
    return (hi ** (j + 1) - lo ** (j + 1)) / ((j + 1) * (hi - lo))


def as_colrow(mat_row_col, ncol, nrow):
    """(row,col) math matrix -> reference (col,row) storage, list [col][row]."""
    return [[mat_row_col[r][c] for r in range(nrow)] for c in range(ncol)]


def vandermonde(pts, ncoef):
    return [[p ** j for j in range(ncoef)] for p in pts]


def gll_to_coefs(n):
    V = minv(vandermonde(gll_points(n), n))
    return as_colrow([[V[r, c] for c in range(n)] for r in range(n)], n, n)


def coefs_to_gll(n):
    return as_colrow(vandermonde(gll_points(n), n), n, n)


def coefs_to_gll_lower(n, m):
    pts = [mp.mpf(0)] if m == 1 else gll_points(m)
    return as_colrow(vandermonde(pts, n), n, m)


def coefs_to_deriv(n):
    D = [[mp.mpf(0)] * n for _ in range(n)]
    for j in range(1, n):
        D[j - 1][j] = mp.mpf(j)
    return as_colrow(D, n, n)


def sten_to_coefs(n):
    hs = (n - 1) // 2
    h = Fraction(1, 2)
    A = [[qcell_avg_monomial(j, c - h, c + h) for j in range(n)] for c in range(-hs, hs + 1)]
    Ai = qinv(A)
    return as_colrow([[Ai[r, c] for c in range(n)] for r in range(n)], n, n)


def weno_sten_to_coefs(n):
    """recon[j][s][ii]: candidate j, stencil cell s, coefficient ii."""
    hs = (n - 1) // 2
    edges = [Fraction(2 * i - 1, 2) for i in range(-hs, hs + 2)]
    rec = [[[mp.mpf(0)] * n for _ in range(n)] for _ in range(hs + 2)]
    for j in range(hs + 1):
        A = [[qcell_avg_monomial(q, edges[i], edges[i + 1]) for q in range(hs + 1)]
             for i in range(j, j + hs + 1)]
        Ai = qinv(A)
        for s in range(hs + 1):
            for ii in range(hs + 1):
                rec[j][s][ii] = Ai[ii, s]
    A = [[qcell_avg_monomial(q, edges[i], edges[i + 1]) for q in range(n)] for i in range(n)]
    Ai = qinv(A)
    for s in range(n):
        for ii in range(n):
            rec[hs + 1][s][ii] = Ai[ii, s]
    # pad to (n, n, n) exactly like SArray<real,3,ord,ord,ord>; unused candidates stay 0
    while len(rec) < n:
        rec.append([[mp.mpf(0)] * n for _ in range(n)])
    return rec


def tv_terms(n):
    """Quadratic form of coefs_to_tv(n) as an ordered list (m, q, coef).

    Order and grouping follow the reference expression: for q = 1..n-1 ascending, for
    m = q%2 ? 1 : 2 ... q step 2; squares are evaluated as c*(a_q*a_q), cross terms as
    (c*a_m)*a_q, summed left to right.
    """
    # coefficient of x^k in (p^(d))^2 for the pair (m, q), truncated to k < n
    def integ_even(k):
        return 2 * HALF ** (k + 1) / (k + 1) if k % 2 == 0 else mp.mpf(0)

    def ff(j, d):  # j!/(j-d)!
        r = mp.mpf(1)
        for t in range(j - d + 1, j + 1):
            r *= t
        return r

    terms = []
    for q in range(1, n):
        for m in range(2 - q % 2, q + 1, 2):
            c = mp.mpf(0)
            for d in range(1, n):
                if d > m or d > q:
                    continue
                k = (m - d) + (q - d)
                if k >= n:
                    continue
                prod = ff(m, d) * ff(q, d)
                c += (prod if m == q else 2 * prod) * integ_even(k)
            if c != 0:
                terms.append((m, q, c))
    return terms


# ----------------------------------------------------------------------------- emitters
ORDS = ((5, 3), (9, 5))


def _arr(name, vals):
    return "static const double %s[%d] = {%s};\n" % (
        name, len(vals), ", ".join(hexlit(to_double(v)) for v in vals))


def _flat2(m):
    return [v for col in m for v in col]


def emit_header() -> str:
    out = []
    out.append("// GENERATED by awflcloud_b200/gen_tables.py -- do not edit by hand.\n")
    out.append("// Exact-value ADER/WENO transform tables, (col,row) storage: out[row] = sum_col M[col*nrow+row]*in[col].\n")
    out.append("#pragma once\n\n")
    for ordv, ngll in ORDS:
        hs = (ordv - 1) // 2
        sfx = "o%d" % ordv
        out.append("// ---- ord = %d, ngll = %d\n" % (ordv, ngll))
        rec = weno_sten_to_coefs(ordv)
        out.append(_arr("awfl_weno_recon_%s" % sfx, [rec[a][b][c] for a in range(ordv) for b in range(ordv) for c in range(ordv)]))
        out.append(_arr("awfl_sten_to_coefs_%s" % sfx, _flat2(sten_to_coefs(ordv))))
        out.append(_arr("awfl_coefs_to_gll_lower_%s" % sfx, _flat2(coefs_to_gll_lower(ordv, ngll))))
        out.append(_arr("awfl_gll_to_coefs_n%d_%s" % (ngll, sfx), _flat2(gll_to_coefs(ngll))))
        out.append(_arr("awfl_coefs_to_deriv_n%d_%s" % (ngll, sfx), _flat2(coefs_to_deriv(ngll))))
        out.append(_arr("awfl_coefs_to_gll_n%d_%s" % (ngll, sfx), _flat2(coefs_to_gll(ngll))))
        out.append(_arr("awfl_gll_pts_ord_%s" % sfx, gll_points(ordv)))
        out.append(_arr("awfl_gll_wts_ord_%s" % sfx, gll_weights(ordv)))
        out.append(_arr("awfl_gll_pts_ngll_%s" % sfx, gll_points(ngll)))
        out.append(_arr("awfl_gll_wts_ngll_%s" % sfx, gll_weights(ngll)))
        for n, tag in ((hs + 1, "lo"), (ordv, "hi")):
            t = tv_terms(n)
            out.append("// coefs_to_tv(%d): terms (m, q, c) evaluated in this order\n" % n)
            out.append("#define AWFL_TV_%s_%s_NTERM %d\n" % (tag.upper(), sfx.upper(), len(t)))
            out.append("static const int awfl_tv_%s_%s_m[%d] = {%s};\n" % (tag, sfx, len(t), ", ".join(str(a) for a, _, _ in t)))
            out.append("static const int awfl_tv_%s_%s_q[%d] = {%s};\n" % (tag, sfx, len(t), ", ".join(str(b) for _, b, _ in t)))
            out.append(_arr("awfl_tv_%s_%s_c" % (tag, sfx), [c for _, _, c in t]))
        out.append("\n")
    return "".join(out)


def emit_tv_header() -> str:
    """C++ (host + device) evaluators of coefs_to_tv, one straight-line function per n,
    in the reference's term order; templated on the arithmetic type."""
    out = ["// GENERATED by awflcloud_b200/gen_tables.py -- do not edit by hand.\n",
           "// coefs_to_tv(n) evaluators: r = c0*(a_q*a_q); r = r + (c*a_m)*a_q ... in the\n",
           "// reference's term order (TransformMatrices.h coefs_to_tv).\n",
           "#pragma once\n\n",
           "#if defined(__CUDACC__)\n#define AWFL_TV_HD __host__ __device__ __forceinline__\n",
           "#else\n#define AWFL_TV_HD inline\n#endif\n\n"]
    done = set()
    for ordv, _ in ORDS:
        hs = (ordv - 1) // 2
        for n in (hs + 1, ordv):
            if n in done:
                continue
            done.add(n)
            out.append("template <class T> AWFL_TV_HD T awfl_tv_n%d(const T *a) {\n" % n)
            for t, (m, q, c) in enumerate(tv_terms(n)):
                lit = "T(%s)" % hexlit(to_double(c))
                term = ("%s * (a[%d] * a[%d])" % (lit, q, q)) if m == q else ("%s * a[%d] * a[%d]" % (lit, m, q))
                out.append(("  T r = %s;\n" % term) if t == 0 else ("  r = r + %s;\n" % term))
            out.append("  return r;\n}\n\n")
    # gradients for the discrete adjoint: g[m] += lam * d(tv)/d(a[m])
    out.append("// Gradients of the quadratic forms above: g[m] += lam * d tv / d a[m].\n")
    for n in sorted(done):
        out.append("template <class T> AWFL_TV_HD void awfl_tv_grad_n%d(const T *a, T lam, T *g) {\n" % n)
        for m, q, c in tv_terms(n):
            if m == q:
                out.append("  g[%d] += lam * (T(%s) * a[%d]);\n" % (q, hexlit(2 * to_double(c)), q))
            else:
                lit = hexlit(to_double(c))
                out.append("  g[%d] += lam * (T(%s) * a[%d]);\n" % (m, lit, q))
                out.append("  g[%d] += lam * (T(%s) * a[%d]);\n" % (q, lit, m))
        out.append("}\n\n")
    return "".join(out)


def _split_bits(x, bits):
    """x rounded to ``bits`` significant bits (so that small-integer multiples are exact)."""
    return _round_mant(mp.mpf(x), bits)


def emit_pow_header() -> str:
    """Tables of the correctly rounded pow (csrc/awfl_pow.cuh):
    log: for j in 0..127, inv_j = double(1 / (1 + (j + 1/2)/128)) and -ln(inv_j) as a
    double-double; exp: 2^(j/64) for j in 0..63 as double-doubles; ln2 split as
    L2HI (42 bits) + L2LO, and ln2/64 split as E1 (36 bits) + E2."""
    out = ["// GENERATED by awflcloud_b200/gen_tables.py -- do not edit by hand.\n",
           "// Tables for awfl_pow.cuh (values exact to 256 bits before rounding).\n",
           "#pragma once\n\n",
           "#ifdef __CUDACC__\n#define AWFL_POW_TABLE __device__ const double\n",
           "#else\n#define AWFL_POW_TABLE static const double\n#endif\n\n"]
    inv, th, tl = [], [], []
    for j in range(128):
        c = 1 + (mp.mpf(j) + HALF) / 128
        iv = float(_round_mant(1 / c, 53))
        lv = -mp.log(mp.mpf(iv))
        hi = float(_round_mant(lv, 53))
        lo = float(_round_mant(lv - mp.mpf(hi), 53))
        inv.append(iv); th.append(hi); tl.append(lo)
    e2h, e2l = [], []
    for j in range(64):
        v = mp.mpf(2) ** (mp.mpf(j) / 64)
        hi = float(_round_mant(v, 53))
        lo = float(_round_mant(v - mp.mpf(hi), 53))
        e2h.append(hi); e2l.append(lo)
    ln2 = mp.log(2)
    l2hi = float(_split_bits(ln2, 42))
    l2lo = float(_round_mant(ln2 - mp.mpf(l2hi), 53))
    q = ln2 / 64
    e1 = float(_split_bits(q, 36))
    e2 = float(_round_mant(q - mp.mpf(e1), 53))
    inv64 = float(_round_mant(64 / ln2, 53))

    def arr(name, vals):
        return "AWFL_POW_TABLE %s[%d] = {%s};\n" % (name, len(vals), ", ".join(hexlit(v) for v in vals))

    out.append(arr("awfl_pow_log_inv", inv))
    out.append(arr("awfl_pow_log_hi", th))
    out.append(arr("awfl_pow_log_lo", tl))
    out.append(arr("awfl_pow_exp_hi", e2h))
    out.append(arr("awfl_pow_exp_lo", e2l))
    out.append("#define AWFL_POW_L2HI %s\n#define AWFL_POW_L2LO %s\n" % (hexlit(l2hi), hexlit(l2lo)))
    out.append("#define AWFL_POW_E1 %s\n#define AWFL_POW_E2 %s\n#define AWFL_POW_INV_E %s\n"
               % (hexlit(e1), hexlit(e2), hexlit(inv64)))
    return "".join(out)


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, "csrc", "awfl_tables.h")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write(emit_header())
    print("wrote", path)
    path = os.path.join(here, "csrc", "awfl_tv.h")
    with open(path, "w") as f:
        f.write(emit_tv_header())
    print("wrote", path)
    path = os.path.join(here, "csrc", "awfl_pow_tables.h")
    with open(path, "w") as f:
        f.write(emit_pow_header())
    print("wrote", path)


if __name__ == "__main__":
    main()
