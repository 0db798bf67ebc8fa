"""Exact algorithmic operation count of one cell-split of the ADER/WENO step.

Runs the per-cell arithmetic of one directional split -- reconstruction of the five
variables (WENO or linear), ADER differential transform, edge time average, one Riemann
flux, the divergence and the apply -- through a counting scalar type, following the same
loops as the FP64 kernels (csrc/awfl_device.cuh), which restate the reference
(Spatial_euler3d_cons_expl_cart_fv_Agrid.h:665-956, 1800-2177; WenoLimiter.h:93-172).

Counts are per cell per split: one face flux per cell (the faces are shared, L+1 faces for
L cells, i.e. one per cell up to the 1/L end face). Each add, subtract, multiply, divide
and square root is one operation; pow is counted separately (``pow``) and once in
``flops``; negations, comparisons and selects are not counted.
"""
from __future__ import annotations

from collections import Counter

HS_OF = {5: 2, 9: 4}
NG_OF = {5: 3, 9: 5}


class N:
    """A number that only counts the arithmetic done with it."""
    c = Counter()

    def _op(self, kind):
        N.c[kind] += 1
        return N()

    def __add__(self, o): return self._op("add")
    __radd__ = __add__
    def __sub__(self, o): return self._op("add")
    def __rsub__(self, o): return self._op("add")
    def __mul__(self, o): return self._op("mul")
    __rmul__ = __mul__
    def __truediv__(self, o): return self._op("div")
    def __rtruediv__(self, o): return self._op("div")
    def __neg__(self): return N()
    def __gt__(self, o): return True


def _pow(a, b):
    N.c["pow"] += 1
    return N()


def _sqrt(a):
    N.c["sqrt"] += 1
    return N()


def _tv(a, n):
    # coefs_to_tv(n): one multiply per square, two per cross term, one add per term after the first
    from .gen_tables import tv_terms
    r = None
    for m, q, _ in tv_terms(n):
        t = 3.0 * (a[q] * a[q]) if m == q else 3.0 * a[m] * a[q]
        r = t if r is None else r + t
    return r


def _weno(u, o):
    hs = HS_OF[o]
    a = [[0.0] * o for _ in range(hs + 2)]
    for i in range(hs + 1):
        for ii in range(hs + 1):
            for s in range(hs + 1):
                a[i][ii] = a[i][ii] + 1.5 * u[i + s]
    for ii in range(o):
        for s in range(o):
            a[hs + 1][ii] = a[hs + 1][ii] + 1.5 * u[s]
    for i in range(hs + 1):
        for ii in range(hs + 1):
            a[hs + 1][ii] = a[hs + 1][ii] - 1.5 * a[i][ii]
    for ii in range(o):
        a[hs + 1][ii] = a[hs + 1][ii] / 1.5
    tv = [_tv(a[i][:hs + 1], hs + 1) for i in range(hs + 1)] + [_tv(a[hs + 1], o)]
    lo = 0.0
    for i in range(hs + 1):
        lo = lo + tv[i]
    lo = lo / (hs + 1)
    tv[hs + 1] = lo + (tv[hs + 1] - lo) * 1.5
    w = [1.5 / (tv[i] * tv[i] + 1e-20) for i in range(hs + 2)]
    for _ in range(2):
        s = 0.0
        for i in range(hs + 2):
            s = s + w[i]
        w = [wi / (s + 1e-20) for wi in w]
        if _ == 0:
            d = 1.5
            w = [wi * (d + d * d - 3.0 * d * wi + wi * wi) / (d * d + wi * (1.0 - 2.0 * d)) for wi in w]
    aw = [0.0] * o
    for i in range(hs + 2):
        for ii in range(o):
            aw[ii] = aw[ii] + w[i] * a[i][ii]
    return aw


def count_cell_split(o: int = 5, direction: int = 0, weno: bool = True) -> Counter:
    """Operation counts of one cell-split (fused recon + flux + divergence + apply)."""
    N.c = Counter()
    ng, na = NG_OF[o], NG_OF[o]
    nm = 1 + direction
    q = [[[None] * ng for _ in range(na)] for _ in range(5)]
    for v in range(5):
        u = [N() for _ in range(o)]
        if weno:
            wc = _weno(u, o)
            for ii in range(ng):
                t = 0.0
                for s in range(o):
                    t = t + 1.5 * wc[s]
                q[v][0][ii] = t
        else:
            for ii in range(ng):
                t = 0.0
                for s in range(o):
                    t = t + 1.5 * u[s]
                q[v][0][ii] = t
    for ii in range(ng):
        q[0][0][ii] = q[0][0][ii] + 1.5
        q[4][0][ii] = q[4][0][ii] + 1.5
    f = [[[None] * ng for _ in range(na)] for _ in range(4)]
    g = [[None] * ng for _ in range(na)]
    src = None
    for ii in range(ng):
        r = q[0][0][ii]
        vel = [q[m][0][ii] / r for m in (1, 2, 3)]
        t = q[4][0][ii] / r
        vn = vel[nm - 1]
        for x, X in enumerate(vel + [t]):
            f[x][0][ii] = r * vn * X
        g[0][ii] = _pow(r * t, 1.4)
        if direction == 2:
            src = -(q[0][0][ii] - 1.5) * 9.81
    sr = [[src] * ng for _ in range(na)]
    for kt in range(1, na):
        for ii in range(ng):
            for x in range(4):
                f[x][kt][ii] = 0.0
            g[kt][ii] = 0.0
    for kt in range(na - 1):
        for ii in range(ng):
            dq = [0.0] * 5
            for s in range(ng):
                D = 1.5
                dq[0] = dq[0] + D * q[nm][kt][s]
                for m in (1, 2, 3):
                    if m == nm:
                        if direction == 2 and kt == 0:
                            dq[m] = dq[m] + D * (f[m - 1][kt][s] + 27.5 * g[kt][s] - 1.5)
                        elif kt == 0:
                            dq[m] = dq[m] + D * (f[m - 1][kt][s] + 27.5 * g[kt][s])
                        else:
                            dq[m] = dq[m] + D * (f[m - 1][kt][s] + 27.5 * g[kt][s] / 2)
                    else:
                        dq[m] = dq[m] + D * f[m - 1][kt][s]
                dq[4] = dq[4] + D * f[3][kt][s]
            for m in range(5):
                q[m][kt + 1][ii] = -dq[m] / 2.0 / (kt + 1.0)
            if direction == 2:
                q[3][kt + 1][ii] = -dq[3] / 2.0 / (kt + 1.0) + sr[kt][ii] / (kt + 1.0)
                sr[kt + 1][ii] = -q[0][kt + 1][ii] * 9.81
        if kt + 1 < na - 1 or True:
            for ii in range(ng):
                tot = [0.0] * 4
                for ir in range(kt + 2):
                    for x in range(4):
                        tot[x] = tot[x] + q[nm][ir][ii] * q[x + 1][kt + 1 - ir][ii] - q[0][ir][ii] * f[x][kt + 1 - ir][ii]
                for x in range(4):
                    f[x][kt + 1][ii] = tot[x] / q[0][0][ii]
                tg = 0.0
                for ir in range(kt + 1):
                    tg = tg + (kt + 1.0 - ir) * (1.4 * g[ir][ii] * q[4][kt + 1 - ir][ii] - q[4][ir][ii] * g[kt + 1 - ir][ii])
                g[kt + 1][ii] = (1.4 * g[0][ii] * q[4][kt + 1][ii] + tg / (kt + 1.0)) / q[4][0][ii]
    for v in range(5):
        for e in (0, ng - 1):
            acc = q[v][0][e]
            dm = 1.5
            for kt in range(1, na):
                acc = acc + q[v][kt][e] * dm / (kt + 1.0)
                dm = dm * 1.5
    if direction == 2:
        dm = 1.5
        for kt in range(1, na):
            for ii in range(ng):
                sr[0][ii] = sr[0][ii] + sr[kt][ii] * dm / (kt + 1.0)
            dm = dm * 1.5
        sa = 0.0
        for ii in range(ng):
            sa = sa + sr[0][ii] * 1.5
    # Riemann flux at one face
    qL = [N() for _ in range(5)]
    qR = [N() for _ in range(5)]
    r = 0.5 * (qL[0] + qR[0])
    if direction == 1:
        vel = [0.5 * (qL[m] + qR[m]) for m in (1, 2, 3)]
        t = 0.5 * (qL[4] + qR[4])
    else:
        vel = [0.5 * (qL[m] / qL[0] + qR[m] / qR[0]) for m in (1, 2, 3)]
        t = 0.5 * (qL[4] / qL[0] + qR[4] / qR[0])
    p = 27.5 * _pow(r * t, 1.4)
    cs = _sqrt(1.4 * p / r)
    vn = vel[direction]
    ta = [x for x in (0, 1, 2) if x != direction]
    w1 = qL[0] - qL[4] / t
    w2 = qL[1 + ta[0]] - vel[ta[0]] * qL[4] / t
    w3 = qL[1 + ta[1]] - vel[ta[1]] * qL[4] / t
    w5 = vn * qR[0] / (2 * cs) - qR[nm] / (2 * cs) + qR[4] / (2 * t)
    w6 = -vn * qL[0] / (2 * cs) + qL[nm] / (2 * cs) + qL[4] / (2 * t)
    q1 = w1 + w5 + w6
    qn = vn * w1 + (vn - cs) * w5 + (vn + cs) * w6
    qa = w2 + vel[ta[0]] * w5 + vel[ta[0]] * w6
    qb = w3 + vel[ta[1]] * w5 + vel[ta[1]] * w6
    q5 = t * w5 + t * w6
    F = [qn, qn * qn / q1 + 27.5 * _pow(q5, 1.4), qn * qa / q1, qn * qb / q1, qn * q5 / q1]
    if direction == 2:
        F[3] = F[3] - 1.5
    # divergence + apply
    for v in range(5):
        d = -(F[v] - N()) / 2.0
        if direction == 2 and v == 3:
            d = sa + d
        elif direction == 2:
            d = 0.0 + d
        _ = N() + 1.5 * d
    c = Counter(N.c)
    c["flops"] = c["add"] + c["mul"] + c["div"] + c["sqrt"] + c["pow"]
    return c


def flops_per_cell_step(o: int = 5, weno: bool = True) -> dict:
    """Sum over the three directional splits of one time step."""
    tot = Counter()
    for d in range(3):
        tot.update(count_cell_split(o, d, weno))
    return dict(tot)


if __name__ == "__main__":
    for o in (5, 9):
        for d in range(3):
            print("ord", o, "dir", d, dict(count_cell_split(o, d)))
        print("ord", o, "per cell-step", flops_per_cell_step(o))
