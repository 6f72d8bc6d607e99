"""Generates ``dg_tables.h``: the 1-D Gauss-Legendre DG operators and the
limiter projection matrices for orders N = 0..9.

Everything is computed here from first principles in 80-digit decimal
arithmetic and only rounded at the end, the way the reference stores its
tables:

* Gauss-Legendre nodes and weights on [0,1] (the reference's
  ``kernels::gaussLegendreNodes/Weights``, GaussLegendreQuadrature.cpp:33-164),
  Gauss-Lobatto nodes in descending order (GaussLobattoQuadrature.cpp:60-80).
* ``FLCoeff[i] = phi_i(0)``, ``FRCoeff[i] = phi_i(1)`` (DGMatrices.h:64-80),
  stored as full doubles.
* ``dudx[l][n] = phi_n'(x_l)`` (DGMatrices.h:50),
  ``Kxi[k][l] = w_l phi_k'(x_l)`` (stiffness, DGMatrices.h:47),
  ``iK1 = (FR FR^T - Kxi)^-1`` laid out so that ``lQi[l] = sum_n iK1[l][n] rhs[n]``
  (DGMatrices.h:58). The reference prints these three with 13 significant
  digits (DGMatrices.cpp:257-288); the same rounding is applied here so that
  the GPU path multiplies by the same numbers as the reference.
* ``fineGridProjector1d[j][n][m] = phi_n((j + x_m)/3)`` (AMR prolongation and
  restriction between a cell and its thirds, DGMatrices.h:109) and
  ``equidistantGridProjector1d[n][i] = phi_n(i/N)`` (plotting at N+1
  equidistant points, DGMatrices.h:99), both with 13 significant digits as
  printed by the reference.
* ``uh2lim[k][i]`` = mean of phi_k over subcell i of 2N+1,
  ``uh2lob[j][i] = phi_j(lobatto_i)``, and ``lim2uh[i][j]``, the constrained
  least-squares inverse of uh2lim that conserves the cell mean
  (LimiterProjectionMatrices.cpp:39-136).

Run ``python gen_tables.py`` to rewrite dg_tables.h next to this file.
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import os

getcontext().prec = 80
MAXN = 9


def legendre(n, x):
    """P_n(x) and P_n'(x) by the three-term recurrence."""
    p0, p1 = Decimal(1), x
    if n == 0:
        return Decimal(1), Decimal(0)
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    if x * x == 1:  # endpoint: P_n'(+-1) = (+-1)^(n-1) n(n+1)/2
        return p1, (x ** (n - 1)) * n * (n + 1) / 2
    dp = n * (x * p1 - p0) / (x * x - 1)
    return p1, dp


def gauss_legendre(b):
    """Nodes/weights of the b-point Gauss-Legendre rule mapped to [0,1], ascending."""
    import math
    xs, ws = [], []
    for i in range(b):
        x = Decimal(math.cos(math.pi * (i + 0.75) / (b + 0.5)))
        for _ in range(200):
            p, dp = legendre(b, x)
            dx = p / dp
            x -= dx
            if abs(dx) < Decimal(10) ** -75:
                break
        p, dp = legendre(b, x)
        w = 2 / ((1 - x * x) * dp * dp)
        xs.append((1 - x) / 2)  # cos ordering is descending in x -> ascending in (1-x)/2
        ws.append(w / 2)
    order = sorted(range(b), key=lambda i: xs[i])
    return [xs[i] for i in order], [ws[i] for i in order]


def gauss_lobatto(b):
    """Nodes/weights of the b-point Gauss-Lobatto rule on [0,1], nodes descending."""
    import math
    if b == 1:
        return [Decimal("0.5")], [Decimal(1)]
    n = b - 1
    xs = [Decimal(1)]
    for i in range(1, n):
        x = Decimal(math.cos(math.pi * i / n))
        for _ in range(200):
            # roots of P_n'(x): Newton on P_n' with P_n'' from the Legendre ODE
            p, dp = legendre(n, x)
            d2p = (2 * x * dp - n * (n + 1) * p) / (1 - x * x)
            dx = dp / d2p
            x -= dx
            if abs(dx) < Decimal(10) ** -75:
                break
        xs.append(x)
    xs.append(Decimal(-1))
    ws = []
    for x in xs:
        p, _ = legendre(n, x)
        ws.append(Decimal(2) / (n * (n + 1) * p * p))
    return [(1 + x) / 2 for x in xs], [w / 2 for w in ws]


def lagrange(nodes, i, x):
    r = Decimal(1)
    for j, xj in enumerate(nodes):
        if j != i:
            r *= (x - xj) / (nodes[i] - xj)
    return r


def lagrange_deriv(nodes, i, x):
    s = Decimal(0)
    for m, xm in enumerate(nodes):
        if m == i:
            continue
        t = Decimal(1) / (nodes[i] - xm)
        for j, xj in enumerate(nodes):
            if j != i and j != m:
                t *= (x - xj) / (nodes[i] - xj)
        s += t
    return s


def invert(a):
    """Gauss-Jordan inverse in Decimal arithmetic."""
    n = len(a)
    m = [row[:] + [Decimal(int(i == j)) for j in range(n)] for i, row in enumerate(a)]
    for c in range(n):
        piv = max(range(c, n), key=lambda r: abs(m[r][c]))
        m[c], m[piv] = m[piv], m[c]
        pv = m[c][c]
        m[c] = [v / pv for v in m[c]]
        for r in range(n):
            if r != c and m[r][c] != 0:
                f = m[r][c]
                m[r] = [vr - f * vc for vr, vc in zip(m[r], m[c])]
    return [row[n:] for row in m]


def sig(x, digits):
    """Round to `digits` significant decimal digits (printf %.{digits-1}e)."""
    if x == 0:
        return 0.0
    return float(format(x, ".%de" % (digits - 1)))


def build(N):
    b = N + 1
    bl = 2 * N + 1
    x, w = gauss_legendre(b)
    xl, wl = gauss_lobatto(b)
    FL = [lagrange(x, i, Decimal(0)) for i in range(b)]
    FR = [lagrange(x, i, Decimal(1)) for i in range(b)]
    D = [[lagrange_deriv(x, n, x[l]) for n in range(b)] for l in range(b)]  # D[l][n] = phi_n'(x_l)
    Kxi = [[w[l] * D[l][k] for l in range(b)] for k in range(b)]
    K1 = [[FR[k] * FR[l] - Kxi[k][l] for l in range(b)] for k in range(b)]
    iK1 = invert(K1)
    # subcell averages of phi_k: exact via b-point Gauss on each subcell
    uh2lim = [[Decimal(0)] * bl for _ in range(b)]
    dxi = Decimal(1) / bl
    for i in range(bl):
        for j in range(b):
            xi = i * dxi + dxi * x[j]
            for k in range(b):
                uh2lim[k][i] += w[j] * lagrange(x, k, xi)
    uh2lob = [[lagrange(x, j, xl[i]) for i in range(b)] for j in range(b)]
    # constrained least squares: minimise |uh2lim^T u - lim|^2 s.t. w.u = mean(lim)
    lsqm = [[Decimal(0)] * (b + 1) for _ in range(b + 1)]
    for i in range(b):
        for j in range(b):
            lsqm[i][j] = sum(2 * uh2lim[i][k] * uh2lim[j][k] for k in range(bl))
        lsqm[i][b] = w[i]
        lsqm[b][i] = -w[i]
    ainv = invert(lsqm)  # the reference's matrixInverse returns lsqm^-1
    lim2uh = [[Decimal(0)] * b for _ in range(bl)]
    for i in range(bl):
        rhs = [2 * uh2lim[j][i] for j in range(b)] + [dxi]
        for j in range(b):
            lim2uh[i][j] = sum(ainv[k][j] * rhs[k] for k in range(b + 1))
    # AMR: fine[j][n][m] = phi_n((j + x_m) / 3), basis n of the coarse cell at
    # node m of its j-th third; plotting: equi[n][i] = phi_n(i / N)
    fine = [[[lagrange(x, n, (j + x[m]) / 3) for m in range(b)] for n in range(b)] for j in range(3)]
    equi = [[lagrange(x, n, Decimal(i) / N) for i in range(b)] for n in range(b)]
    return dict(
        fineGridProjector1d=[sig(fine[j][n][m], 13) for j in range(3) for n in range(b) for m in range(b)],
        equidistantGridProjector1d=[sig(equi[n][i], 13) for n in range(b) for i in range(b)],
        nodes=[float(v) for v in x], weights=[float(v) for v in w],
        lobatto_nodes=[float(v) for v in xl], lobatto_weights=[float(v) for v in wl],
        FLCoeff=[float(v) for v in FL], FRCoeff=[float(v) for v in FR],
        FCoeff=[sig(v, 13) for v in FL] + [sig(v, 13) for v in FR],
        Kxi=[sig(Kxi[k][l], 13) for k in range(b) for l in range(b)],
        iK1=[sig(iK1[k][l], 13) for k in range(b) for l in range(b)],
        dudx=[sig(D[l][n], 13) for l in range(b) for n in range(b)],
        uh2lim=[float(uh2lim[k][i]) for k in range(b) for i in range(bl)],
        lim2uh=[float(lim2uh[i][j]) for i in range(bl) for j in range(b)],
        uh2lob=[float(uh2lob[j][i]) for j in range(b) for i in range(b)],
    )


NAMES = ["nodes", "weights", "lobatto_nodes", "lobatto_weights", "FLCoeff", "FRCoeff", "FCoeff",
         "Kxi", "iK1", "dudx", "uh2lim", "lim2uh", "uh2lob", "fineGridProjector1d", "equidistantGridProjector1d"]


def all_tables():
    return {N: build(N) for N in range(1, MAXN + 1)}


def write_header(path):
    tabs = all_tables()
    out = ["// Generated by gen_tables.py -- do not edit.",
           "// 1-D DG operators on [0,1] at Gauss-Legendre nodes and the limiter",
           "// projections, orders 1..%d, flattened row-major per order." % MAXN,
           "#pragma once", ""]
    for name in NAMES:
        offs, flat = [], []
        for N in range(1, MAXN + 1):
            offs.append(len(flat))
            flat.extend(tabs[N][name])
        out.append("static const int exa_tab_%s_off[%d] = {0, %s};" % (name, MAXN + 1, ", ".join(map(str, offs))))
        out.append("static const double exa_tab_%s[%d] = {" % (name, len(flat)))
        for i in range(0, len(flat), 4):
            out.append("  " + ", ".join("%.17g" % v for v in flat[i:i + 4]) + ",")
        out.append("};")
        out.append("")
    with open(path, "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    write_header(os.path.join(os.path.dirname(os.path.abspath(__file__)), "dg_tables.h"))
