#!/usr/bin/env python3
"""Generate ``quadrature_rules.h``: the symmetric quadrature rules of the DG solver.

The solver must integrate with the same rules as DG-Parallel to reproduce its
discretisation (a different rule of the same degree changes the nonlinear
volume and face integrals at the truncation-error level).  DG-Parallel selects

* triangles: the Dunavant rules of degree 1..10 with 1,3,4,6,7,12,13,16,19,25
  points (``GaussQuadratureTri.cc:138-168``, weights scaled by 1/2 in
  ``Integrator.cc:69``),
* tetrahedra: the Keast-type rules of degree 1,2,3,4,6,8 with 1,4,5,14,24,45
  points (``GaussQuadratureTet.cc:349-380``, weights scaled by 1/6 in
  ``Integrator.cc:92-97``),
* edges: Gauss-Legendre with ``n = floor(order/2)+1`` points on [-1,1]
  (``GaussLegendre1D.cc:271-274``),

and, for the solver's alternative rule option, Keast's 11-point tet rule of
degree 4 (the triangle alternatives are rules of the table above).

Each rule is written here as its orbit structure (barycentric symmetry classes)
with a low-precision seed for every orbit parameter and weight; the seed only
selects the solution branch.  The rule itself is the solution of its moment
equations (exact integration of every monomial up to the rule's degree), which
this script solves by Gauss-Newton in extended precision, so the emitted values
are correct to the last bit of a double rather than truncated decimal tables.
Gauss-Legendre nodes are Newton-refined roots of the Legendre polynomials.

Usage: python gen_quadrature.py > quadrature_rules.h
"""
import itertools
import math
import sys

import numpy as np

LD = np.longdouble

# --- orbit structures --------------------------------------------------------
# triangle orbits in barycentric coordinates (l0, l1, l2); reference point is
# (u, v) = (l1, l2) on the triangle (0,0),(1,0),(0,1).
#   ("S3",  w)          centroid
#   ("S21", a, w)       (a, a, 1-2a) and its 3 distinct permutations
#   ("S111", a, b, w)   (a, b, 1-a-b) and its 6 permutations
# weights are normalised to sum to 1 over the rule.
TRI_RULES = {
    1: [("S3", 1.0)],
    2: [("S21", 0.166667, 0.333333)],
    3: [("S3", -0.5625), ("S21", 0.2, 0.520833)],
    4: [("S21", 0.091576, 0.109952), ("S21", 0.445948, 0.223382)],
    5: [("S3", 0.225), ("S21", 0.101287, 0.125939), ("S21", 0.470142, 0.132394)],
    6: [("S21", 0.063089, 0.050845), ("S21", 0.249287, 0.116786),
        ("S111", 0.053145, 0.310352, 0.082851)],
    7: [("S3", -0.14957), ("S21", 0.260346, 0.175615), ("S21", 0.06513, 0.053347),
        ("S111", 0.04869, 0.312865, 0.077114)],
    8: [("S3", 0.144316), ("S21", 0.459293, 0.095092), ("S21", 0.170569, 0.103217),
        ("S21", 0.050547, 0.032458), ("S111", 0.008395, 0.263113, 0.02723)],
    9: [("S3", 0.097136), ("S21", 0.489683, 0.031335), ("S21", 0.43709, 0.077828),
        ("S21", 0.188204, 0.079648), ("S21", 0.04473, 0.025578),
        ("S111", 0.036838, 0.221963, 0.043284)],
    10: [("S3", 0.090818), ("S21", 0.485578, 0.036726), ("S21", 0.109482, 0.045321),
         ("S111", 0.141707, 0.30794, 0.072758), ("S111", 0.025004, 0.246673, 0.028327),
         ("S111", 0.009541, 0.066803, 0.009422)],
}

# tetrahedron orbits in barycentric coordinates (l0..l3); reference point is
# (u, v, w) = (l1, l2, l3) on the tet (0,0,0),(1,0,0),(0,1,0),(0,0,1).
#   ("S4", w)              centroid
#   ("S31", a, w)          (a, a, a, 1-3a), 4 points
#   ("S22", a, w)          (a, a, 1/2-a, 1/2-a), 6 points
#   ("S211", a, b, w)      (a, a, b, 1-2a-b), 12 points
TET_RULES = {
    1: [("S4", 1.0)],
    2: [("S31", 0.138197, 0.25)],
    3: [("S4", -0.8), ("S31", 0.166667, 0.45)],
    4: [("S22", 0.0, 0.019048), ("S31", 0.100527, 0.08859), ("S31", 0.314373, 0.132839)],
    6: [("S31", 0.214603, 0.039923), ("S31", 0.040674, 0.010077),
        ("S31", 0.322338, 0.055357), ("S211", 0.063661, 0.269672, 0.048214)],
    8: [("S4", -0.235962), ("S31", 0.127471, 0.024488), ("S31", 0.032079, 0.003949),
        ("S22", 0.049777, 0.026306), ("S22", 0.18373, 0.08298),
        ("S211", 0.231901, 0.022918, 0.025443), ("S211", 0.03797, 0.193746, 0.013432)],
}
# Alternative tet rules offered besides DG-Parallel's (the solver's rule option
# for workloads stated with other point counts): Keast's 11-point rule of
# degree 4 (a negative centroid weight).
TET_ALT_RULES = {
    4: [("S4", -0.078933), ("S31", 0.071429, 0.045733), ("S22", 0.100596, 0.149333)],
}
# parameters that define a rule exactly and are kept fixed (the edge-midpoint
# orbit of the 14-point tet rule sits at a = 0).
FIXED = {("TET", 4, 0, 0)}


def perms_unique(t):
    seen = []
    for p in itertools.permutations(t):
        if p not in seen:
            seen.append(p)
    return seen


def expand(dim, orbits, params):
    """Orbit list + flat parameter vector -> list of (barycentric tuple, weight)."""
    pts = []
    k = 0
    for orb in orbits:
        kind = orb[0]
        npar = len(orb) - 2
        vals = params[k:k + npar]
        w = params[k + npar]
        k += npar + 1
        if kind == "S3":
            base = (LD(1) / 3,) * 3
        elif kind == "S21":
            a = vals[0]
            base = (a, a, 1 - 2 * a)
        elif kind == "S111":
            a, b = vals
            base = (a, b, 1 - a - b)
        elif kind == "S4":
            base = (LD(1) / 4,) * 4
        elif kind == "S31":
            a = vals[0]
            base = (a, a, a, 1 - 3 * a)
        elif kind == "S22":
            a = vals[0]
            base = (a, a, LD(1) / 2 - a, LD(1) / 2 - a)
        elif kind == "S211":
            a, b = vals
            base = (a, a, b, 1 - 2 * a - b)
        else:
            raise ValueError(kind)
        # permutations are formed on a symbolic index pattern so that equal
        # parameter values produce the same number of points as the orbit type
        pattern = {"S3": (0, 0, 0), "S21": (0, 0, 1), "S111": (0, 1, 2),
                   "S4": (0, 0, 0, 0), "S31": (0, 0, 0, 1), "S22": (0, 0, 1, 1),
                   "S211": (0, 0, 1, 2)}[kind]
        distinct = {}
        for i, pi in enumerate(pattern):
            distinct.setdefault(pi, base[i])
        for pp in perms_unique(pattern):
            pts.append((tuple(distinct[i] for i in pp), w))
    return pts


def moments(dim, deg):
    """Exact integrals of monomials over the reference simplex normalised to volume 1."""
    out = []
    vol = LD(1) / math.factorial(dim)
    for exps in itertools.product(range(deg + 1), repeat=dim):
        if sum(exps) > deg:
            continue
        num = 1
        for e in exps:
            num *= math.factorial(e)
        exact = LD(num) / LD(math.factorial(sum(exps) + dim)) / vol
        out.append((exps, exact))
    return out


def residual(dim, orbits, params, mom):
    pts = expand(dim, orbits, params)
    r = []
    for exps, exact in mom:
        q = LD(0)
        for bary, w in pts:
            ref = bary[1:]
            t = w
            for x, e in zip(ref, exps):
                t = t * x ** e
            q += t
        r.append(q - exact)
    return np.array(r, dtype=LD)


def solve(kind, order, orbits):
    """kind: TRI, TET or TETALT (an alternative tet rule: no fixed parameters)."""
    dim = 2 if kind == "TRI" else 3
    params = []
    fixed = []
    for oi, orb in enumerate(orbits):
        for j, v in enumerate(orb[1:]):
            params.append(LD(v))
            fixed.append((kind, order, oi, j) in FIXED)
    params = np.array(params, dtype=LD)
    mom = moments(dim, order)
    free = [i for i, f in enumerate(fixed) if not f]
    for _ in range(60):
        r = residual(dim, orbits, params, mom)
        if float(np.max(np.abs(r))) < 1e-19:
            break
        J = np.zeros((len(r), len(free)), dtype=LD)
        h = LD(2) ** -30
        for c, i in enumerate(free):
            p1 = params.copy()
            p1[i] += h
            p2 = params.copy()
            p2[i] -= h
            J[:, c] = (residual(dim, orbits, p1, mom) - residual(dim, orbits, p2, mom)) / (2 * h)
        step, *_ = np.linalg.lstsq(J.astype(np.float64), r.astype(np.float64), rcond=None)
        params[free] -= step.astype(LD)
    r = residual(dim, orbits, params, mom)
    err = float(np.max(np.abs(r)))
    if err > 1e-15:
        raise RuntimeError(f"{kind} order {order}: moment residual {err}")
    return expand(dim, orbits, params), err


def gauss_legendre(n):
    """Nodes ascending on [-1,1] and weights, Newton on P_n in extended precision."""
    nodes = []
    weights = []
    for i in range(n):
        x = LD(math.cos(math.pi * (i + 0.75) / (n + 0.5)))
        for _ in range(100):
            p0, p1 = LD(1), x
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
            dp = n * (x * p1 - p0) / (x * x - 1)
            dx = p1 / dp
            x -= dx
            if abs(float(dx)) < 1e-21:
                break
        p0, p1 = LD(1), x
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
        dp = n * (x * p1 - p0) / (x * x - 1)
        nodes.append(x)
        weights.append(2 / ((1 - x * x) * dp * dp))
    order = sorted(range(n), key=lambda i: float(nodes[i]))
    return [nodes[i] for i in order], [weights[i] for i in order]


def fmt(x):
    return "%.17e" % float(x)


def main():
    out = sys.stdout
    out.write("// Generated by gen_quadrature.py -- do not edit.\n")
    out.write("// Symmetric simplex rules solved from their moment equations; weights sum to 1\n")
    out.write("// (multiply by the reference measure 1/2 or 1/6).  Points are (u,v[,w]).\n")
    out.write("// Plain C/C++ data (no namespace) so both the solver and the C oracle include it.\n")
    out.write("#ifndef DGP_QUADRATURE_RULES_H\n#define DGP_QUADRATURE_RULES_H\n\n")
    index = []
    for kind, rules in (("TRI", TRI_RULES), ("TET", TET_RULES)):
        dim = 2 if kind == "TRI" else 3
        for order, orbits in sorted(rules.items()):
            pts, err = solve(kind, order, orbits)
            name = f"dgp_q_{kind.lower()}{order}"
            out.write(f"// {kind} degree {order}: {len(pts)} points, max moment residual {err:.1e}\n")
            out.write(f"static const double {name}[{len(pts)}][{dim + 1}] = {{\n")
            for bary, w in pts:
                out.write("  {" + ", ".join(fmt(x) for x in bary[1:]) + ", " + fmt(w) + "},\n")
            out.write("};\n")
            index.append((kind, order, len(pts), name))
    for order, orbits in sorted(TET_ALT_RULES.items()):
        pts, err = solve("TETALT", order, orbits)
        name = f"dgp_q_tet{order}_{len(pts)}"
        out.write(f"// TET degree {order} (alternative): {len(pts)} points, max moment residual {err:.1e}\n")
        out.write(f"static const double {name}[{len(pts)}][4] = {{\n")
        for bary, w in pts:
            out.write("  {" + ", ".join(fmt(x) for x in bary[1:]) + ", " + fmt(w) + "},\n")
        out.write("};\n")
        index.append(("TETALT", order, len(pts), name))
    out.write("\n")
    for n in range(1, 11):
        x, w = gauss_legendre(n)
        out.write(f"static const double dgp_q_gl{n}[{n}][2] = {{\n")
        for xi, wi in zip(x, w):
            out.write("  {" + fmt(xi) + ", " + fmt(wi) + "},\n")
        out.write("};\n")
    out.write("\ntypedef struct { int dim, degree, npts; const double* data; } dgp_q_rule;\n")
    out.write("static const dgp_q_rule dgp_q_tri_rules[] = {\n")
    for kind, order, n, name in index:
        if kind == "TRI":
            out.write(f"  {{2, {order}, {n}, &{name}[0][0]}},\n")
    out.write("};\nstatic const dgp_q_rule dgp_q_tet_rules[] = {\n")
    for kind, order, n, name in index:
        if kind == "TET":
            out.write(f"  {{3, {order}, {n}, &{name}[0][0]}},\n")
    out.write("};\nstatic const dgp_q_rule dgp_q_tet_alt_rules[] = {\n")
    for kind, order, n, name in index:
        if kind == "TETALT":
            out.write(f"  {{3, {order}, {n}, &{name}[0][0]}},\n")
    out.write("};\nstatic const double* const dgp_q_gauss_legendre[11] = {0")
    for n in range(1, 11):
        out.write(f", &dgp_q_gl{n}[0][0]")
    out.write("};\n\n#endif\n")


if __name__ == "__main__":
    main()
