"""The generated quadrature rules integrate monomials exactly to their degree
and are symmetric (the face-orientation maps rely on it)."""
import itertools
import math
import os
import re

import numpy as np
import pytest

from cases import ROOT

HDR = os.path.join(ROOT, "dg-parallel_b200", "csrc", "quadrature_rules.h")


def rules():
    src = open(HDR).read()
    out = {}
    for m in re.finditer(r"static const double dgp_q_(tri|tet|gl)(\d+)\[(\d+)\]\[\d\] = \{(.*?)\};", src, re.S):
        rows = [list(map(float, r.strip(" {},").split(","))) for r in m.group(4).strip().split("\n")]
        out[(m.group(1), int(m.group(2)))] = np.array(rows)
    return out


R = rules()


@pytest.mark.parametrize("key", sorted(k for k in R if k[0] in ("tri", "tet")))
def test_simplex_rule_exact(key):
    kind, deg = key
    P = R[key]
    dim = 2 if kind == "tri" else 3
    assert abs(P[:, -1].sum() - 1.0) < 1e-14
    for exps in itertools.product(range(deg + 1), repeat=dim):
        if sum(exps) > deg:
            continue
        exact = math.prod(math.factorial(e) for e in exps) / math.factorial(sum(exps) + dim)
        exact *= math.factorial(dim)
        q = np.sum(P[:, -1] * np.prod([P[:, i] ** e for i, e in enumerate(exps)], axis=0))
        assert abs(q - exact) <= 1e-14 * max(1.0, exact), (exps, q, exact)


@pytest.mark.parametrize("n", range(1, 11))
def test_gauss_legendre(n):
    P = R[("gl", n)]
    x, w = P[:, 0], P[:, 1]
    assert np.all(np.diff(x) > 0)
    for k in range(2 * n):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(np.sum(w * x ** k) - exact) < 1e-14


@pytest.mark.parametrize("deg", [1, 3, 5, 7])
def test_face_rules_symmetric(deg):
    P = R[("tri", deg)]
    pts = {(round(u, 12), round(v, 12)) for u, v, _ in P}
    for u, v, _ in P:
        lam = (1 - u - v, u, v)
        for p in itertools.permutations(range(3)):
            assert (round(lam[p[1]], 12), round(lam[p[2]], 12)) in pts
