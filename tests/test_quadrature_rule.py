"""The quadrature rule option (DGP_RULE_WORKLOAD): at P2 the point counts the
workloads state -- triangles the 7-point volume rule of degree 5, tets the
11-point volume rule and the 6-point face rule of degree 4 -- instead of
DG-Parallel's rules (6-point triangle volume, 14-point tet volume, 7-point tet
faces).  The reference has no such option, so the CUDA path is pinned against
the oracle with the same rule, and the rule itself against its moments.
"""
import itertools
import math
import os
import re

import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import SCALAR2D, SCALAR3D, TM110, rel
from oracle_bind import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
RULES_H = os.path.join(HERE, "..", "dg-parallel_b200", "csrc", "quadrature_rules.h")


def _table(name):
    text = open(RULES_H).read()
    m = re.search(r"static const double " + name + r"\[(\d+)\]\[(\d+)\] = \{(.*?)\};", text, re.S)
    rows = re.findall(r"\{([^{}]*)\}", m.group(3))
    return np.array([[float(v) for v in r.split(",")] for r in rows])


def test_alternative_tet_rule_integrates_degree_4():
    """Keast's 11-point rule: every monomial of degree <= 4 over the reference
    tet (weights sum to 1, i.e. times the volume 1/6)."""
    q = _table("dgp_q_tet4_11")
    assert q.shape == (11, 4)
    for e in itertools.product(range(5), repeat=3):
        if sum(e) > 4:
            continue
        exact = math.factorial(e[0]) * math.factorial(e[1]) * math.factorial(e[2]) / math.factorial(sum(e) + 3)
        got = np.sum(q[:, 3] * q[:, 0] ** e[0] * q[:, 1] ** e[1] * q[:, 2] ** e[2]) / 6.0
        assert abs(got - exact) < 1e-16, (e, got, exact)
    assert q[:, 3].min() < 0  # the centroid weight is negative


def _tri(tmp_path, n=8):
    m = meshgen.tri_square(n, n, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=1)
    p = str(tmp_path / f"tri{n}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _tet(tmp_path, n=3, tag=1):
    m = meshgen.tet_cube(n, seed=3, boundary_tag=tag)
    p = str(tmp_path / f"tet{n}_{tag}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def test_oracle_rule_changes_the_discretisation_only_slightly(tmp_path):
    msh = _tri(tmp_path)
    a = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, dgp.FIELD_GAUSS, SCALAR2D, rule=0)
    b = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, dgp.FIELD_GAUSS, SCALAR2D, rule=1)
    # the projection uses the volume rule too
    d = rel(b.state(), a.state())
    assert 1e-14 < d < 1e-2
    for o in (a, b):
        t = 0.0
        for _ in range(3):
            dt = o.cfl_dt(0.1)
            o.step(t, dt)
            t += dt
    assert 1e-14 < rel(b.state(), a.state()) < 1e-2
    # orders other than P2 keep the reference rule
    c = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 3, dgp.FIELD_GAUSS, SCALAR2D, rule=0)
    e = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 3, dgp.FIELD_GAUSS, SCALAR2D, rule=1)
    assert np.array_equal(c.state(), e.state())


CASES = [
    ("scalar_tri", "tri", dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D, 1),
    ("scalar_tet", "tet", dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS3D, SCALAR3D, 1),
    ("maxwell3d_pec", "tet", dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, TM110, 40000),
]


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fused", "separate"])
@pytest.mark.parametrize("cid,kind,law,flux,field,prm,tag", CASES)
def test_gpu_workload_rule_matches_oracle(tmp_path, cid, kind, law, flux, field, prm, tag, form):
    msh = _tri(tmp_path) if kind == "tri" else _tet(tmp_path, tag=tag)
    o = Oracle(msh, law, flux, 2, field, prm, rule=1)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(law, flux, field, prm), 2, dgp.FP64, rule=dgp.RULE_WORKLOAD)
    try:
        s.set_fused(form == "fused")
    except dgp.DGPError as e:
        assert e.code == -3 and form == "fused"
        pytest.skip("no fused stage kernel for this solver")
    assert rel(s.get_state(), o.state()) < 1e-12
    assert rel(s.rhs(0.0), o.rhs(0.0)) < 1e-11
    t = 0.0
    for _ in range(4):
        dt = o.cfl_dt(0.1)
        assert abs(s.cfl_dt(0.1) - dt) <= 1e-13 * dt
        s.step(t, dt)
        o.step(t, dt)
        t += dt
        assert rel(s.get_state(), o.state()) < 1e-12
    # the reference rule gives a different state
    r = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(law, flux, field, prm), 2, dgp.FP64)
    assert rel(r.get_state(), o.state()) > 1e-14


@pytest.mark.gpu
def test_gpu_workload_rule_refused_where_not_built(tmp_path):
    msh = _tri(tmp_path)
    law = dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D)
    with pytest.raises(dgp.DGPError) as ei:
        dgp.Solver(dgp.Mesh.from_msh(msh), law, 3, dgp.FP64, rule=dgp.RULE_WORKLOAD)
    assert ei.value.code == -3
    with pytest.raises(dgp.DGPError) as ei:
        dgp.Solver(dgp.Mesh.from_msh(msh), law, 2, dgp.FP64, rule=7)
    assert ei.value.code == -1
