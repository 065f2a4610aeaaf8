"""Edge cases: meshes of one or two cells (every face a boundary face, tiles
almost empty), limiters on them, probes on shared vertices, and CPU-side
checks of the small-mesh oracle runs."""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import SCALAR2D, SCALAR3D, SINE, params, rel
from oracle_bind import Oracle

WIDE = params(velocity=(1.0, 0.5, 0.0), center=(0.3, 0.3, 0.0), width=0.1)


def _one_triangle(tmp_path):
    m = meshgen.Mesh(2, np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.2, 0.9, 0.0]]),
                     np.array([[0, 1, 2]]), np.array([[0, 1], [1, 2], [2, 0]]), np.array([1, 1, 1]))
    p = str(tmp_path / "one_tri.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _two_triangles(tmp_path):
    m = meshgen.Mesh(2, np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0], [0.0, 1.0, 0.0]]),
                     np.array([[0, 1, 2], [0, 2, 3]]), np.array([[0, 1], [1, 2], [2, 3], [3, 0]]),
                     np.array([1, 1, 1, 1]))
    p = str(tmp_path / "two_tri.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _one_tet(tmp_path):
    m = meshgen.Mesh(3, np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.1, 0.2, 1.0]]),
                     np.array([[0, 1, 2, 3]]), np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]),
                     np.array([1, 1, 1, 1]))
    p = str(tmp_path / "one_tet.msh")
    meshgen.write_msh_v1(m, p)
    return p


def test_oracle_runs_on_single_cells(tmp_path):
    for msh, field, prm in ((_one_triangle(tmp_path), dgp.FIELD_GAUSS, WIDE),
                            (_one_tet(tmp_path), dgp.FIELD_GAUSS3D, SCALAR3D)):
        o = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, field, prm)
        t, n = o.run(0.0, 0.0, 0.1, 5)
        assert n == 5 and np.isfinite(o.state()).all()
        o.close()


def test_oracle_limiters_leave_isolated_cells_alone(tmp_path):
    # no interior neighbour: neither limiter has anything to compare with
    msh = _one_triangle(tmp_path)
    for kind in (1, 2):
        o = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, dgp.FIELD_GAUSS, SCALAR2D)
        before = o.state()
        o.set_limiter(kind)
        trig = o.limit()
        assert not trig.any() and np.array_equal(o.state(), before)
        o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["tri", "tet"])
@pytest.mark.parametrize("prec", [dgp.FP64, dgp.MIXED])
def test_gpu_single_cell_matches_oracle(tmp_path, which, prec):
    msh, field, prm = ((_one_triangle(tmp_path), dgp.FIELD_GAUSS, WIDE) if which == "tri"
                       else (_one_tet(tmp_path), dgp.FIELD_GAUSS3D, SCALAR3D))
    o = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, field, prm)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, field, prm), 2, prec)
    assert s.ncells == 1
    tg, ng = s.run(0.0, 0.0, 0.1, 5)
    to, no = o.run(0.0, 0.0, 0.1, 5)
    assert ng == no == 5 and abs(tg - to) <= 1e-14 * to
    assert rel(s.get_state(), o.state()) < (1e-12 if prec == dgp.FP64 else 1e-5)
    s.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("limiter", [dgp.LIMITER_MOMENT, dgp.LIMITER_BARTH])
def test_gpu_limiters_on_two_cells_match_oracle(tmp_path, limiter):
    msh = _two_triangles(tmp_path)
    prm = params(amplitude=1.0)
    o = Oracle(msh, dgp.LAW_BURGERS2D, dgp.FLUX_LLF, 3, dgp.FIELD_SINE, prm)
    o.set_limiter(1 if limiter == dgp.LIMITER_MOMENT else 2)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, prm), 3,
                   dgp.FP64, limiter)
    s.set_state(o.state())
    assert np.array_equal(s.limit(), o.limit())
    assert rel(s.get_state(), o.state()) < 1e-14
    dt = 0.5 * o.cfl_dt(0.1)
    for k in range(4):
        o.step(k * dt, dt)
        s.step(k * dt, dt)
    assert rel(s.get_state(), o.state()) < 1e-12
    s.close()
    o.close()


@pytest.mark.gpu
def test_gpu_probe_on_a_shared_vertex_takes_the_lowest_cell(tmp_path):
    msh = _two_triangles(tmp_path)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, WIDE), 2,
                   dgp.FP64)
    # vertex 0 and the diagonal midpoint belong to both cells; cell 0 wins
    pr = dgp.Probe(s, np.array([[0.0, 0.0], [0.5, 0.5], [0.8, 0.1], [0.1, 0.8]]))
    assert pr.found.all()
    v = pr.eval()
    c = s.get_state()
    assert np.isfinite(v).all()
    # the two cells' polynomials differ at the shared points: the value is cell 0's
    s.set_state(np.concatenate([c[:1], np.zeros_like(c[1:])]))
    v0 = pr.eval()
    assert v0[0, 0] == v[0, 0] and v0[1, 0] == v[1, 0] and v0[3, 0] == 0.0
    pr.close()
    s.close()
