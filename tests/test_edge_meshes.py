"""Edge-case meshes through both stage forms against the oracle: a single
cell (every face on the boundary, one partial tile), two cells, and cell
counts that leave the last tile ragged (70 triangles against 32-cell tiles,
162 tets against 14- and 21-cell tiles)."""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import SCALAR2D, TM110, VORTEX, rel
from oracle_bind import Oracle


def _single_triangle(tmp_path, box=1.0, tag=1):
    m = meshgen.Mesh(dim=2, vertices=np.array([[0.1, 0.2, 0.0], [0.9, 0.15, 0.0], [0.4, 0.95, 0.0]]) * box,
                     cells=np.array([[0, 1, 2]]), bfaces=np.array([[0, 1], [1, 2], [2, 0]]),
                     btags=np.array([tag, tag, tag]))
    p = str(tmp_path / f"one{box:g}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _tri(tmp_path, nx, ny, box=1.0, seed=1):
    m = meshgen.tri_square(nx, ny, 0.0, box, 0.0, box, jitter=0.15, seed=seed)
    p = str(tmp_path / f"tri{nx}x{ny}_{box:g}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _tet(tmp_path, n, tag):
    m = meshgen.tet_cube(n, seed=3, boundary_tag=tag)
    p = str(tmp_path / f"tet{n}_{tag}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def test_edge_meshes_load_in_the_oracle(tmp_path):
    for msh, n in ((_single_triangle(tmp_path), 1), (_tri(tmp_path, 1, 1), 2), (_tri(tmp_path, 7, 5), 70)):
        o = Oracle(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, dgp.FIELD_GAUSS, SCALAR2D)
        assert o.ncells == n


CASES = [
    ("one_scalar_p2", "one", 1.0, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D, 2, 1),
    ("one_euler_p3", "one", 10.0, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX, 3, 1),
    ("two_euler_p2", "two", 10.0, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX, 2, 1),
    ("ragged_euler_p3", "7x5", 10.0, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX, 3, 1),
    ("ragged_scalar_p4", "7x5", 1.0, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D, 4, 1),
    ("ragged_maxwell_p2", "tet", 1.0, dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, TM110, 2, 40000),
    ("ragged_maxwell_p1", "tet", 1.0, dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, TM110, 1, 40000),
]


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fused", "separate"])
@pytest.mark.parametrize("cid,kind,box,law,flux,field,prm,order,tag", CASES)
def test_gpu_edge_mesh_matches_oracle(tmp_path, cid, kind, box, law, flux, field, prm, order, tag, form):
    if kind == "one":
        msh = _single_triangle(tmp_path, box)
    elif kind == "two":
        msh = _tri(tmp_path, 1, 1, box)
    elif kind == "7x5":
        msh = _tri(tmp_path, 7, 5, box, seed=2)
    else:
        msh = _tet(tmp_path, 3, tag)
    o = Oracle(msh, law, flux, order, field, prm)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(law, flux, field, prm), order, dgp.FP64)
    try:
        s.set_fused(form == "fused")
    except dgp.DGPError as e:
        assert e.code == -3 and form == "fused"
        pytest.skip("no fused stage kernel for this solver")
    assert rel(s.get_state(), o.state()) < 1e-12
    assert rel(s.rhs(0.2), o.rhs(0.2)) < 1e-11
    t = 0.0
    for _ in range(3):
        dt = o.cfl_dt(0.1)
        assert abs(s.cfl_dt(0.1) - dt) <= 1e-13 * dt
        rg = s.step(t, dt)
        ro = o.step(t, dt)
        t += dt
        assert rel(s.get_state(), o.state()) < 1e-12
        assert abs(rg - ro) <= 1e-9 * ro + 1e-300
    # the device loop from the same state
    s.set_state(o.state())
    tg, ng = s.run(t, 0.0, 0.1, 5)
    to, no = o.run(t, 0.0, 0.1, 5)
    assert ng == no == 5 and abs(tg - to) <= 1e-14 * to
    assert rel(s.get_state(), o.state()) < 1e-11


@pytest.mark.gpu
def test_gpu_switching_stage_forms_mid_run_matches_oracle(tmp_path):
    """Steps alternating between the fused and the separate stage form (with a
    state set from the host in between) give the oracle's states: the switch
    refreshes the face-point traces that only the separate form reads."""
    msh = _tri(tmp_path, 9, 7, 10.0, seed=2)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 3, dgp.FIELD_VORTEX, VORTEX)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX), 3,
                   dgp.FP64)
    assert s.fused
    t = 0.0
    for k, form in enumerate((True, True, False, False, True, False)):
        s.set_fused(form)
        if k == 3:
            s.set_state(o.state())  # set while separate
        if k == 4:
            s.set_state(o.state())  # set while fused, stepped fused
        dt = o.cfl_dt(0.1)
        s.step(t, dt)
        o.step(t, dt)
        t += dt
        assert rel(s.get_state(), o.state()) < 1e-12, k
    # a state set in the fused form, then the switch before the first step
    s.set_fused(True)
    s.set_state(o.state())
    s.set_fused(False)
    dt = o.cfl_dt(0.1)
    s.step(t, dt)
    o.step(t, dt)
    assert rel(s.get_state(), o.state()) < 1e-12
