"""The P0 fallback pinned against DG-Parallel itself.

Fixtures (tests/golden/p0_*.npz, made by make_golden.py through
oracle/_ref/ref_driver --p0-rhs): the projected vortex with a few cells'
density pushed away from its mean, then one assembly as the reference's serial
path does it (DGAnalysis.cc:392-417): every cell's volume term, which zeroes
the modes k >= 1 of a cell with a non-physical value at a volume quadrature
point (DGCell::computeVolumeContribution, DGCell.cc:197-221), then every face,
collecting the cells with a non-physical trace, then DGCell::setToZero on each
(DGCell.cc:785-811).  The cases reach the volume correction alone, the face
pass alone (an adjacent pair of cells among them), and both.

The reference reverses and re-adds contributions where the library zeroes the
marked cells first and assembles once, so the right-hand sides agree to
rounding (REF_RHS_TOL), and the dropped cells exactly.
"""
import numpy as np
import pytest

import dgp
from cases import REF_RHS_TOL, VORTEX, golden, rel
from oracle_bind import Oracle

P0_CASES = ["p0_euler_roe_p2_volume", "p0_euler_roe_p1_faces", "p0_euler_roe_p1_both", "p0_euler_roe_p3_both"]


def _order(g):
    args = list(g["args"])
    return int(args[args.index("--order") + 1])


@pytest.mark.parametrize("name", P0_CASES)
def test_oracle_p0_matches_reference(name):
    msh, g = golden(name)
    order = _order(g)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, order, dgp.FIELD_VORTEX, VORTEX)
    o.set_p0_fallback(True)
    o.set_state(g["state"])
    r, n = o.rhs_p0(0.0)
    assert n == len(g["dropped"])
    assert list(np.nonzero(o.bad_cells())[0]) == list(g["dropped"])
    assert np.array_equal(o.state(), g["after"])  # zeroed modes, the rest untouched
    assert rel(r, g["rhs"]) < REF_RHS_TOL[order]


def test_fixtures_cover_both_triggers():
    faces = [len(golden(n)[1]["zeroed_by_faces"]) for n in P0_CASES]
    vol = [len(set(golden(n)[1]["dropped"]) - set(golden(n)[1]["zeroed_by_faces"])) for n in P0_CASES]
    assert faces[0] == 0 and vol[0] > 0  # volume correction alone
    assert faces[1] > 0 and vol[1] == 0  # face pass alone
    assert faces[2] > 0 and vol[2] > 0 and faces[3] > 0 and vol[3] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", P0_CASES)
def test_gpu_p0_matches_reference(name):
    msh, g = golden(name)
    order = _order(g)
    mesh = dgp.Mesh.from_msh(msh)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX)
    s = dgp.Solver(mesh, law, order, dgp.FP64)
    s.set_state(g["state"])
    r = s.rhs(0.0)
    assert rel(r, g["rhs"]) < REF_RHS_TOL[order]
    assert s.status()[0] > 0  # the non-physical points are counted
    # with the fallback off the same assembly differs
    s.set_p0_fallback(False)
    s.set_state(g["state"])
    assert not rel(s.rhs(0.0), g["rhs"]) < REF_RHS_TOL[order]


@pytest.mark.gpu
@pytest.mark.parametrize("name", P0_CASES)
def test_gpu_p0_step_matches_oracle(name):
    """One SSP-RK3 step from the perturbed state: the dropped cells persist
    into u_n, later stages drop again what they find."""
    msh, g = golden(name)
    order = _order(g)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, order, dgp.FIELD_VORTEX, VORTEX)
    o.set_p0_fallback(True)
    o.set_state(g["state"])
    mesh = dgp.Mesh.from_msh(msh)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX)
    s = dgp.Solver(mesh, law, order, dgp.FP64)
    s.set_state(g["state"])
    dt = o.cfl_dt(0.1)
    for k in range(2):
        o.step(k * dt, dt)
        s.step(k * dt, dt)
    assert rel(s.get_state(), o.state()) < 1e-12
