"""Local time stepping (DGAnalysis mode 5): the size bins of
DGAnalysis::sortCellsBySize and RungeKuttaTVD2adaptive::advanceInTime.

The fixtures (tests/golden/lts_*.npz, written by make_golden.py) come from the
reference's own integrator and binning code run by oracle/_ref/ref_driver_lts,
with the integrator's two range helpers (TimeIntegrator::assembleVolume /
assembleBoundary(begin, end, t), shipped with empty bodies) given the bodies of
their whole-mesh versions.  Bars: bins and roles bit-exact; states against the
reference within the per-order REF_TOL; CUDA FP64 against the C restatement
1e-12 (summation order and contraction in the assembly differ, the
coefficient updates round alike); the mode-5 step 1e-13.
"""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import REF_TOL, SCALAR2D, SCALAR3D, VORTEX, golden, rel
from oracle_bind import Oracle

LTS_CASES = {
    "lts_scalar_graded_p2": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 2, SCALAR2D),
    "lts_euler_roe_graded_p2": (dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX),
    "lts_scalar_tet_graded_p2": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS3D, 2, SCALAR3D),
}
ORACLE_IDS = {dgp.LAW_SCALAR: 0, dgp.LAW_EULER2D: 2}
FP64_TOL = 1e-12


def _oracle(msh, law, flux, field, order, prm):
    return Oracle(msh, ORACLE_IDS[law], flux, order, field, prm)


@pytest.mark.parametrize("name", sorted(LTS_CASES))
def test_oracle_matches_reference_lts(name):
    law, flux, field, order, prm = LTS_CASES[name]
    msh, g = golden(name)
    o = _oracle(msh, law, flux, field, order, prm)
    assert o.lts_setup() == int(g["nbins"])
    b, r = o.lts_bins()
    assert np.array_equal(b, g["bins"][:, 0]) and np.array_equal(r, g["bins"][:, 1])
    # every role occurs: the interface paths of the integrator are exercised
    assert set(r.tolist()) == {0, 1, 2} and len(set(b.tolist())) == int(g["nbins"])
    E = o.ncells
    assert rel(o.state().reshape(E, -1), g["states"][0]) < REF_TOL[order]
    t = 0.0
    for k in range(1, int(g["steps"]) + 1):
        dt = o.lts_dt(0.1)
        assert abs(dt - g["log"][k - 1, 1]) <= 1e-13 * dt
        assert o.lts_step(t, dt) == 0.0
        t += dt
        assert rel(o.state().reshape(E, -1), g["states"][k]) < REF_TOL[order]
    assert np.abs(g["states"][-1] - g["states"][0]).max() > 1e-3  # the state moved


def test_oracle_lts_rejects_meshes_the_reference_rejects(tmp_path):
    # equal cell sizes: no bin (the reference stops with "cells were lost")
    m = meshgen.tri_square(4, 4, jitter=0.0)
    p = str(tmp_path / "u.msh")
    meshgen.write_msh_v1(m, p)
    assert _oracle(p, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 1, SCALAR2D).lts_setup() == -1
    # the smallest cell just above max / 2^bins but below it times 1.0001:
    # in no bin; a steeper grading: neighbours more than one bin apart
    for (n, ratio), code in (((8, 2.0), -3), ((6, 3.0), -5)):
        m = meshgen.tri_graded(n, n, ratio=ratio)
        p = str(tmp_path / f"s{n}.msh")
        meshgen.write_msh_v1(m, p)
        assert _oracle(p, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 1, SCALAR2D).lts_setup() == code


def _solver(msh, law, flux, field, order, prm, precision=dgp.FP64, limiter=dgp.LIMITER_NONE, p0=False):
    """Local time stepping runs without the P0 fallback (on by default for the
    Euler laws): p0=False turns it off, as a caller must before enabling it."""
    mesh = dgp.Mesh.from_msh(msh)
    s = dgp.Solver(mesh, dgp.Law(law, flux, field, prm), order, precision, limiter)
    if not p0:
        s.set_p0_fallback(False)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(LTS_CASES))
def test_gpu_lts_matches_reference_and_oracle(name):
    law, flux, field, order, prm = LTS_CASES[name]
    msh, g = golden(name)
    s = _solver(msh, law, flux, field, order, prm)
    o = _oracle(msh, law, flux, field, order, prm)
    nb = s.set_time_stepping(dgp.STEPPING_LOCAL)
    assert nb == int(g["nbins"]) == o.lts_setup()
    b, r = s.lts_bins()
    assert np.array_equal(b, g["bins"][:, 0]) and np.array_equal(r, g["bins"][:, 1])
    E = s.ncells
    assert s.launches_per_step() > 0
    t = 0.0
    for k in range(1, int(g["steps"]) + 1):
        dt = s.cfl_dt(0.1)
        assert abs(dt - g["log"][k - 1, 1]) <= 1e-13 * dt
        assert abs(dt - o.lts_dt(0.1)) <= 1e-13 * dt
        assert s.step(t, dt) == 0.0
        o.lts_step(t, dt)
        t += dt
        assert rel(s.get_state().reshape(E, -1), g["states"][k]) < REF_TOL[order]
        assert rel(s.get_state(), o.state()) < FP64_TOL
    assert s.status()[0] == 0


@pytest.mark.gpu
def test_gpu_lts_run_device_loop_matches_oracle():
    """dgp_run with local time stepping: the mode-5 step computed on the
    device every step, stretched to land on tend, in CUDA graphs."""
    law, flux, field, order, prm = LTS_CASES["lts_scalar_graded_p2"]
    msh, _ = golden("lts_scalar_graded_p2")
    s = _solver(msh, law, flux, field, order, prm)
    o = _oracle(msh, law, flux, field, order, prm)
    s.set_time_stepping(dgp.STEPPING_LOCAL)
    o.lts_setup()
    # step limit (one 8-step graph + one-step graphs)
    t_g, n_g = s.run(0.0, 0.0, 0.1, 11)
    t_o = 0.0
    for _ in range(11):
        dt = o.lts_dt(0.1)
        o.lts_step(t_o, dt)
        t_o += dt
    assert n_g == 11 and abs(t_g - t_o) <= 1e-13 * t_o
    assert rel(s.get_state(), o.state()) < FP64_TOL
    # end time: N = ceil((tend - t) / dt), dt = (tend - t) / N each step
    tend = t_o + 0.01
    t_g, n_g = s.run(t_g, tend, 0.1, 0)
    n_o = 0
    while t_o < tend:
        dt = o.lts_dt(0.1)
        n = int(np.ceil((tend - t_o) / dt))
        dt = (tend - t_o) / n
        o.lts_step(t_o, dt)
        t_o += dt
        n_o += 1
    assert n_g == n_o and abs(t_g - t_o) <= 1e-13 * t_o
    assert rel(s.get_state(), o.state()) < FP64_TOL


@pytest.mark.gpu
def test_gpu_lts_modes_and_errors(tmp_path):
    law, flux, field, order, prm = LTS_CASES["lts_scalar_graded_p2"]
    msh, _ = golden("lts_scalar_graded_p2")
    # back to SSP-RK3: the same steps as a solver that never switched
    s = _solver(msh, law, flux, field, order, prm)
    ref = _solver(msh, law, flux, field, order, prm)
    assert s.set_time_stepping(dgp.STEPPING_LOCAL) == 4
    assert s.set_time_stepping(dgp.STEPPING_SSPRK3) == 0
    dt = ref.cfl_dt(0.1)
    assert s.cfl_dt(0.1) == dt
    s.step(0.0, dt)
    ref.step(0.0, dt)
    assert np.array_equal(s.get_state(), ref.get_state())
    # meshes the reference rejects, and configurations not built
    m = meshgen.tri_square(4, 4, jitter=0.0)
    p = str(tmp_path / "u.msh")
    meshgen.write_msh_v1(m, p)
    u = _solver(p, law, flux, field, 1, prm)
    with pytest.raises(dgp.DGPError) as ei:
        u.set_time_stepping(dgp.STEPPING_LOCAL)
    assert ei.value.code == -1
    with pytest.raises(dgp.DGPError) as ei:
        _solver(msh, law, flux, field, order, prm, precision=dgp.MIXED).set_time_stepping(dgp.STEPPING_LOCAL)
    assert ei.value.code == -3
    with pytest.raises(dgp.DGPError) as ei:
        _solver(msh, law, flux, field, order, prm,
                limiter=dgp.LIMITER_BARTH).set_time_stepping(dgp.STEPPING_LOCAL)
    assert ei.value.code == -3
    with pytest.raises(dgp.DGPError):
        s.set_time_stepping(7)
    # the P0 fallback (on by default for the Euler laws) and local time
    # stepping exclude each other, whichever is asked for second
    law_e, flux_e, field_e, order_e, prm_e = LTS_CASES["lts_euler_roe_graded_p2"]
    msh_e, _ = golden("lts_euler_roe_graded_p2")
    e = _solver(msh_e, law_e, flux_e, field_e, order_e, prm_e, p0=True)
    with pytest.raises(dgp.DGPError) as ei:
        e.set_time_stepping(dgp.STEPPING_LOCAL)
    assert ei.value.code == -3 and "P0" in str(ei.value)
    e.set_p0_fallback(False)
    assert e.set_time_stepping(dgp.STEPPING_LOCAL) == 3
    with pytest.raises(dgp.DGPError) as ei:
        e.set_p0_fallback(True)
    assert ei.value.code == -3
    e.set_time_stepping(dgp.STEPPING_SSPRK3)
    e.set_p0_fallback(True)
