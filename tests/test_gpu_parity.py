"""GPU parity: the CUDA path through the C ABI against DG-Parallel's own output
(golden fixtures) and against the C oracle on the same seeded meshes.

Tolerances are relative (max |a - b| / max |b|):
* FP64 vs the oracle: 1e-12 on states, 1e-11 on the assembled RHS (whose
  volume and face parts cancel); the two differ only in summation order and
  FMA contraction.
* FP64 vs DG-Parallel: the per-order REF_TOL of tests/cases.py (the reference's
  truncated basis tables dominate).
* mixed (FP32) vs the oracle: 2e-5 on states after the steps taken.
"""
import os

import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import (GOLDEN_CASES, PULSE3D, REF_RHS_TOL, REF_TOL, SCALAR2D, SCALAR3D, SINE, TM110,
                   VORTEX, golden, rel)
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
RHS_TOL = 1e-11


def solver_for(msh, law, flux, field, order, prm, precision=dgp.FP64):
    mesh = dgp.Mesh.from_msh(msh)
    lw = dgp.Law(law, flux, field, prm)
    return dgp.Solver(mesh, lw, order, precision)


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_gpu_matches_reference_golden(name):
    law, flux, field, order, prm = GOLDEN_CASES[name]
    msh, g = golden(name)
    s = solver_for(msh, law, flux, field, order, prm)
    E = s.ncells
    tol = REF_TOL[order]
    assert rel(s.get_state().reshape(E, -1), g["states"][0]) < tol
    assert rel(s.rhs(0.0).reshape(E, -1), g["rhs"]) < REF_RHS_TOL[order]
    t = 0.0
    for k in range(1, int(g["steps"]) + 1):
        dt = s.cfl_dt(0.1)
        assert abs(dt - g["log"][k - 1, 1]) <= max(1e-13, tol) * dt
        resid = s.step(t, dt)
        t += dt
        assert rel(s.get_state().reshape(E, -1), g["states"][k]) < tol
        assert abs(resid - g["log"][k - 1, 3]) <= 1e-8 * g["log"][k - 1, 3]


def _tri(tmp_path, n, box=(0.0, 1.0), seed=1, tag=1):
    m = meshgen.tri_square(n, n, box[0], box[1], box[0], box[1], seed=seed, boundary_tag=tag)
    p = str(tmp_path / f"tri{n}_{seed}_{tag}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _tet(tmp_path, n, seed=3, tag=1):
    m = meshgen.tet_cube(n, seed=seed, boundary_tag=tag)
    p = str(tmp_path / f"tet{n}_{seed}_{tag}.msh")
    meshgen.write_msh_v1(m, p)
    return p


# (id, mesh kind, mesh size, law, flux, field, params, orders, boundary tag)
ORACLE_CASES = [
    ("scalar", "tri", 8, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D, [0, 1, 2, 3, 4], 1),
    ("euler_godunov", "trib", 8, dgp.LAW_EULER2D, dgp.FLUX_GODUNOV, dgp.FIELD_VORTEX, VORTEX, [1, 2, 3, 4], 1),
    ("euler_roe", "trib", 8, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX, [0, 1, 2, 3, 4], 1),
    ("euler_llf", "trib", 8, dgp.LAW_EULER2D, dgp.FLUX_LLF, dgp.FIELD_VORTEX, VORTEX, [1, 2, 3, 4], 1),
    ("euler_wall", "trib", 6, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX, [2], 40000),
    ("burgers_central", "tri", 8, dgp.LAW_BURGERS2D, dgp.FLUX_CENTRAL, dgp.FIELD_SINE, SINE, [1, 2, 3, 4], 1),
    ("burgers_llf", "tri", 8, dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, SINE, [1, 2, 3, 4], 1),
    ("scalar3d", "tet", 3, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS3D, SCALAR3D, [0, 1, 2, 3], 1),
    ("euler3d", "tet", 3, dgp.LAW_EULER3D, dgp.FLUX_GODUNOV, dgp.FIELD_PULSE3D, PULSE3D, [1, 2, 3], 1),
    ("maxwell3d_pec", "tet", 3, dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, TM110, [1, 2, 3], 40000),
    ("maxwell3d_far", "tet", 3, dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, TM110, [2], 1),
]
PARAMS = [(c[0], o) for c in ORACLE_CASES for o in c[7]]


@pytest.mark.parametrize("form", ["fused", "separate"])
@pytest.mark.parametrize("cid,order", PARAMS)
def test_gpu_matches_oracle(tmp_path, cid, order, form):
    """Both stage forms: the fused stage kernel and the separate face and
    element kernels (whichever the solver picks by default, the other by
    dgp_set_fused)."""
    case = next(c for c in ORACLE_CASES if c[0] == cid)
    _, kind, n, law, flux, field, prm, _, tag = case
    if kind == "tri":
        msh = _tri(tmp_path, n, tag=tag)
    elif kind == "trib":
        msh = _tri(tmp_path, n, box=(0.0, 10.0), seed=2, tag=tag)
    else:
        msh = _tet(tmp_path, n, tag=tag)
    o = Oracle(msh, law, flux, order, field, prm)
    s = solver_for(msh, law, flux, field, order, prm)
    try:
        s.set_fused(form == "fused")
    except dgp.DGPError as e:
        assert e.code == -3 and form == "fused"
        pytest.skip("no fused stage kernel for this solver")
    assert s.fused == (form == "fused")
    E = s.ncells
    assert rel(s.get_state(), o.state()) < FP64_TOL
    assert rel(s.rhs(0.0), o.rhs(0.0)) < RHS_TOL
    assert rel(s.rhs(0.37), o.rhs(0.37)) < RHS_TOL  # time-dependent boundary data
    t = 0.0
    for _ in range(4):
        dt_g, dt_o = s.cfl_dt(0.1), o.cfl_dt(0.1)
        assert abs(dt_g - dt_o) <= 1e-13 * dt_o
        rg = s.step(t, dt_o)
        ro = o.step(t, dt_o)
        t += dt_o
        assert rel(s.get_state(), o.state()) < FP64_TOL
        assert abs(rg - ro) <= 1e-9 * ro + 1e-300
    assert s.status()[0] == 0


def test_run_device_loop_matches_oracle(tmp_path):
    msh = _tri(tmp_path, 12, box=(0.0, 10.0), seed=2)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 3, dgp.FIELD_VORTEX, VORTEX)
    s = solver_for(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 3, VORTEX)
    assert s.fused and s.launches_per_step() == 4  # 3 stage launches + the finalize
    tg, ng = s.run(0.0, 0.05, 0.1)
    to, no = o.run(0.0, 0.05, 0.1, 0)
    assert ng == no and tg == to
    assert rel(s.get_state(), o.state()) < 1e-11
    # fixed step count, continuing from the current state and time
    tg2, ng2 = s.run(tg, 0.0, 0.1, 7)
    to2, no2 = o.run(to, 0.0, 0.1, 7)
    assert ng2 == no2 == 7 and abs(tg2 - to2) <= 1e-15 * to2
    assert rel(s.get_state(), o.state()) < 1e-11


@pytest.mark.parametrize("tensor_cores", [False, True])
def test_mixed_precision_tracks_fp64(tmp_path, tensor_cores):
    """The mixed form (FP32 right-hand side; with tensor_cores, its volume
    contraction on tcgen05 as split TF32) against the FP64 oracle."""
    msh = _tri(tmp_path, 8, box=(0.0, 10.0), seed=2)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 3, dgp.FIELD_VORTEX, VORTEX)
    s = solver_for(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 3, VORTEX, dgp.MIXED)
    s.set_tensor_cores(tensor_cores)
    assert rel(s.get_state(), o.state()) < 1e-6
    t = 0.0
    for _ in range(5):
        dt = o.cfl_dt(0.1)
        s.step(t, dt)
        o.step(t, dt)
        t += dt
    assert rel(s.get_state(), o.state()) < 2e-5


def test_rounding_probe_perturbs_at_fp32_level(tmp_path):
    """The FP64 kernel with terms rounded to FP32: no mask leaves the FP64
    result; each mask moves it by FP32 rounding, never more than the mixed form."""
    msh = _tri(tmp_path, 8, box=(0.0, 10.0), seed=2)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 3, dgp.FIELD_VORTEX, VORTEX)
    dts = []
    t = 0.0
    for _ in range(3):
        dts.append(o.cfl_dt(0.1))
        o.step(t, dts[-1])
        t += dts[-1]
    ref = o.state()
    for mask in (0, 1, 2, 4, 8, 16, 32, 64, 127):
        s = solver_for(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 3, VORTEX)
        s.set_rounding_probe(mask)
        t = 0.0
        for dt in dts:
            s.step(t, dt)
            t += dt
        err = rel(s.get_state(), ref)
        if mask == 0:
            assert err < FP64_TOL
        else:
            assert 1e-12 < err < 2e-5, (mask, err)
    u = solver_for(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 2, SCALAR2D)
    with pytest.raises(dgp.DGPError) as ei:
        u.set_rounding_probe(2)
    assert ei.value.code == -3


def test_tensor_cores_refused_where_not_built(tmp_path):
    msh = _tri(tmp_path, 4, box=(0.0, 10.0), seed=2)
    s = solver_for(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 3, VORTEX, dgp.FP64)
    with pytest.raises(dgp.DGPError) as ei:
        s.set_tensor_cores(True)
    assert ei.value.code == -3
    s.set_tensor_cores(False)


def test_state_roundtrip_and_totals(tmp_path):
    msh = _tri(tmp_path, 8, box=(0.0, 10.0), seed=2)
    s = solver_for(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX)
    c = np.random.default_rng(0).standard_normal(s.shape)
    s.set_state(c)
    assert np.array_equal(s.get_state(), c)
    s.project(0.0)
    tot0 = s.totals()
    # the projection conserves the cell integrals: total mass = integral of the
    # vortex density over [0,10]^2 (free stream 1 minus the core deficit)
    n = 2000
    x = (np.arange(n) + 0.5) * (10.0 / n)
    X, Y = np.meshgrid(x, x)
    r2 = (X - 5.0) ** 2 + (Y - 5.0) ** 2
    T = 1.0 - 0.4 * 25.0 / (8.0 * 1.4 * np.pi ** 2) * np.exp(1.0 - r2)
    mass = float((T ** 2.5).sum() * (10.0 / n) ** 2)
    assert abs(tot0[0] - mass) < 1e-4 * mass
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 2, dgp.FIELD_VORTEX, VORTEX)
    assert abs(s.l2_error(0.0, 0) - o.l2_error(0.0, 0)) <= 1e-12 * o.l2_error(0.0, 0)


def test_device_pointer_state(tmp_path):
    torch = pytest.importorskip("torch")
    msh = _tri(tmp_path, 6)
    s = solver_for(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 2, SCALAR2D)
    host = s.get_state()
    buf = torch.zeros(host.size, dtype=torch.float64, device="cuda")
    s.get_state_device(buf.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(buf.cpu().numpy().reshape(s.shape), host)
    buf2 = buf * 2.0
    s.set_state_device(buf2.data_ptr())
    assert np.array_equal(s.get_state(), 2.0 * host)


def test_unsupported_and_invalid(tmp_path):
    msh = _tri(tmp_path, 4)
    mesh = dgp.Mesh.from_msh(msh)
    with pytest.raises(dgp.DGPError) as e:
        dgp.Solver(mesh, dgp.Law(dgp.LAW_EULER3D, dgp.FLUX_GODUNOV, dgp.FIELD_PULSE3D, PULSE3D), 2)
    assert e.value.code == -3
    with pytest.raises(dgp.DGPError) as e:
        dgp.Solver(mesh, dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D), 7)
    assert e.value.code == -3


@pytest.mark.parametrize("law_id, flux, field, prm", [
    (dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX),
    (dgp.LAW_MAXWELL2D, dgp.FLUX_UPWIND, dgp.FIELD_TM2D, TM110),
])
def test_law_set_bc_equals_retagged_mesh(tmp_path, law_id, flux, field, prm):
    """dgp_law_set_bc: faces tagged 1 declared walls step exactly as the same
    mesh tagged 40000 with the default rule, and 40000 declared far field as
    the mesh tagged 1."""
    box = (0.0, 10.0) if law_id == dgp.LAW_EULER2D else (0.0, 1.0)
    far = _tri(tmp_path, 6, box=box, seed=2, tag=1)
    wall = _tri(tmp_path, 6, box=box, seed=2, tag=40000)

    def run(msh, bcs):
        law = dgp.Law(law_id, flux, field, prm)
        for bid, kind in bcs:
            law.set_bc(bid, kind)
        s = dgp.Solver(dgp.Mesh.from_msh(msh), law, 2)
        t = 0.0
        for _ in range(3):
            dt = 0.5 * s.cfl_dt(0.1) if law_id == dgp.LAW_EULER2D else 0.005
            s.step(t, dt)
            t += dt
        return s.get_state()

    a = run(far, [(1, dgp.BC_WALL)])
    b = run(wall, [])
    assert np.array_equal(a, b)
    c = run(wall, [(40000, dgp.BC_FARFIELD)])
    d = run(far, [])
    assert np.array_equal(c, d)
    assert not np.array_equal(a, d)
