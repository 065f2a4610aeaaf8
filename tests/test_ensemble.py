"""Batched ensembles: independent instances of uneven size and mixed order run
in shared kernels per (law, flux, element, order) group.

Every cell of an instance sees the same arithmetic in the same order as in a
single solver on that instance's mesh (instances start on tile boundaries, so
the tiles, face order and reductions coincide): ensemble results must equal
single-solver results exactly, and the single solver is checked against the
oracle elsewhere.
"""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import params, rel
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu

# (cells per side, seed, order, amplitude)
INSTANCES = [(6, 11, 1, 0.6), (9, 12, 2, 1.2), (5, 13, 1, 1.0), (12, 14, 3, 0.8), (8, 15, 2, 1.4),
             (7, 16, 4, 0.5), (10, 17, 1, 0.9)]


def _instances(tmp_path):
    paths, laws, orders, prms = [], [], [], []
    for n, seed, order, amp in INSTANCES:
        m = meshgen.tri_square(n, n, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=seed)
        p = str(tmp_path / f"ens_{n}_{seed}.msh")
        meshgen.write_msh_v1(m, p)
        prm = params(amplitude=amp)
        paths.append(p)
        prms.append(prm)
        laws.append(dgp.Law(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, prm))
        orders.append(order)
    return paths, laws, orders, prms


@pytest.mark.parametrize("limiter", [dgp.LIMITER_NONE, dgp.LIMITER_MOMENT])
def test_ensemble_equals_single_solvers(tmp_path, limiter):
    paths, laws, orders, prms = _instances(tmp_path)
    meshes = [dgp.Mesh.from_msh(p) for p in paths]
    ens = dgp.Ensemble(meshes, laws, orders, dgp.FP64, limiter)
    assert len(set(ens.groups)) == 4  # P1..P4
    ens.project(0.0)
    t, steps, ms, total = ens.run(0.0, 0.15, 0.1)
    assert np.allclose(t, 0.15, rtol=0, atol=1e-12)
    assert (ms > 0).all() and total >= ms.max() - 1e-9
    for i, p in enumerate(paths):
        s = dgp.Solver(dgp.Mesh.from_msh(p), laws[i], orders[i], dgp.FP64, limiter)
        s.project(0.0)
        ts, ns = s.run(0.0, 0.15, 0.1)
        assert ns == steps[i] and abs(ts - t[i]) < 1e-14
        assert rel(ens.get_state(i), s.get_state()) == 0.0
        assert np.allclose(ens.totals(i), s.totals(), rtol=1e-14, atol=0)


def test_ensemble_instance_matches_oracle(tmp_path):
    paths, laws, orders, prms = _instances(tmp_path)
    meshes = [dgp.Mesh.from_msh(p) for p in paths]
    ens = dgp.Ensemble(meshes, laws, orders, dgp.FP64, dgp.LIMITER_MOMENT)
    ens.project(0.0)
    t, steps, ms, total = ens.run(0.0, 0.1, 0.1)
    for i in (0, 3):
        o = Oracle(paths[i], dgp.LAW_BURGERS2D, dgp.FLUX_LLF, orders[i], dgp.FIELD_SINE, prms[i])
        o.set_limiter(True)
        o.limit()
        to, no = o.run(0.0, 0.1, 0.1, 0)
        assert no == steps[i]
        assert rel(ens.get_state(i), o.state()) < 1e-9


def test_ensemble_set_state_and_max_steps(tmp_path):
    paths, laws, orders, prms = _instances(tmp_path)
    meshes = [dgp.Mesh.from_msh(p) for p in paths]
    ens = dgp.Ensemble(meshes, laws, orders, dgp.FP64)
    c0 = [ens.get_state(i) for i in range(ens.n)]
    for i in range(ens.n):
        ens.set_state(i, c0[i] * 0.5)
        assert np.array_equal(ens.get_state(i), c0[i] * 0.5)
    t, steps, ms, total = ens.run(0.0, 0.0, 0.1, max_steps=5)
    assert (steps == 5).all()
    assert np.isfinite(ens.get_state(2)).all()


def test_ensemble_mixed_form(tmp_path):
    paths, laws, orders, prms = _instances(tmp_path)
    meshes = [dgp.Mesh.from_msh(p) for p in paths]
    e64 = dgp.Ensemble(meshes, laws, orders, dgp.FP64, dgp.LIMITER_MOMENT)
    e32 = dgp.Ensemble(meshes, laws, orders, dgp.MIXED, dgp.LIMITER_MOMENT)
    for e in (e64, e32):
        e.project(0.0)
        e.run(0.0, 0.05, 0.1)
    for i in range(e64.n):
        assert rel(e32.get_state(i), e64.get_state(i)) < 1e-3
        tot64, tot32 = e64.totals(i), e32.totals(i)
        assert abs(tot32[0] - tot64[0]) < 1e-4 * max(1.0, abs(tot64[0]))


def test_autotune_picks_a_built_shape(tmp_path):
    m = meshgen.tri_square(24, 24, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)
    p = str(tmp_path / "vortex24.msh")
    meshgen.write_msh_v1(m, p)
    from cases import VORTEX
    mesh = dgp.Mesh.from_msh(p)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX)
    best, ms = dgp.autotune(mesh, law, 3, dgp.FP64, 0, iters=3)
    assert best in (64, 128, 256) and all(x > 0 for x in ms)
    s = dgp.Solver(mesh, law, 3)
    assert s.block()[0] == best


@pytest.mark.parametrize("order", [1, 4])
def test_tile_shapes_give_identical_states(tmp_path, order):
    # every cell sees the same arithmetic whatever the tile: states agree exactly
    m = meshgen.tri_square(20, 20, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=3)
    p = str(tmp_path / "b20.msh")
    meshgen.write_msh_v1(m, p)
    law = dgp.Law(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, params(amplitude=1.0))
    out = {}
    for block in (64, 128, 256):
        dgp.tune_set(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, 2, order, dgp.FP64, 800, block)
        s = dgp.Solver(dgp.Mesh.from_msh(p), law, order, dgp.FP64, dgp.LIMITER_MOMENT)
        assert s.block()[0] == block
        s.project(0.0)
        s.run(0.0, 0.12, 0.1)
        out[block] = s.get_state()
    dgp.tune_set(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, 2, order, dgp.FP64, 800, 128)
    assert np.array_equal(out[64], out[128]) and np.array_equal(out[256], out[128])


def test_autotune_ensemble_groups(tmp_path):
    paths, laws, orders, prms = _instances(tmp_path)
    meshes = [dgp.Mesh.from_msh(p) for p in paths]
    dgp.autotune_ensemble(meshes, laws, orders, dgp.FP64, dgp.LIMITER_MOMENT, iters=2)
    ens = dgp.Ensemble(meshes, laws, orders, dgp.FP64, dgp.LIMITER_MOMENT)
    for g in set(ens.groups):
        assert ens.group_block(g)[0] in (64, 128, 256)


def test_ensemble_fused_form_equals_single_solvers(tmp_path):
    """Euler (Roe) instances at P1-P3, which run the fused stage kernel by
    default: the ensemble instantiation of that kernel (per-instance time
    controls, the finalize per instance) takes the single solvers' steps to the
    same times and gives their states to the last rounding (the two
    instantiations are compiled separately and may contract a multiply-add
    differently)."""
    from cases import VORTEX
    specs = [(6, 21, 1), (9, 22, 2), (7, 23, 3), (8, 24, 2), (5, 25, 3)]
    paths, laws, orders = [], [], []
    for n, seed, order in specs:
        m = meshgen.tri_square(n, n, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=seed)
        p = str(tmp_path / f"ensv_{n}_{seed}.msh")
        meshgen.write_msh_v1(m, p)
        paths.append(p)
        laws.append(dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX))
        orders.append(order)
    meshes = [dgp.Mesh.from_msh(p) for p in paths]
    ens = dgp.Ensemble(meshes, laws, orders, dgp.FP64, dgp.LIMITER_NONE)
    ens.project(0.0)
    t, steps, ms, total = ens.run(0.0, 0.05, 0.1)
    for i, p in enumerate(paths):
        s = dgp.Solver(dgp.Mesh.from_msh(p), laws[i], orders[i], dgp.FP64)
        assert s.fused
        s.project(0.0)
        ts, ns = s.run(0.0, 0.05, 0.1)
        assert ns == steps[i] and abs(ts - t[i]) < 1e-14
        assert rel(ens.get_state(i), s.get_state()) < 1e-15
