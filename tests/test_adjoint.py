"""Discrete adjoint: the gradient of a receiver objective through SSP-RK3
steps of fixed size, checked against central finite differences of the same
forward map (FP64), and the mixed form against the FP64 gradient.

J = sum_r (rho(x_r, T) - rho_obs_r)^2, rho_obs from a forward run with a
different vortex strength (or amplitude, or width).  The forward map is the
device operator with a fixed dt, so finite differences see exactly the
function the adjoint differentiates.
"""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import PULSE3D, SCALAR2D, TM110, VORTEX, params, rel

pytestmark = pytest.mark.gpu


def _mesh(tmp_path, n, box, seed, dim=2):
    if dim == 2:
        m = meshgen.tri_square(n, n, box[0], box[1], box[0], box[1], jitter=0.15, seed=seed)
    else:
        m = meshgen.tet_cube(n, box[0], box[1], jitter=0.1, seed=seed)
    p = str(tmp_path / f"adj{dim}_{n}_{seed}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _receivers(rng, n, lo, hi, dim=2):
    return rng.uniform(lo, hi, size=(n, dim))


def _setup(msh, law_id, flux, field, order, prm, prm_obs, pts, nsteps, every, precision=dgp.FP64):
    mesh = dgp.Mesh.from_msh(msh)
    # observations: forward run with the perturbed parameters
    so = dgp.Solver(mesh, dgp.Law(law_id, flux, field, prm_obs), order, dgp.FP64)
    so.project(0.0)
    s = dgp.Solver(mesh, dgp.Law(law_id, flux, field, prm), order, precision)
    s.project(0.0)
    dt = 0.5 * s.cfl_dt(0.1)
    so.set_receivers(pts, np.zeros(len(pts)))
    so.forward_checkpointed(0.0, dt, nsteps, every)
    obs, _ = so.receiver_values()
    s.set_receivers(pts, obs)
    return s, dt


def _fd_check(s, dt, nsteps, every, ndir, eps, tol, seed=5):
    u0 = s.get_state()
    J0 = s.forward_checkpointed(0.0, dt, nsteps, every)
    g = s.backward()
    assert J0 > 0 and np.isfinite(g).all() and np.abs(g).max() > 0
    rng = np.random.default_rng(seed)
    for _ in range(ndir):
        d = rng.standard_normal(u0.shape)
        s.set_state(u0 + eps * d)
        jp = s.forward_checkpointed(0.0, dt, nsteps, every)
        s.set_state(u0 - eps * d)
        jm = s.forward_checkpointed(0.0, dt, nsteps, every)
        fd = (jp - jm) / (2 * eps)
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= tol * max(abs(fd), abs(ad)), (fd, ad)
    s.set_state(u0)
    return g


def test_adjoint_euler_roe_matches_fd(tmp_path):
    msh = _mesh(tmp_path, 12, (0.0, 10.0), 2)
    pts = _receivers(np.random.default_rng(4), 64, 1.0, 9.0)
    obs_prm = VORTEX.copy()
    obs_prm[8] = 5.5
    s, dt = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX, obs_prm, pts, 24, 5)
    _fd_check(s, dt, 24, 5, 4, 1e-6, 1e-6)


def test_adjoint_euler_llf_matches_fd(tmp_path):
    msh = _mesh(tmp_path, 10, (0.0, 10.0), 3)
    pts = _receivers(np.random.default_rng(7), 32, 1.0, 9.0)
    obs_prm = VORTEX.copy()
    obs_prm[8] = 5.5
    s, dt = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_LLF, dgp.FIELD_VORTEX, 3, VORTEX, obs_prm, pts, 12, 4)
    _fd_check(s, dt, 12, 4, 3, 1e-6, 1e-5)


def test_adjoint_scalar_is_exact_for_linear_operator(tmp_path):
    msh = _mesh(tmp_path, 10, (0.0, 1.0), 1)
    pts = _receivers(np.random.default_rng(8), 16, 0.1, 0.9)
    obs_prm = SCALAR2D.copy()
    obs_prm[6] = 0.02
    s, dt = _setup(msh, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 2, SCALAR2D, obs_prm, pts, 20, 7)
    # J is quadratic in u0: central differences are exact up to rounding
    _fd_check(s, dt, 20, 7, 3, 1e-3, 1e-8)


def test_adjoint_burgers_llf_matches_fd(tmp_path):
    msh = _mesh(tmp_path, 10, (0.0, 1.0), 9)
    pts = _receivers(np.random.default_rng(9), 16, 0.1, 0.9)
    s, dt = _setup(msh, dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, 2, params(amplitude=0.3),
                   params(amplitude=0.35), pts, 15, 4)
    _fd_check(s, dt, 15, 4, 3, 1e-7, 1e-5)


def test_adjoint_maxwell_tets_matches_fd(tmp_path):
    msh = _mesh(tmp_path, 3, (0.0, 1.0), 3, dim=3)
    pts = _receivers(np.random.default_rng(10), 12, 0.15, 0.85, dim=3)
    obs_prm = TM110.copy()
    obs_prm[10] = 1.1
    s, dt = _setup(msh, dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, 1, TM110, obs_prm, pts, 10, 3)
    _fd_check(s, dt, 10, 3, 2, 1e-3, 1e-8)


def test_adjoint_seed_and_checkpoint_interval_invariance(tmp_path):
    msh = _mesh(tmp_path, 8, (0.0, 10.0), 2)
    pts = _receivers(np.random.default_rng(4), 16, 1.0, 9.0)
    obs_prm = VORTEX.copy()
    obs_prm[8] = 5.5
    s, dt = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX, obs_prm, pts, 12, 4)
    u0 = s.get_state()
    s.forward_checkpointed(0.0, dt, 12, 4)
    g4 = s.backward()
    s.set_state(u0)
    s.forward_checkpointed(0.0, dt, 12, 12)
    g12 = s.backward()
    # recomputation reproduces the forward states exactly
    assert np.array_equal(g4, g12)
    # every == 0 keeps all stage states instead of recomputing: same gradient
    s.set_state(u0)
    s.forward_checkpointed(0.0, dt, 12, 12)
    uT = s.get_state()
    s.set_state(u0)
    s.forward_checkpointed(0.0, dt, 12, 0)
    assert np.array_equal(s.get_state(), uT)
    g0 = s.backward()
    assert np.array_equal(g0, g4)
    assert np.array_equal(s.get_state(), uT)
    # an explicit seed: d/du0 of <c, u_T> for a fixed c
    s.set_state(u0)
    s.forward_checkpointed(0.0, dt, 12, 3)
    c = np.random.default_rng(3).standard_normal(u0.shape)
    gc = s.backward(c)
    d = np.random.default_rng(4).standard_normal(u0.shape)
    eps = 1e-6
    s.set_state(u0 + eps * d)
    s.forward_checkpointed(0.0, dt, 12, 3)
    up = s.get_state()
    s.set_state(u0 - eps * d)
    s.forward_checkpointed(0.0, dt, 12, 3)
    um = s.get_state()
    fd = float(np.sum(c * (up - um))) / (2 * eps)
    assert abs(fd - float(np.sum(gc * d))) <= 1e-6 * abs(fd)


def test_adjoint_mixed_form_close_to_fp64(tmp_path):
    msh = _mesh(tmp_path, 12, (0.0, 10.0), 2)
    pts = _receivers(np.random.default_rng(4), 64, 1.0, 9.0)
    obs_prm = VORTEX.copy()
    obs_prm[8] = 5.5
    s64, dt = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX, obs_prm, pts, 20, 5)
    s32, _ = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX, obs_prm, pts, 20, 5,
                    precision=dgp.MIXED)
    s64.forward_checkpointed(0.0, dt, 20, 5)
    s32.forward_checkpointed(0.0, dt, 20, 5)
    g64, g32 = s64.backward(), s32.backward()
    assert rel(g32, g64) < 1e-3


def test_adjoint_refused_where_not_built(tmp_path):
    """Periodic edges: the partner's cotangent would leave the slot layout."""
    m = meshgen.tri_square(5, 4, -1.0, 1.0, -1.0, 1.0, jitter=0.15, seed=7, side_tags=(610, 510, 610, 510))
    p = str(tmp_path / "periodic.msh")
    meshgen.write_msh_v1(m, p)
    s = dgp.Solver(dgp.Mesh.from_msh(p), dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D), 2)
    with pytest.raises(dgp.DGPError) as ei:
        s.forward_checkpointed(0.0, 1e-3, 2, 1)
    assert ei.value.code == -3


def test_adjoint_euler_exact_godunov_matches_fd(tmp_path):
    """The exact Riemann solver differentiated through its Newton iteration."""
    msh = _mesh(tmp_path, 12, (0.0, 10.0), 2)
    pts = _receivers(np.random.default_rng(4), 64, 1.0, 9.0)
    obs_prm = VORTEX.copy()
    obs_prm[8] = 5.5
    s, dt = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_GODUNOV, dgp.FIELD_VORTEX, 2, VORTEX, obs_prm, pts, 16, 5)
    _fd_check(s, dt, 16, 5, 4, 1e-6, 1e-6)


def test_adjoint_euler3d_exact_godunov_matches_fd(tmp_path):
    msh = _mesh(tmp_path, 3, (0.0, 1.0), 3, dim=3)
    pts = _receivers(np.random.default_rng(4), 16, 0.2, 0.8, dim=3)
    obs_prm = PULSE3D.copy()
    obs_prm[6] = 0.06
    s, dt = _setup(msh, dgp.LAW_EULER3D, dgp.FLUX_GODUNOV, dgp.FIELD_PULSE3D, 1, PULSE3D, obs_prm, pts, 8, 3)
    _fd_check(s, dt, 8, 3, 3, 1e-6, 1e-6)


def test_adjoint_matches_cpu_fp64_directional_derivative(tmp_path):
    """An independent FP64 reference for the gradient: central differences of
    the C restatement's forward map (CPU, the reference's algorithm in FP64,
    the same fixed-dt SSP-RK3 steps) along seeded directions, against <g, d>
    of the GPU adjoint.  The receiver objective of both final states is
    evaluated by the same linear functional (the library's receivers)."""
    from oracle_bind import Oracle
    msh = _mesh(tmp_path, 8, (0.0, 10.0), 2)
    pts = _receivers(np.random.default_rng(11), 16, 1.0, 9.0)
    obs_prm = VORTEX.copy()
    obs_prm[8] = 5.5
    nsteps, every = 12, 4
    s, dt = _setup(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 2, VORTEX, obs_prm, pts, nsteps, every)
    u0 = s.get_state()
    s.forward_checkpointed(0.0, dt, nsteps, every)
    g = s.backward()
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 2, dgp.FIELD_VORTEX, VORTEX)

    def J_cpu(u):
        o.set_state(u.reshape(-1))
        for k in range(nsteps):
            o.step(k * dt, dt)
        s.set_state(o.state())
        return s.receiver_values()[1]

    rng = np.random.default_rng(13)
    eps = 1e-6
    for _ in range(4):
        d = rng.standard_normal(u0.shape)
        d /= np.linalg.norm(d)
        fd = (J_cpu(u0 + eps * d) - J_cpu(u0 - eps * d)) / (2 * eps)
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), abs(ad)), (fd, ad)


def _barth_solver(tmp_path, order=2, beta=5.0):
    """The vortex on a coarse mesh, Barth limiter after every stage (the
    vortex core spans a few cells, so the limiter acts)."""
    msh = _mesh(tmp_path, 10, (0.0, 10.0), 2)
    prm = VORTEX.copy()
    prm[8] = beta
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, prm), order,
                   dgp.FP64, dgp.LIMITER_BARTH)
    s.project(0.0)
    return s


def test_adjoint_frozen_barth_limiter_matches_fd_of_the_frozen_map(tmp_path):
    """With the Barth limiter the adjoint linearises the limiter with its
    active set frozen (the recorded slope factors as a fixed linear map).  Its
    gradient equals central differences of exactly that map: forward passes
    that replay the recorded factors (dgp_adjoint_freeze_limiter)."""
    nsteps = 12
    so = _barth_solver(tmp_path, beta=5.5)
    pts = _receivers(np.random.default_rng(4), 48, 1.0, 9.0)
    dt = 0.5 * so.cfl_dt(0.1)
    so.set_receivers(pts, np.zeros(len(pts)))
    so.forward_checkpointed(0.0, dt, nsteps, 0)
    obs, _ = so.receiver_values()
    s = _barth_solver(tmp_path)
    s.set_receivers(pts, obs)
    u0 = s.get_state()
    J0 = s.forward_checkpointed(0.0, dt, nsteps, 0)
    assert s.limiter_triggers().any()  # the limiter acted in the last pass
    g = s.backward()
    assert J0 > 0 and np.isfinite(g).all()
    # the same gradient when the backward pass recomputes segments
    s.set_state(u0)
    assert s.forward_checkpointed(0.0, dt, nsteps, 4) == J0
    assert np.array_equal(s.backward(), g)
    # central differences of the frozen map
    s.set_state(u0)
    s.forward_checkpointed(0.0, dt, nsteps, 0)  # records the factors again
    s.adjoint_freeze_limiter(True)
    with pytest.raises(dgp.DGPError):
        s.forward_checkpointed(0.0, dt, nsteps, 4)  # replay needs a recorded pass
    rng = np.random.default_rng(5)
    eps = 1e-6
    for _ in range(4):
        d = rng.standard_normal(u0.shape)
        s.set_state(u0 + eps * d)
        jp = s.forward_checkpointed(0.0, dt, nsteps, 0)
        s.set_state(u0 - eps * d)
        jm = s.forward_checkpointed(0.0, dt, nsteps, 0)
        fd = (jp - jm) / (2 * eps)
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), abs(ad)), (fd, ad)
    s.adjoint_freeze_limiter(False)
    # frozen and unfrozen forward passes agree at the recorded state itself
    s.set_state(u0)
    assert s.forward_checkpointed(0.0, dt, nsteps, 0) == J0


def test_adjoint_moment_limiter_refused(tmp_path):
    msh = _mesh(tmp_path, 6, (0.0, 1.0), 1)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE,
                                                   params(amplitude=0.25)), 2, dgp.FP64, dgp.LIMITER_MOMENT)
    with pytest.raises(dgp.DGPError) as ei:
        s.forward_checkpointed(0.0, 1e-3, 2, 1)
    assert ei.value.code == -3
    with pytest.raises(dgp.DGPError):
        s.adjoint_freeze_limiter(True)
