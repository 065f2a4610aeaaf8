"""Point and line probes (DGPointSensor / DGLineSensor / DGTresholdLineSensor,
DGSensor.cc:88-186) evaluated on the device, on demand and inside a run."""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import REF_TOL, SCALAR3D, VORTEX, golden, rel


def test_line_points_match_the_line_sensor_samples():
    p = dgp.line_points((0.0, 1.0, 0.0), (2.0, 3.0, 0.0), 5)
    assert p.shape == (5, 3)
    assert np.allclose(p[:, 0], [0.0, 0.5, 1.0, 1.5, 2.0])
    assert np.allclose(p[:, 1], [1.0, 1.5, 2.0, 2.5, 3.0])


def test_first_crossing():
    v = np.array([[0.0], [0.2], [0.6], [0.9], [0.3]])
    assert dgp.first_crossing(v, 0, 0.5) == 2
    assert dgp.first_crossing(v, 0, 2.0) == -1
    # touching the threshold is not a crossing (strict inequalities)
    assert dgp.first_crossing(np.array([[0.0], [0.5], [1.0]]), 0, 0.5) == -1


def _vortex_solver(n=24, order=3, prec=dgp.FP64):
    m = meshgen.tri_square(n, n, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)
    mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, 100, m.bfaces, m.btags)
    s = dgp.Solver(mesh, dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX), order, prec)
    s.project(0.0)
    return s


@pytest.mark.gpu
def test_gpu_probe_values_match_receivers_and_exact_field():
    s = _vortex_solver()
    rng = np.random.default_rng(11)
    pts = rng.uniform(0.5, 9.5, size=(40, 2))
    pr = dgp.Probe(s, pts)
    assert pr.found.all()
    v = pr.eval()
    # the receivers evaluate field 0 through their own kernel
    s.set_receivers(pts, np.zeros(len(pts)))
    rho, _ = s.receiver_values()
    assert np.array_equal(v[:, 0], rho)
    # the projection of the vortex is close to it at P3
    ex = np.array([dgp_exact_vortex(p) for p in pts])
    assert np.abs(v - ex).max() < 1e-2
    pr.close()
    s.close()


def dgp_exact_vortex(p, beta=5.0, gamma=1.4, x0=5.0, y0=5.0):
    # isentropic vortex at t = 0 (free stream (1, 1, 1, 1))
    x, y = p[0] - x0, p[1] - y0
    r2 = x * x + y * y
    du = -beta / (2 * np.pi) * np.exp((1 - r2) / 2) * y
    dv = beta / (2 * np.pi) * np.exp((1 - r2) / 2) * x
    T = 1 - (gamma - 1) * beta ** 2 / (8 * gamma * np.pi ** 2) * np.exp(1 - r2)
    rho = T ** (1 / (gamma - 1))
    u, v = 1 + du, 1 + dv
    pr = rho ** gamma
    return np.array([rho, rho * u, rho * v, pr / (gamma - 1) + 0.5 * rho * (u * u + v * v)])


@pytest.mark.gpu
def test_gpu_probe_outside_points_are_nan():
    s = _vortex_solver(n=8, order=1)
    pr = dgp.Probe(s, np.array([[5.0, 5.0], [11.0, 5.0], [-0.5, 3.0]]))
    assert list(pr.found) == [True, False, False]
    v = pr.eval()
    assert np.isfinite(v[0]).all() and np.isnan(v[1:]).all()
    pr.close()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [dgp.FP64, dgp.MIXED])
def test_gpu_probe_records_inside_the_run(prec):
    s = _vortex_solver(n=16, order=2, prec=prec)
    line = dgp.line_points((1.0, 5.0), (9.0, 5.0), 33)
    pr = dgp.Probe(s, line)
    pr.record(every=3, max_samples=16)
    t, n = s.run(0.0, 0.0, 0.1, 30)
    assert n == 30
    times, vals = pr.samples()
    assert len(times) == 10 and vals.shape == (10, 33, 4)
    assert np.all(np.diff(times) > 0) and abs(times[-1] - t) <= 1e-12 * t
    # the last sample is the final state
    assert np.array_equal(vals[-1], pr.eval())
    # recording runs inside the step graph: the same run without a recorder
    # reaches the same state
    final = s.get_state()
    s2 = _vortex_solver(n=16, order=2, prec=prec)
    s2.run(0.0, 0.0, 0.1, 30)
    assert np.array_equal(s2.get_state(), final)
    # a second run restarts the samples; stopping removes the recorder
    s.run(t, 0.0, 0.1, 6)
    assert len(pr.samples()[0]) == 2
    pr.record(every=0, max_samples=0)
    s.run(t, 0.0, 0.1, 6)
    pr.close()
    s.close()
    s2.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,law,flux,field,prm", [
    ("probes_euler_roe_p2", dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX),
    ("probes_scalar_tet_p2", dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS3D, SCALAR3D),
])
def test_gpu_probes_match_reference_point_sensor(name, law, flux, field, prm):
    """Pinned against DG-Parallel's own point evaluation (DGPointSensor through
    DGCell::inCell) on the reference's state after three steps: the same points
    found, the same values to the basis-table floor."""
    msh, g = golden(name)
    order = int(list(g["args"])[list(g["args"]).index("--order") + 1])
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(law, flux, field, prm), order, dgp.FP64)
    E = s.ncells
    s.set_state(g["state"].reshape(E, s.nfields, -1))
    pts = g["points"][:, : (2 if "tet" not in name else 3)]
    pr = dgp.Probe(s, pts)
    assert np.array_equal(pr.found, g["cell"] >= 0)
    v = pr.eval()
    ok = g["cell"] >= 0
    assert np.isnan(v[~ok]).all()
    assert rel(v[ok], g["values"][ok]) < REF_TOL[order]
