"""Error norms of DGError.cc (field, pressure and entropy errors; L1, L2, Linf;
the volume rule of degree 2p or the rule of degree 2(p+1)).

CPU: the oracle's restatement against its own L2 density error, against
hand-made states with known errors, and against the norms DG-Parallel itself
computes (fixtures).  GPU: the CUDA reduction against the oracle on the same
state and against the same fixtures.
"""
import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import VORTEX, SCALAR2D, golden
from oracle_bind import Oracle


def _vortex_msh(tmp_path, n=6):
    m = meshgen.tri_square(n, n, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)
    p = str(tmp_path / f"vortex{n}.msh")
    meshgen.write_msh_v1(m, p)
    return p


def _evolved_oracle(msh, order=2, steps=3):
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, order, dgp.FIELD_VORTEX, VORTEX)
    o.run(0.0, 0.0, 0.1, steps)
    return o


def test_oracle_norms_l2_density_equals_l2_error(tmp_path):
    o = _evolved_oracle(_vortex_msh(tmp_path))
    n = o.error_norms(0.0, 0, 1)
    # the state is at t > 0; compare at the same (arbitrary) time
    assert abs(n[1] - o.l2_error(0.0, 0)) <= 1e-14 * max(n[1], 1e-300)
    assert n[0] >= 0 and n[2] >= 0
    o.close()


def test_oracle_norms_vanish_on_the_projection_of_a_constant(tmp_path):
    # a constant state equal to the far field: every error vanishes except the
    # projection error of the exact vortex
    o = _evolved_oracle(_vortex_msh(tmp_path), steps=0)
    for q in (0, 1, 2, 3, -1, -2):
        for rule in (0, 1):
            l1, l2, li = o.error_norms(0.0, q, rule)
            assert 0.0 <= l1 and 0.0 <= l2 and 0.0 <= li
            # the projection error of P2 on this mesh is small but not zero
            assert li < 0.5
    o.close()


def test_oracle_norms_scalar_constant_shift(tmp_path):
    # a state shifted by a constant c from the projection: Linf of the
    # difference grows by at most |c|, L1 by at most |c| |domain|
    m = meshgen.tri_square(6, 6, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=1)
    p = str(tmp_path / "sq.msh")
    meshgen.write_msh_v1(m, p)
    o = Oracle(p, dgp.LAW_SCALAR, dgp.FLUX_UPWIND, 2, dgp.FIELD_GAUSS, SCALAR2D)
    base = o.error_norms(0.0, 0, 0)
    c = o.state()
    c[:, 0, 0] += 0.25 / np.sqrt(2.0)  # mean shift 0.25 (phi_0 = sqrt 2)
    o.set_state(c)
    shifted = o.error_norms(0.0, 0, 0)
    assert shifted[2] <= base[2] + 0.25 + 1e-12
    assert shifted[0] <= base[0] + 0.25 * 1.0 + 1e-12
    assert shifted[2] >= 0.25 - base[2] - 1e-12
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2, 3])
def test_gpu_norms_match_oracle(tmp_path, order):
    msh = _vortex_msh(tmp_path)
    o = _evolved_oracle(msh, order)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX),
                   order, dgp.FP64)
    s.set_state(o.state())
    t = 0.37
    for q in (0, 1, 2, 3, -1, -2):
        for rule in (0, 1):
            g = s.error_norms(t, q, rule)
            r = o.error_norms(t, q, rule)
            assert np.allclose(g, r, rtol=1e-12, atol=0.0), (q, rule, g, r)
    assert abs(s.error_norms(t, 0, 1)[1] - s.l2_error(t, 0)) <= 1e-13 * s.l2_error(t, 0)
    s.close()
    o.close()


# DGAnalysis's norms (DGPref.cc:249-381) as the reference computes them on its
# own state after five steps (tests/golden/norms_*.npz, ref_driver --norms):
# name -> (quantity, rule, index into (L1, L2, Linf))
REFERENCE_NORMS = {
    "ExactError": (0, 0, 0),
    "LinfError": (0, 0, 2),
    "densityErrorL2": (0, 1, 1),
    "PressureError": (-1, 0, 0),
    "entropyErrorL1": (-2, 0, 0),
    "pressureErrorL2": (-1, 1, 1),
    "entropyErrorL2": (-2, 1, 1),
}
NORM_CASES = [
    ("norms_euler_roe_p3", dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX, 3),
    ("norms_scalar_p2", dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, SCALAR2D, 2),
]
# the reference's basis tables (decimal, ~1e-11 at P3) set the floor
NORM_TOL = 1e-10


def _reference_norms(g):
    return {k: float(g[k]) for k in REFERENCE_NORMS if k in g.files}


@pytest.mark.parametrize("name,law,flux,field,prm,order", NORM_CASES)
def test_oracle_norms_match_reference(name, law, flux, field, prm, order):
    msh, g = golden(name)
    o = Oracle(msh, law, flux, order, field, prm)
    o.set_state(g["state"].reshape(o.shape))
    t = float(g["t"])
    for k, ref in _reference_norms(g).items():
        q, rule, i = REFERENCE_NORMS[k]
        got = o.error_norms(t, q, rule)[i]
        assert abs(got - ref) <= NORM_TOL * ref, (k, got, ref)
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,law,flux,field,prm,order", NORM_CASES)
def test_gpu_norms_match_reference(name, law, flux, field, prm, order):
    msh, g = golden(name)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), dgp.Law(law, flux, field, prm), order, dgp.FP64)
    s.set_state(g["state"].reshape(s.shape))
    t = float(g["t"])
    for k, ref in _reference_norms(g).items():
        q, rule, i = REFERENCE_NORMS[k]
        got = s.error_norms(t, q, rule)[i]
        assert abs(got - ref) <= NORM_TOL * ref, (k, got, ref)
    s.close()
