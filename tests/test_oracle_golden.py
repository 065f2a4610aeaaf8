"""The C oracle against DG-Parallel's own output (golden fixtures made by
tests/golden/make_golden.py from the reference compiled from source)."""
import numpy as np
import pytest

from cases import GOLDEN_CASES, REF_RHS_TOL, REF_TOL, golden, rel
from oracle_bind import Oracle, lib


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_reference(name):
    law, flux, field, order, prm = GOLDEN_CASES[name]
    msh, g = golden(name)
    o = Oracle(msh, law, flux, order, field, prm)
    dim = 3 if "tet" in name or "3d" in name else 2
    # connectivity: identical face set, left/right cells, local faces and ids
    conn = o.connectivity(dim)
    assert set(map(tuple, conn)) == set(map(tuple, g["conn"].astype(np.int32)))
    tol = REF_TOL[order]
    states = g["states"]
    assert rel(o.state().reshape(o.ncells, -1), states[0]) < tol
    assert rel(o.rhs(0.0).reshape(o.ncells, -1), g["rhs"]) < REF_RHS_TOL[order]
    t = 0.0
    for k in range(1, int(g["steps"]) + 1):
        dt = o.cfl_dt(0.1)
        assert abs(dt - g["log"][k - 1, 1]) <= max(1e-13, tol) * dt
        resid = o.step(t, dt)
        t += dt
        assert rel(o.state().reshape(o.ncells, -1), states[k]) < tol
        assert abs(resid - g["log"][k - 1, 3]) <= 1e-9 * abs(g["log"][k - 1, 3]) + 1e-300


def test_glibc_rand_restatement():
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    for seed in [1, 2, 3, 7, 100, 4096, 65537, 123456, 2**31 - 1]:
        libc.srand(seed)
        assert libc.rand() == lib().or_glibc_rand_first(seed)


def test_oracle_run_lands_on_tend():
    name = "scalar_tri_p2"
    law, flux, field, order, prm = GOLDEN_CASES[name]
    msh, _ = golden(name)
    o = Oracle(msh, law, flux, order, field, prm)
    t, n = o.run(0.0, 0.01, 0.1, 0)
    assert n > 0 and abs(t - 0.01) < 1e-15
