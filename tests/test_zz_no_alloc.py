"""dgp_rhs_noalloc: the right-hand side for callers that cannot allocate.

Some host codes cannot call cudaMalloc when they need a right-hand side (their
device memory belongs to another allocator, or they cannot afford the
synchronisation an allocation implies).  dgp_rhs_noalloc serves them: state in
and RHS out are the caller's device buffers and every intermediate lives in a
32 MiB static device array inside the library.  These tests call it through the
C ABI and check it against dgp_rhs, twice in a row (the static array keeps the
previous call's contents), and check that a mesh too large for the array is
refused.  The file is named to be collected last.
"""
import ctypes
import os

import numpy as np
import pytest

import dgp
from dgp import meshgen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 RHS tolerance of the parity tests (same kernels, same inputs)


def rhs_noalloc(solver, state_ptr, t, out_ptr):
    f = dgp.lib().dgp_rhs_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f(solver.h, ctypes.c_void_p(state_ptr), t, ctypes.c_void_p(out_ptr))


def vortex_solver(path, n, order=3, precision=dgp.FP64):
    meshgen.write_msh_v1(meshgen.tri_square(n, n, 0.0, 10.0, 0.0, 10.0, seed=2), path)
    prm = dgp.law_params(velocity=(1.0, 1.0, 0.0), center=(5.0, 5.0, 0.0), gamma=1.4, beta=5.0)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, prm)
    return dgp.Solver(dgp.Mesh.from_msh(path), law, order, precision)


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("fused", [True, False])
def test_rhs_noalloc_matches_rhs_on_consecutive_calls(tmp_path, fused):
    torch = pytest.importorskip("torch")
    s = vortex_solver(str(tmp_path / "v12.msh"), 12)
    s.set_fused(fused)
    s.run(0.0, 0.0, 0.1, 3)  # a non-trivial state
    for t in (0.02, 0.31):   # two calls in a row, different states and times
        state = s.get_state()
        ref = s.rhs(t)
        dev_state = torch.from_numpy(state.ravel().copy()).cuda()
        dev_out = torch.full_like(dev_state, float("nan"))
        torch.cuda.synchronize()
        dgp.check(rhs_noalloc(s, dev_state.data_ptr(), t, dev_out.data_ptr()))
        got = dev_out.cpu().numpy().reshape(s.shape)
        assert np.isfinite(got).all()
        assert rel(got, ref) < TOL
        s.step(t, 1e-3)  # move to another state for the second call


@pytest.mark.parametrize("fused,n", [(False, 136), (True, 170)])
def test_rhs_noalloc_refuses_meshes_beyond_the_scratch(tmp_path, fused, n):
    """Separate form: 36992 cells need ~36 MiB of intermediates (state, RHS,
    slots, traces); fused form: 57800 cells need ~37 MiB (state and RHS)."""
    torch = pytest.importorskip("torch")
    s = vortex_solver(str(tmp_path / f"v{n}.msh"), n)
    s.set_fused(fused)
    n = int(np.prod(s.shape))
    dev_state = torch.zeros(n, dtype=torch.float64, device="cuda")
    dev_out = torch.zeros_like(dev_state)
    rc = rhs_noalloc(s, dev_state.data_ptr(), 0.0, dev_out.data_ptr())
    assert rc == -1
    assert "32 MiB" in dgp.lib().dgp_last_error().decode()
