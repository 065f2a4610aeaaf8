"""The fused stage kernel's bounded wait for its bulk copies: a wait that gives
up is reported by dgp_status as DGP_ERR_CUDA, the CTA drains its copies and
writes nothing, and the last stage's completion count still reaches its
finalize, so the next launches run normally.

The bound is set through dgp_set_copy_wait_limit; one poll, counted from the
copies' issue, cannot see data that has to come from device memory, so every
CTA gives up.  Nothing faults and nothing waits without a bound.
"""
import os

import numpy as np
import pytest

import dgp
from dgp import meshgen
from oracle_bind import Oracle


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.gpu
def test_bounded_copy_wait_reports_and_recovers(tmp_path):
    prm = dgp.law_params(velocity=(1.0, 1.0, 0.0), center=(5.0, 5.0, 0.0), gamma=1.4, beta=5.0)
    msh = os.path.join(str(tmp_path), "vortex16.msh")
    meshgen.write_msh_v1(meshgen.tri_square(16, 16, 0.0, 10.0, 0.0, 10.0, seed=2), msh)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, prm)
    s = dgp.Solver(dgp.Mesh.from_msh(msh), law, 3)
    o = Oracle(msh, dgp.LAW_EULER2D, dgp.FLUX_ROE, 3, dgp.FIELD_VORTEX, prm)
    u0 = s.get_state()
    dt = o.cfl_dt(0.1)
    assert s.status() == (0, -1)

    s.set_copy_wait_limit(1)
    s.step(0.0, dt)
    with pytest.raises(dgp.DGPError) as ei:
        s.status()
    assert ei.value.code == -4 and "bounded wait" in str(ei.value)
    # reported once
    assert s.status() == (0, -1)

    # default bound again: steps from the same state match the oracle, through
    # dgp_step and through the device loop (whose last stage finalizes the
    # time step: the completion count was left at zero)
    s.set_copy_wait_limit(0)
    s.set_state(u0)
    s.step(0.0, dt)
    o.step(0.0, dt)
    assert rel(s.get_state(), o.state()) < 1e-12
    s.set_state(u0)
    t, n = s.run(0.0, 0.0, 0.1, 3)
    o.set_state(u0)
    t_o = 0.0
    for _ in range(3):
        d = o.cfl_dt(0.1)
        o.step(t_o, d)
        t_o += d
    assert n == 3 and abs(t - t_o) <= 1e-13 * t_o
    assert rel(s.get_state(), o.state()) < 1e-12
    assert s.status()[0] == 0
