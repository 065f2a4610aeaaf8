"""The drop-in boundary end to end: DG-Parallel's own driver code (mesh import,
DGCell projection, CFL reduction, output) steps its cells through the
reference-side shim dg-parallel_b200/integration/GpuTimeIntegrator.h
(oracle/_ref/ref_driver_gpu --gpu 1) instead of its RungeKuttaTVD3, and the
states match the reference's own integration step by step.  The shim reads
the library's law and flux ids off the reference's law object
(GpuConservationLaw)."""
import os
import subprocess

import numpy as np
import pytest

from cases import GOLDEN, REF_TOL, ROOT

REF = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "ref_driver_gpu")

CASES = {
    "scalar_tri_p2": ["--case", "gauss", "--order", "2"],
    "euler_roe_p3": ["--case", "vortex", "--flux", "roe", "--order", "3"],
    "euler_godunov_p2": ["--case", "vortex", "--flux", "exact", "--order", "2"],
    "burgers_p2": ["--case", "sine", "--order", "2", "--amp", "0.25"],
    "maxwell2d_wall_p2": ["--case", "tm2d", "--order", "2"],
    "scalar_tet_p2": ["--case", "gauss3d", "--order", "2", "--ax", "1", "--ay", "0.5", "--az", "0.25",
                      "--cx", "0.5", "--cy", "0.5", "--cz", "0.5", "--s", "0.05"],
}


def _states(path):
    blocks = open(path).read().split("step ")[1:]
    return [np.array([list(map(float, ln.split())) for ln in b.split("\n")[1:] if ln.strip()]) for b in blocks]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_driver_steps_through_the_shim(tmp_path, name):
    if not (os.path.exists(REF) and os.path.exists(REF_GPU)):
        pytest.skip("reference drivers not built (make -C oracle ref ref_gpu)")
    msh = os.path.join(GOLDEN, name + ".msh")
    args = ["--mesh", msh, "--steps", "4", "--cfl", "0.1"] + CASES[name]
    cpu, gpu = str(tmp_path / "cpu"), str(tmp_path / "gpu")
    subprocess.run([REF] + args + ["--state", cpu], check=True, capture_output=True, timeout=300)
    subprocess.run([REF_GPU] + args + ["--gpu", "1", "--state", gpu], check=True, capture_output=True,
                   timeout=300)
    a, b = _states(cpu), _states(gpu)
    assert len(a) == len(b) == 5
    order = int(CASES[name][CASES[name].index("--order") + 1])
    for k in range(5):
        err = np.abs(b[k] - a[k]).max() / np.abs(a[k]).max()
        # the reference's decimal basis tables set the floor (tests/cases.py)
        assert err <= 10 * REF_TOL[order], (k, err)
