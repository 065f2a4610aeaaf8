"""Case definitions shared by the parity tests: law/flux/field ids and the
parameters matching the golden fixtures' driver arguments."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "dg-parallel_b200"))
GOLDEN = os.path.join(ROOT, "tests", "golden")

import dgp  # noqa: E402


def params(**kw) -> np.ndarray:
    return dgp.law_params(**kw)


SCALAR2D = params(velocity=(1.0, 0.5, 0.0), center=(0.3, 0.3, 0.0), width=0.01)
VORTEX = params(velocity=(1.0, 1.0, 0.0), center=(5.0, 5.0, 0.0), gamma=1.4, beta=5.0)
SINE = params(amplitude=0.25)
SCALAR3D = params(velocity=(1.0, 0.5, 0.25), center=(0.5, 0.5, 0.5), width=0.05)
PULSE3D = params(velocity=(1.0, 0.5, 0.25), center=(0.5, 0.5, 0.5), width=0.05, gamma=1.4)
TM110 = params(cavity=1.0)
SCALAR_PERIODIC = params(velocity=(1.0, 0.5, 0.0), center=(0.2, -0.1, 0.0), width=0.1)

# golden case -> (law, flux, field, order, params)
GOLDEN_CASES = {
    "scalar_tri_p1": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 1, SCALAR2D),
    "scalar_tri_p2": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 2, SCALAR2D),
    "scalar_tri_p3": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 3, SCALAR2D),
    "scalar_tri_p4": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 4, SCALAR2D),
    "euler_godunov_p2": (dgp.LAW_EULER2D, dgp.FLUX_GODUNOV, dgp.FIELD_VORTEX, 2, VORTEX),
    "euler_godunov_p3": (dgp.LAW_EULER2D, dgp.FLUX_GODUNOV, dgp.FIELD_VORTEX, 3, VORTEX),
    "euler_roe_p1": (dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 1, VORTEX),
    "euler_roe_p3": (dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 3, VORTEX),
    "euler_roe_p4": (dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, 4, VORTEX),
    "burgers_p2": (dgp.LAW_BURGERS2D, dgp.FLUX_CENTRAL, dgp.FIELD_SINE, 2, SINE),
    "scalar_tet_p2": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS3D, 2, SCALAR3D),
    "euler3d_p1": (dgp.LAW_EULER3D, dgp.FLUX_GODUNOV, dgp.FIELD_PULSE3D, 1, PULSE3D),
    "euler3d_p2": (dgp.LAW_EULER3D, dgp.FLUX_GODUNOV, dgp.FIELD_PULSE3D, 2, PULSE3D),
    # periodic edges (510 left/right, 610 bottom/top) on [-1,1]^2
    "scalar_periodic_p2": (dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, 2, SCALAR_PERIODIC),
    "burgers_periodic_p3": (dgp.LAW_BURGERS2D, dgp.FLUX_CENTRAL, dgp.FIELD_SINE, 3, SINE),
    # Maxwell2d, TM cavity mode (far field; reflection on 40000)
    "maxwell2d_p1": (dgp.LAW_MAXWELL2D, dgp.FLUX_UPWIND, dgp.FIELD_TM2D, 1, TM110),
    "maxwell2d_p2": (dgp.LAW_MAXWELL2D, dgp.FLUX_UPWIND, dgp.FIELD_TM2D, 2, TM110),
    "maxwell2d_p3": (dgp.LAW_MAXWELL2D, dgp.FLUX_UPWIND, dgp.FIELD_TM2D, 3, TM110),
    "maxwell2d_wall_p2": (dgp.LAW_MAXWELL2D, dgp.FLUX_UPWIND, dgp.FIELD_TM2D, 2, TM110),
}

# Relative tolerance (max abs difference / max abs value) of the oracle -- exact
# Gram-Schmidt basis and full-precision rules -- against DG-Parallel's output.
# DG-Parallel evaluates its basis from decimal tables (OrthoSFTri.h,
# TetOrtho.h) whose coefficients carry relative errors growing with the order
# (up to 2.5e-11 at P3 and 8e-9 at P4), and its 3-point triangle rule is
# truncated at 1e-14.  Measured on the golden cases: states <= 4.5e-13 (P1),
# 9.5e-14 (P2), 7e-13 (P3), 1.1e-10 (P4); assembled RHS <= 8.2e-12 (P1-P3),
# 6e-10 (P4).
REF_TOL = {1: 1e-12, 2: 2e-13, 3: 2e-12, 4: 3e-10}
REF_RHS_TOL = {1: 2e-11, 2: 2e-11, 3: 2e-11, 4: 2e-9}


def golden(name):
    return os.path.join(GOLDEN, name + ".msh"), np.load(os.path.join(GOLDEN, name + ".npz"))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
