"""ctypes binding of the C oracle (oracle/_build/liboracle.so) for the tests.

The oracle is the checker: it restates DG-Parallel's CPU algorithm in plain C
(see oracle/dg_oracle.h).  Only tests, the smoke check and the bench's CPU
baseline use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)
    L = ctypes.CDLL(ORACLE_SO)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    pD = ctypes.POINTER(ctypes.c_double)
    pI = ctypes.POINTER(ctypes.c_int)
    L.or_create.restype = P
    L.or_create.argtypes = [ctypes.c_char_p, I, I, I, I, pD]
    L.or_create_rule.restype = P
    L.or_create_rule.argtypes = [ctypes.c_char_p, I, I, I, I, pD, I]
    for f in ("or_num_cells", "or_num_faces", "or_num_fields", "or_num_modes"):
        getattr(L, f).argtypes = [P]
        getattr(L, f).restype = I
    L.or_destroy.argtypes = [P]
    L.or_connectivity.argtypes = [P, pI]
    L.or_connectivity.restype = I
    L.or_face_normals.argtypes = [P, pD]
    L.or_get_state.argtypes = [P, pD]
    L.or_set_state.argtypes = [P, pD]
    L.or_project.argtypes = [P, D]
    L.or_rhs.argtypes = [P, D, pD]
    L.or_rhs_p0.argtypes = [P, D, pD]
    L.or_rhs_p0.restype = I
    L.or_cfl_dt.argtypes = [P, D]
    L.or_cfl_dt.restype = D
    L.or_step.argtypes = [P, D, D]
    L.or_step.restype = D
    L.or_run.argtypes = [P, D, D, D, I, pI]
    L.or_run.restype = D
    L.or_l2_error.argtypes = [P, D, I]
    L.or_l2_error.restype = D
    L.or_error_norms.argtypes = [P, D, I, I, ctypes.POINTER(ctypes.c_double)]
    L.or_error_norms.restype = I
    pU8 = ctypes.POINTER(ctypes.c_uint8)
    L.or_set_limiter.argtypes = [P, I]
    L.or_limit.argtypes = [P, pU8]
    L.or_limit.restype = I
    L.or_set_p0_fallback.argtypes = [P, I]
    L.or_bad_cells.argtypes = [P, pU8]
    L.or_triggers.argtypes = [P, pU8]
    L.or_lts_setup.argtypes = [P]
    L.or_lts_setup.restype = I
    L.or_lts_bins.argtypes = [P, pI, pI]
    L.or_lts_step.argtypes = [P, D, D]
    L.or_lts_step.restype = D
    L.or_lts_dt.argtypes = [P, D]
    L.or_lts_dt.restype = D
    L.or_glibc_rand_first.argtypes = [ctypes.c_uint]
    L.or_glibc_rand_first.restype = ctypes.c_uint
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    def __init__(self, msh: str, law: int, flux: int, order: int, field: int, params, rule: int = 0):
        p = np.ascontiguousarray(params, dtype=np.float64)
        self.h = lib().or_create_rule(msh.encode(), law, flux, order, field, _dp(p), rule)
        if not self.h:
            raise RuntimeError(f"oracle could not load {msh}")
        L = lib()
        self.ncells = L.or_num_cells(self.h)
        self.nfaces = L.or_num_faces(self.h)
        self.nfields = L.or_num_fields(self.h)
        self.nmodes = L.or_num_modes(self.h)
        self.shape = (self.ncells, self.nfields, self.nmodes)

    def connectivity(self, dim):
        n = dim + 5
        out = np.zeros(self.nfaces * n, dtype=np.int32)
        lib().or_connectivity(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return out.reshape(self.nfaces, n)

    def state(self):
        out = np.zeros(self.shape)
        lib().or_get_state(self.h, _dp(out))
        return out

    def set_state(self, c):
        c = np.ascontiguousarray(c, dtype=np.float64)
        lib().or_set_state(self.h, _dp(c))

    def rhs(self, t):
        out = np.zeros(self.shape)
        lib().or_rhs(self.h, t, _dp(out))
        return out

    def rhs_p0(self, t):
        """RHS of one assembly with the P0 fallback (when on); the marked
        cells' modes k >= 1 are zeroed in the state.  (rhs, marked cells)"""
        out = np.zeros(self.shape)
        n = lib().or_rhs_p0(self.h, t, _dp(out))
        return out, n

    def cfl_dt(self, cfl):
        return lib().or_cfl_dt(self.h, cfl)

    def step(self, t, dt):
        return lib().or_step(self.h, t, dt)

    def run(self, t0, tend, cfl, nsteps):
        n = ctypes.c_int()
        t = lib().or_run(self.h, t0, tend, cfl, nsteps, ctypes.byref(n))
        return t, n.value

    def l2_error(self, t, field=0):
        return lib().or_l2_error(self.h, t, field)

    def error_norms(self, t, quantity=0, rule=1):
        out = np.zeros(3)
        rc = lib().or_error_norms(self.h, t, quantity, rule, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert rc == 0
        return out

    def set_limiter(self, on=True):
        """on: True / 1 triangle moment limiter, 2 Barth limiter, False / 0 off."""
        lib().or_set_limiter(self.h, int(on) if not isinstance(on, bool) else (1 if on else 0))

    def set_p0_fallback(self, on=True):
        lib().or_set_p0_fallback(self.h, 1 if on else 0)

    def limit(self):
        """Apply the triangle moment limiter once; per-cell trigger degrees."""
        trig = np.zeros(self.ncells, dtype=np.uint8)
        lib().or_limit(self.h, trig.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return trig

    def triggers(self):
        """Trigger degrees of the last limiter application."""
        out = np.zeros(self.ncells, dtype=np.uint8)
        lib().or_triggers(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return out

    def bad_cells(self):
        out = np.zeros(self.ncells, dtype=np.uint8)
        lib().or_bad_cells(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return out

    def lts_setup(self):
        """Size bins of DGAnalysis::sortCellsBySize; number of bins or < 0."""
        return lib().or_lts_setup(self.h)

    def lts_bins(self):
        bins = np.zeros(self.ncells, dtype=np.int32)
        role = np.zeros(self.ncells, dtype=np.int32)
        pI = ctypes.POINTER(ctypes.c_int)
        lib().or_lts_bins(self.h, bins.ctypes.data_as(pI), role.ctypes.data_as(pI))
        return bins, role

    def lts_step(self, t, dt):
        return lib().or_lts_step(self.h, t, dt)

    def lts_dt(self, cfl):
        return lib().or_lts_dt(self.h, cfl)

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
