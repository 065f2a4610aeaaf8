"""ctypes binding of libdgp.so (the C ABI in include/dgp.h).

This module only marshals arguments; every computation runs in the CUDA
library.  Importing it loads ``dg-parallel_b200/lib/libdgp.so`` and raises if the
library is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libdgp.so")

LAW_SCALAR, LAW_BURGERS2D, LAW_EULER2D, LAW_EULER3D, LAW_MAXWELL3D, LAW_MAXWELL2D = range(6)
FLUX_UPWIND, FLUX_CENTRAL, FLUX_GODUNOV, FLUX_ROE, FLUX_LLF = range(5)
FIELD_GAUSS, FIELD_VORTEX, FIELD_PULSE3D, FIELD_SINE, FIELD_GAUSS3D, FIELD_TM110, FIELD_TM2D = range(7)
BC_DEFAULT, BC_FARFIELD, BC_WALL = range(3)
RULE_REFERENCE, RULE_WORKLOAD = range(2)  # quadrature: DG-Parallel's, the workloads' P2 point counts
FP64, MIXED = 0, 1
LIMITER_NONE, LIMITER_MOMENT, LIMITER_BARTH = 0, 1, 2
STEPPING_SSPRK3, STEPPING_LOCAL = 0, 5
NPARAMS = 16

ERRORS = {-1: "invalid argument", -2: "I/O", -3: "unsupported", -4: "CUDA", -5: "non-physical",
          -6: "out of memory"}


class DGPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dgp error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    """Load libdgp.so once; raises FileNotFoundError when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run dg-parallel_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    pI = ctypes.POINTER(ctypes.c_int)
    pD = ctypes.POINTER(ctypes.c_double)
    pP = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "dgp_last_error": ([], ctypes.c_char_p),
        "dgp_set_device": ([I], I),
        "dgp_version": ([], I),
        "dgp_mesh_from_msh": ([ctypes.c_char_p, pP], I),
        "dgp_mesh_from_arrays": ([I, I, pD, pI, I, pI, I, I, pI, pI, pP], I),
        "dgp_mesh_from_msh_ex": ([ctypes.c_char_p, I, pP], I),
        "dgp_mesh_from_arrays_ex": ([I, I, pD, pI, I, pI, I, I, pI, pI, I, pP], I),
        "dgp_mesh_info": ([P, pI, pI, pI, pI], I),
        "dgp_mesh_connectivity": ([P, pI], I),
        "dgp_mesh_face_geometry": ([P, pD], I),
        "dgp_mesh_destroy": ([P], I),
        "dgp_law_create": ([I, I, I, pD, pP], I),
        "dgp_law_set_bc": ([P, I, I], I),
        "dgp_law_destroy": ([P], I),
        "dgp_solver_create": ([P, P, I, I, I, pP], I),
        "dgp_solver_create_ex": ([P, P, I, I, I, I, pP], I),
        "dgp_solver_destroy": ([P], I),
        "dgp_solver_info": ([P, pI, pI, pI, pI], I),
        "dgp_project": ([P, D], I),
        "dgp_set_state": ([P, pD], I),
        "dgp_get_state": ([P, pD], I),
        "dgp_set_state_device": ([P, P], I),
        "dgp_get_state_device": ([P, P], I),
        "dgp_rhs": ([P, D, pD], I),
        "dgp_cfl_dt": ([P, D, pD], I),
        "dgp_step": ([P, D, D, pD], I),
        "dgp_run": ([P, D, D, D, I, pD, pI], I),
        "dgp_status": ([P, pI, pI], I),
        "dgp_l2_error": ([P, D, I, pD], I),
        "dgp_error_norms": ([P, D, I, I, pD], I),
        "dgp_checkpoint_write": ([P, ctypes.c_char_p, D, I], I),
        "dgp_checkpoint_read": ([P, ctypes.c_char_p, pD, pI], I),
        "dgp_probe_create": ([P, I, pD, pP, pI], I),
        "dgp_probe_destroy": ([P], I),
        "dgp_probe_info": ([P, pI, pI], I),
        "dgp_probe_eval": ([P, pD], I),
        "dgp_probe_record": ([P, I, I], I),
        "dgp_probe_samples": ([P, pI, pD, pD], I),
        "dgp_totals": ([P, pD], I),
        "dgp_synchronize": ([P], I),
        "dgp_solver_stream": ([P, pP], I),
        "dgp_profile_kernels": ([P, I, ctypes.POINTER(ctypes.c_float)], I),
        "dgp_limit": ([P, ctypes.POINTER(ctypes.c_uint8)], I),
        "dgp_limiter_triggers": ([P, ctypes.POINTER(ctypes.c_uint8)], I),
        "dgp_set_p0_fallback": ([P, I], I),
        "dgp_set_copy_wait_limit": ([P, I], I),
        "dgp_set_tensor_cores": ([P, I], I),
        "dgp_set_rounding_probe": ([P, I], I),
        "dgp_launches_per_step": ([P, pI], I),
        "dgp_set_time_stepping": ([P, I, pI], I),
        "dgp_lts_bins": ([P, pI, pI], I),
        "dgp_ensemble_create": ([I, pP, pP, pI, I, I, pP], I),
        "dgp_ensemble_destroy": ([P], I),
        "dgp_ensemble_info": ([P, I, pI, pI, pI, pI], I),
        "dgp_ensemble_project": ([P, D], I),
        "dgp_ensemble_get_state": ([P, I, pD], I),
        "dgp_ensemble_set_state": ([P, I, pD], I),
        "dgp_ensemble_run": ([P, D, D, D, I, pD, pI, pD, pD], I),
        "dgp_ensemble_totals": ([P, I, pD], I),
        "dgp_ensemble_l2_error": ([P, I, D, I, pD], I),
        "dgp_ensemble_launches_per_step": ([P, pI], I),
        "dgp_autotune": ([P, P, I, I, I, I, pI, ctypes.POINTER(ctypes.c_float)], I),
        "dgp_autotune_ensemble": ([I, pP, pP, pI, I, I, I], I),
        "dgp_tune_set": ([I, I, I, I, I, I, I], I),
        "dgp_adjoint_set_receivers": ([P, I, pD, pD], I),
        "dgp_receiver_values": ([P, pD, pD], I),
        "dgp_forward_checkpointed": ([P, D, D, I, I, pD], I),
        "dgp_adjoint_freeze_limiter": ([P, I], I),
        "dgp_backward": ([P, pD, pD], I),
        "dgp_solver_block": ([P, pI, pI], I),
        "dgp_solver_fused": ([P, pI], I),
        "dgp_set_fused": ([P, I], I),
        "dgp_ensemble_group_block": ([P, I, pI, pI], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != 0:
        raise DGPError(rc, lib().dgp_last_error().decode())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def law_params(velocity=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0), width=1.0, gamma=1.4, beta=5.0,
               amplitude=1.0, cavity=1.0) -> np.ndarray:
    p = np.zeros(NPARAMS)
    p[0:3] = velocity
    p[3:6] = center
    p[6] = width
    p[7] = gamma
    p[8] = beta
    p[9] = amplitude
    p[10] = cavity
    return p


class Mesh:
    def __init__(self, handle):
        self.h = handle
        dim, e, f, v = (ctypes.c_int() for _ in range(4))
        check(lib().dgp_mesh_info(self.h, ctypes.byref(dim), ctypes.byref(e), ctypes.byref(f),
                                  ctypes.byref(v)))
        self.dim, self.ncells, self.nfaces, self.nvertices = dim.value, e.value, f.value, v.value

    @classmethod
    def from_msh(cls, path: str, gpu_faces: bool = False) -> "Mesh":
        """gpu_faces: match the faces on the current CUDA device."""
        h = ctypes.c_void_p()
        check(lib().dgp_mesh_from_msh_ex(path.encode(), 1 if gpu_faces else 0, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, dim, xyz, cells, cell_tag=100, bfaces=None, btags=None,
                    vertex_ids=None, gpu_faces: bool = False) -> "Mesh":
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        nb = 0 if bfaces is None else len(bfaces)
        bf = np.ascontiguousarray(bfaces if nb else np.zeros((1, dim)), dtype=np.int32)
        bt = np.ascontiguousarray(btags if nb else np.zeros(1), dtype=np.int32)
        vids = None if vertex_ids is None else np.ascontiguousarray(vertex_ids, dtype=np.int32)
        h = ctypes.c_void_p()
        check(lib().dgp_mesh_from_arrays_ex(dim, xyz.shape[0], _dp(xyz), _ip(vids) if vids is not None else None,
                                            cells.shape[0], _ip(cells), cell_tag, nb, _ip(bf), _ip(bt),
                                            1 if gpu_faces else 0, ctypes.byref(h)))
        return cls(h)

    def connectivity(self) -> np.ndarray:
        n = self.dim + 5
        out = np.zeros(self.nfaces * n, dtype=np.int32)
        check(lib().dgp_mesh_connectivity(self.h, _ip(out)))
        return out.reshape(self.nfaces, n)

    def face_geometry(self) -> np.ndarray:
        out = np.zeros(self.nfaces * 4)
        check(lib().dgp_mesh_face_geometry(self.h, _dp(out)))
        return out.reshape(self.nfaces, 4)

    def close(self):
        if self.h:
            lib().dgp_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Law:
    def __init__(self, kind: int, flux: int, field: int, params=None):
        p = np.ascontiguousarray(params if params is not None else np.zeros(NPARAMS), dtype=np.float64)
        self.h = ctypes.c_void_p()
        self.kind, self.flux, self.field = kind, flux, field
        check(lib().dgp_law_create(kind, flux, field, _dp(p), ctypes.byref(self.h)))

    def set_bc(self, boundary_id: int, kind: int):
        """Boundary condition of the faces classified boundary_id (BC_DEFAULT,
        BC_FARFIELD, BC_WALL) for solvers created from this law afterwards."""
        check(lib().dgp_law_set_bc(self.h, int(boundary_id), int(kind)))

    def close(self):
        if self.h:
            lib().dgp_law_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """TimeIntegrator-style driver of one mesh + law on the current CUDA device."""

    def __init__(self, mesh: Mesh, law: Law, order: int, precision: int = FP64, limiter: int = 0,
                 rule: int = 0):
        self.mesh, self.law = mesh, law
        self.h = ctypes.c_void_p()
        check(lib().dgp_solver_create_ex(mesh.h, law.h, order, precision, limiter, rule, ctypes.byref(self.h)))
        m, n, e, f = (ctypes.c_int() for _ in range(4))
        check(lib().dgp_solver_info(self.h, ctypes.byref(m), ctypes.byref(n), ctypes.byref(e),
                                    ctypes.byref(f)))
        self.nfields, self.nmodes, self.ncells, self.nfaces = m.value, n.value, e.value, f.value
        self.shape = (self.ncells, self.nfields, self.nmodes)

    def project(self, t: float = 0.0):
        check(lib().dgp_project(self.h, t))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """State [cell][field][mode] in file order; `out` (C-contiguous float64,
        e.g. a pinned buffer) is filled in place when given."""
        if out is None:
            out = np.zeros(self.shape)
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == np.prod(self.shape)
        check(lib().dgp_get_state(self.h, _dp(out)))
        return out

    def set_state(self, c: np.ndarray):
        c = np.ascontiguousarray(c, dtype=np.float64).reshape(self.shape)
        check(lib().dgp_set_state(self.h, _dp(c)))

    def set_state_device(self, ptr: int):
        check(lib().dgp_set_state_device(self.h, ctypes.c_void_p(ptr)))

    def get_state_device(self, ptr: int):
        check(lib().dgp_get_state_device(self.h, ctypes.c_void_p(ptr)))

    def rhs(self, t: float) -> np.ndarray:
        out = np.zeros(self.shape)
        check(lib().dgp_rhs(self.h, t, _dp(out)))
        return out

    def cfl_dt(self, cfl: float) -> float:
        dt = ctypes.c_double()
        check(lib().dgp_cfl_dt(self.h, cfl, ctypes.byref(dt)))
        return dt.value

    def step(self, t: float, dt: float) -> float:
        r = ctypes.c_double()
        check(lib().dgp_step(self.h, t, dt, ctypes.byref(r)))
        return r.value

    def run(self, t0: float, tend: float, cfl: float, max_steps: int = 0) -> tuple[float, int]:
        t = ctypes.c_double()
        n = ctypes.c_int()
        check(lib().dgp_run(self.h, t0, tend, cfl, max_steps, ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    def status(self) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        check(lib().dgp_status(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def l2_error(self, t: float, field: int = 0) -> float:
        e = ctypes.c_double()
        check(lib().dgp_l2_error(self.h, t, field, ctypes.byref(e)))
        return e.value

    def write_checkpoint(self, path: str, t: float, iteration: int = 0):
        """DGAnalysis::write's data stream (readable by DGAnalysis::read)."""
        check(lib().dgp_checkpoint_write(self.h, path.encode(), t, iteration))

    def read_checkpoint(self, path: str) -> tuple[float, int]:
        """Load a DGAnalysis::write / dgp_checkpoint_write file; returns (t, iteration)."""
        t = ctypes.c_double()
        it = ctypes.c_int()
        check(lib().dgp_checkpoint_read(self.h, path.encode(), ctypes.byref(t), ctypes.byref(it)))
        return t.value, it.value

    def error_norms(self, t: float, quantity: int = 0, rule: int = 1) -> np.ndarray:
        """(L1, L2, Linf) against the exact field: quantity >= 0 a field, -1 the
        pressure, -2 the entropy deviation (Euler); rule 0 the volume rule of
        degree 2p, 1 the rule of degree 2(p+1)."""
        out = np.zeros(3)
        check(lib().dgp_error_norms(self.h, t, quantity, rule, _dp(out)))
        return out

    def totals(self) -> np.ndarray:
        out = np.zeros(self.nfields)
        check(lib().dgp_totals(self.h, _dp(out)))
        return out

    def stream(self) -> int:
        """cudaStream_t of the solver (for CUDA events recorded on it)."""
        h = ctypes.c_void_p()
        check(lib().dgp_solver_stream(self.h, ctypes.byref(h)))
        return h.value or 0

    def profile_kernels(self, iters: int = 20) -> np.ndarray:
        """Mean ms of [stage 1, stage 2, last stage with the CFL reduction] of
        the fused stage kernel; for solvers that are not fused (see `fused`):
        [face kernel, element kernel (inner stage), element kernel (last
        stage with the CFL reduction)]."""
        out = (ctypes.c_float * 3)()
        check(lib().dgp_profile_kernels(self.h, iters, out))
        return np.array(out[:], dtype=np.float64)

    def limit(self) -> np.ndarray:
        """Apply the triangle moment limiter once; per-cell trigger degree
        (0: untouched), file order."""
        out = np.zeros(self.ncells, dtype=np.uint8)
        check(lib().dgp_limit(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    def limiter_triggers(self) -> np.ndarray:
        out = np.zeros(self.ncells, dtype=np.uint8)
        check(lib().dgp_limiter_triggers(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    @property
    def fused(self) -> bool:
        """True when each stage runs as one fused stage kernel."""
        f = ctypes.c_int()
        check(lib().dgp_solver_fused(self.h, ctypes.byref(f)))
        return bool(f.value)

    def set_fused(self, on: bool = True):
        """Stages as the fused stage kernel (True) or as the separate face and
        element kernels (False)."""
        check(lib().dgp_set_fused(self.h, 1 if on else 0))

    def set_p0_fallback(self, on: bool = True):
        check(lib().dgp_set_p0_fallback(self.h, 1 if on else 0))

    def set_tensor_cores(self, on: bool = True):
        """Mixed form: run the volume contraction on the tcgen05 tensor cores
        (TF32 with split operands) instead of FP32 FMAs."""
        check(lib().dgp_set_tensor_cores(self.h, 1 if on else 0))

    def set_rounding_probe(self, mask: int = 0):
        """FP64 solver: round the terms selected by mask to FP32 (1 geometry,
        2 face traces, 4 volume values, 8 volume flux products, 16 face slots,
        32 contraction result, 64 tables) -- the mixed form's error, term by term."""
        check(lib().dgp_set_rounding_probe(self.h, int(mask)))

    def set_copy_wait_limit(self, polls: int = 0):
        """Bound the fused stage kernel's first wait for its bulk copies, in
        polls from the copies' issue (0: the default); a wait that gives up
        surfaces as DGP_ERR_CUDA in the next status()."""
        check(lib().dgp_set_copy_wait_limit(self.h, int(polls)))

    def launches_per_step(self) -> int:
        n = ctypes.c_int()
        check(lib().dgp_launches_per_step(self.h, ctypes.byref(n)))
        return n.value

    def set_time_stepping(self, mode: int = STEPPING_LOCAL) -> int:
        """DGAnalysis's timeSteppingMode: STEPPING_LOCAL (5) bins the cells by
        size and steps with RungeKuttaTVD2adaptive; STEPPING_SSPRK3 (0) goes
        back to SSP-RK3.  Returns the number of size bins (0 for SSP-RK3)."""
        n = ctypes.c_int()
        check(lib().dgp_set_time_stepping(self.h, mode, ctypes.byref(n)))
        return n.value

    def lts_bins(self):
        """(bin, role) per cell in file order; role 0 inner, 1 large and 2
        small on an interface between bins."""
        bins = np.zeros(self.ncells, dtype=np.int32)
        role = np.zeros(self.ncells, dtype=np.int32)
        pI = ctypes.POINTER(ctypes.c_int)
        check(lib().dgp_lts_bins(self.h, bins.ctypes.data_as(pI), role.ctypes.data_as(pI)))
        return bins, role

    def block(self) -> tuple[int, int]:
        """(threads, cells per element-kernel tile) of the tile shape in use."""
        b, te = ctypes.c_int(), ctypes.c_int()
        check(lib().dgp_solver_block(self.h, ctypes.byref(b), ctypes.byref(te)))
        return b.value, te.value

    # ---- discrete adjoint
    def set_receivers(self, points: np.ndarray, observed: np.ndarray):
        """J = sum_r (field0(x_r, T) - observed_r)^2; points (n, dim)."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        obs = np.ascontiguousarray(observed, dtype=np.float64)
        self._nrec = len(obs)
        check(lib().dgp_adjoint_set_receivers(self.h, len(obs), _dp(pts), _dp(obs)))

    def receiver_values(self) -> tuple[np.ndarray, float]:
        rho = np.zeros(self._nrec)
        J = ctypes.c_double()
        check(lib().dgp_receiver_values(self.h, _dp(rho), ctypes.byref(J)))
        return rho, J.value

    def adjoint_freeze_limiter(self, on: bool = True):
        """Later recorded forward passes replay the Barth slope factors of the
        last one (the frozen map the backward pass linearises)."""
        check(lib().dgp_adjoint_freeze_limiter(self.h, 1 if on else 0))

    def forward_checkpointed(self, t0: float, dt: float, nsteps: int, every: int) -> float:
        J = ctypes.c_double()
        check(lib().dgp_forward_checkpointed(self.h, t0, dt, nsteps, every, ctypes.byref(J)))
        return J.value

    def backward(self, seed: np.ndarray | None = None) -> np.ndarray:
        """dJ/du0 of the last forward_checkpointed (seed: dJ/du_T, default the
        receiver objective's)."""
        out = np.zeros(self.shape)
        sd = None
        if seed is not None:
            sd = np.ascontiguousarray(seed, dtype=np.float64).reshape(self.shape)
        check(lib().dgp_backward(self.h, _dp(sd) if sd is not None else None, _dp(out)))
        return out

    def synchronize(self):
        check(lib().dgp_synchronize(self.h))

    def close(self):
        if self.h:
            lib().dgp_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Probe:
    """Point probe (DGPointSensor; a line sensor is a Probe over line_points):
    every field at every point, evaluated on the device, on demand or recorded
    inside the steps of a run."""

    def __init__(self, solver: "Solver", points):
        pts = np.ascontiguousarray(points, dtype=np.float64)
        self.solver = solver
        self.n = pts.shape[0]
        self.nfields = solver.nfields
        found = np.zeros(self.n, dtype=np.int32)
        h = ctypes.c_void_p()
        check(lib().dgp_probe_create(solver.h, self.n, _dp(pts), ctypes.byref(h), _ip(found)))
        self.h = h
        self.found = found.astype(bool)

    def eval(self) -> np.ndarray:
        """[n][fields] of the current state (NaN outside the mesh)."""
        out = np.zeros((self.n, self.nfields))
        check(lib().dgp_probe_eval(self.h, _dp(out)))
        return out

    def record(self, every: int, max_samples: int):
        """Sample after every `every`-th step of the following runs (0: stop)."""
        self.max_samples = max_samples
        check(lib().dgp_probe_record(self.h, every, max_samples))

    def samples(self):
        """(times [k], values [k][n][fields]) of the last run."""
        k = ctypes.c_int()
        ms = max(getattr(self, "max_samples", 0), 1)
        t = np.zeros(ms)
        v = np.zeros((ms, self.n, self.nfields))
        check(lib().dgp_probe_samples(self.h, ctypes.byref(k), _dp(t), _dp(v)))
        return t[:k.value].copy(), v[:k.value].copy()

    def close(self):
        if self.h:
            lib().dgp_probe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_device(device: int):
    """CUDA device of the calling thread for the solvers created afterwards."""
    check(lib().dgp_set_device(int(device)))


def line_points(p1, p2, n: int) -> np.ndarray:
    """DGLineSensor's samples: p1 + (p2 - p1) i / (n - 1), i = 0..n-1."""
    p1 = np.asarray(p1, dtype=np.float64)
    p2 = np.asarray(p2, dtype=np.float64)
    return p1[None, :] + (p2 - p1)[None, :] * (np.arange(n, dtype=np.float64) / (n - 1))[:, None]


def first_crossing(values: np.ndarray, field: int, threshold: float) -> int:
    """DGTresholdLineSensor: index of the first sample whose field value lies on
    the other side of `threshold` from the previous sample's (-1: none)."""
    v = values[:, field]
    for i in range(1, len(v)):
        if (v[i] > threshold and v[i - 1] < threshold) or (v[i] < threshold and v[i - 1] > threshold):
            return i
    return -1


def autotune(mesh: "Mesh", law: "Law", order: int, precision: int = FP64, limiter: int = 0,
             iters: int = 10):
    """Time the tile shapes (64/128/256 threads) on this mesh; the fastest is
    used by solvers created afterwards for the same configuration and size.
    Returns (best block, ms per step of each candidate, -1 where not built)."""
    best = ctypes.c_int()
    ms = (ctypes.c_float * 3)()
    check(lib().dgp_autotune(mesh.h, law.h, order, precision, limiter, iters, ctypes.byref(best), ms))
    return best.value, [float(x) for x in ms]


def tune_set(law: int, flux: int, dim: int, order: int, precision: int, cells: int, block: int):
    """Record a tile shape by hand for meshes of `cells` cells (same size bucket)."""
    check(lib().dgp_tune_set(law, flux, dim, order, precision, cells, block))


def autotune_ensemble(meshes, laws, orders, precision: int = FP64, limiter: int = 0, iters: int = 5):
    n = len(meshes)
    mh = (ctypes.c_void_p * n)(*[m.h.value for m in meshes])
    lh = (ctypes.c_void_p * n)(*[l.h.value for l in laws])
    od = np.ascontiguousarray(orders, dtype=np.int32)
    check(lib().dgp_autotune_ensemble(n, mh, lh, _ip(od), precision, limiter, iters))


class Ensemble:
    """Independent instances (mesh, law, order) run batched on one GPU; states
    and results are per instance."""

    def __init__(self, meshes, laws, orders, precision: int = FP64, limiter: int = 0):
        n = len(meshes)
        assert len(laws) == n and len(orders) == n
        self.meshes, self.laws = list(meshes), list(laws)
        mh = (ctypes.c_void_p * n)(*[m.h.value for m in meshes])
        lh = (ctypes.c_void_p * n)(*[l.h.value for l in laws])
        od = np.ascontiguousarray(orders, dtype=np.int32)
        self.h = ctypes.c_void_p()
        check(lib().dgp_ensemble_create(n, mh, lh, _ip(od), precision, limiter, ctypes.byref(self.h)))
        self.n = n
        self.shapes, self.groups = [], []
        for i in range(n):
            m, k, e, g = (ctypes.c_int() for _ in range(4))
            check(lib().dgp_ensemble_info(self.h, i, ctypes.byref(m), ctypes.byref(k), ctypes.byref(e),
                                          ctypes.byref(g)))
            self.shapes.append((e.value, m.value, k.value))
            self.groups.append(g.value)

    def project(self, t: float = 0.0):
        check(lib().dgp_ensemble_project(self.h, t))

    def get_state(self, i: int) -> np.ndarray:
        out = np.zeros(self.shapes[i])
        check(lib().dgp_ensemble_get_state(self.h, i, _dp(out)))
        return out

    def set_state(self, i: int, c: np.ndarray):
        c = np.ascontiguousarray(c, dtype=np.float64).reshape(self.shapes[i])
        check(lib().dgp_ensemble_set_state(self.h, i, _dp(c)))

    def run(self, t0: float, tend: float, cfl: float, max_steps: int = 0):
        """Returns (final times, steps, per-instance device ms, total device ms)."""
        t = np.zeros(self.n)
        steps = np.zeros(self.n, dtype=np.int32)
        ms = np.zeros(self.n)
        tot = ctypes.c_double()
        check(lib().dgp_ensemble_run(self.h, t0, tend, cfl, max_steps, _dp(t), _ip(steps), _dp(ms),
                                     ctypes.byref(tot)))
        return t, steps, ms, tot.value

    def totals(self, i: int) -> np.ndarray:
        out = np.zeros(self.shapes[i][1])
        check(lib().dgp_ensemble_totals(self.h, i, _dp(out)))
        return out

    def l2_error(self, i: int, t: float, field: int = 0) -> float:
        e = ctypes.c_double()
        check(lib().dgp_ensemble_l2_error(self.h, i, t, field, ctypes.byref(e)))
        return e.value

    def launches_per_step(self) -> int:
        n = ctypes.c_int()
        check(lib().dgp_ensemble_launches_per_step(self.h, ctypes.byref(n)))
        return n.value

    def group_block(self, g: int) -> tuple[int, int]:
        """(threads, cells per element-kernel tile) of kernel group g."""
        b, te = ctypes.c_int(), ctypes.c_int()
        check(lib().dgp_ensemble_group_block(self.h, g, ctypes.byref(b), ctypes.byref(te)))
        return b.value, te.value

    def close(self):
        if self.h:
            lib().dgp_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

