#!/usr/bin/env python3
"""Regenerate the golden fixtures of tests/golden/ from DG-Parallel itself.

Runs oracle/_ref/ref_driver -- the reference's own C++ code compiled from its
sources by ``make -C oracle ref`` -- on small seeded meshes and stores, per
case, the mesh file and an .npz with:

* ``conn``   faces as (sorted vertex ids, eL, eR, lfL, lfR, classification id)
* ``geom``   left-outward unit normal and measure per face (same row order)
* ``states`` coefficients [step][cell][field*mode] (file order), step 0 = the
             L2 projection of the initial field, then after each RK3 step
* ``rhs``    assembled right-hand side of the projected state at t = 0
* ``log``    per step: dt, time, residual

(further case tables below store what their comment names)

The reference run uses one worker thread so that stage times are honoured (see
oracle/ref_driver.cc).  Usage: python tests/golden/make_golden.py [case ...]
(the local time stepping cases need ``make -C oracle ref_lts``)
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "dg-parallel_b200"))
from dgp import meshgen  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

# name: (mesh builder, driver arguments, steps)
SQUARE = dict(nx=4, ny=4, seed=1)
VORTEX_BOX = dict(nx=4, ny=4, x0=0.0, x1=10.0, y0=0.0, y1=10.0, seed=2)
PERIODIC_BOX = dict(nx=5, ny=4, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, seed=7, side_tags=(610, 510, 610, 510))
CASES = {
    "scalar_tri_p1": ("tri", SQUARE, ["--case", "gauss", "--order", "1"], 3),
    "scalar_tri_p2": ("tri", SQUARE, ["--case", "gauss", "--order", "2"], 3),
    "scalar_tri_p3": ("tri", SQUARE, ["--case", "gauss", "--order", "3"], 3),
    "scalar_tri_p4": ("tri", SQUARE, ["--case", "gauss", "--order", "4"], 3),
    "euler_godunov_p2": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "exact", "--order", "2"], 3),
    "euler_godunov_p3": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "exact", "--order", "3"], 3),
    "euler_roe_p1": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "roe", "--order", "1"], 3),
    "euler_roe_p3": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "roe", "--order", "3"], 3),
    "euler_roe_p4": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "roe", "--order", "4"], 3),
    "burgers_p2": ("tri", SQUARE, ["--case", "sine", "--order", "2", "--amp", "0.25"], 3),
    "scalar_tet_p2": ("tet", dict(n=2, seed=3), ["--case", "gauss3d", "--order", "2", "--ax", "1",
                                                  "--ay", "0.5", "--az", "0.25", "--cx", "0.5",
                                                  "--cy", "0.5", "--cz", "0.5", "--s", "0.05"], 3),
    "euler3d_p1": ("tet", dict(n=2, seed=3), ["--case", "pulse3d", "--order", "1", "--ax", "1",
                                               "--ay", "0.5", "--az", "0.25", "--cx", "0.5",
                                               "--cy", "0.5", "--cz", "0.5", "--s", "0.05"], 3),
    "euler3d_p2": ("tet", dict(n=2, seed=3), ["--case", "pulse3d", "--order", "2", "--ax", "1",
                                               "--ay", "0.5", "--az", "0.25", "--cx", "0.5",
                                               "--cy", "0.5", "--cz", "0.5", "--s", "0.05"], 3),
    # periodic in x (sides tagged 510) and y (610) on [-1,1]^2
    "scalar_periodic_p2": ("tri", PERIODIC_BOX, ["--case", "gauss", "--order", "2", "--cx", "0.2",
                                                  "--cy", "-0.1", "--s", "0.1"], 4),
    "burgers_periodic_p3": ("tri", PERIODIC_BOX, ["--case", "sine", "--order", "3", "--amp", "0.25"], 4),
    # Maxwell2d (MaxwellLaw.cc) with a TM cavity mode: far field, and the
    # reflection of faces tagged 40000
    "maxwell2d_p1": ("tri", SQUARE, ["--case", "tm2d", "--order", "1"], 3),
    "maxwell2d_p2": ("tri", SQUARE, ["--case", "tm2d", "--order", "2"], 3),
    "maxwell2d_p3": ("tri", SQUARE, ["--case", "tm2d", "--order", "3"], 3),
    "maxwell2d_wall_p2": ("tri", dict(SQUARE, boundary_tag=40000), ["--case", "tm2d", "--order", "2"], 3),
}


# Barth limiter fixtures: the reference's own DGBarthLimiter::limit applied to
# every cell of the state after `steps` steps (ref_driver --barth); stored as
# ``pre`` (the state handed to the limiter, [cell][field*mode]), ``post`` (the
# limited coefficients) and ``slope`` (details->limSlope per cell and field).
BARTH_CASES = {
    "barth_scalar_tri_p1": ("tri", SQUARE, ["--case", "gauss", "--order", "1"], 2),
    "barth_scalar_tri_p2": ("tri", SQUARE, ["--case", "gauss", "--order", "2"], 0),
    "barth_scalar_tri12_p2": ("tri", dict(nx=12, ny=12, seed=1), ["--case", "gauss", "--order", "2",
                                                                   "--s", "0.1"], 2),
    "barth_euler_roe_p2": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "roe", "--order", "2"], 2),
    "barth_scalar_tet_p2": ("tet", dict(n=2, seed=3), ["--case", "gauss3d", "--order", "2", "--ax", "1",
                                                        "--ay", "0.5", "--az", "0.25", "--cx", "0.5",
                                                        "--cy", "0.5", "--cz", "0.5", "--s", "0.05"], 0),
}


# Workload-size fixtures.  ``config1_scalar_p2_32x32``: the scalar advection
# workload as its definition states it -- the unit square cut into a 32x32 grid
# of 2048 jittered triangles (seed 1, +-0.15h), P2, upwind flux, u0 =
# exp(-((x-0.3)^2+(y-0.3)^2)/0.01), a = (1, 0.5), 200 SSP-RK3 steps at CFL 0.1
# (the reference's own 6-point volume rule); stores the states at steps 0 and
# 200, the per-step log, the connectivity and the RHS at t = 0.
# ``l2_euler_roe_p3``: DGAnalysis::densityErrorL2 of the reference after five
# steps of the P3 vortex (``l2`` the total, ``l2_cells`` each cell's squared
# error, ``state`` the final state, ``t`` the final time).
SIZE_CASES = {
    "config1_scalar_p2_32x32": ("tri", dict(nx=32, ny=32, seed=1), ["--case", "gauss", "--order", "2"], 200),
}
L2_CASES = {
    "l2_euler_roe_p3": ("tri", dict(nx=8, ny=8, x0=0.0, x1=10.0, y0=0.0, y1=10.0, seed=2),
                        ["--case", "vortex", "--flux", "roe", "--order", "3"], 5),
}

# The P0 fallback (DGCell::setToZero) as the reference's serial assembly
# applies it (DGAnalysis.cc:392-417): the projected vortex with the listed
# cells' density pushed away from its mean by a|c_0| (ref_driver --p0-rhs;
# cell 34 shares an edge with cell 37).  ``state`` the perturbed state,
# ``after`` the state after the fallback, ``rhs`` the right-hand side,
# ``dropped`` the cells whose modes k >= 1 were zeroed (by the volume
# correction of computeVolumeContribution or by the faces), ``zeroed_by_faces``
# the setToZero calls of the face pass (file order, repeats kept).  The cases
# reach the volume correction alone, the face pass alone, and both.
P0_BOX = dict(nx=10, ny=10, x0=0.0, x1=10.0, y0=0.0, y1=10.0, jitter=0.15, seed=2)
P0_VORTEX = ["--case", "vortex", "--flux", "roe"]
P0_CASES = {
    "p0_euler_roe_p2_volume": ("tri", P0_BOX, P0_VORTEX + ["--order", "2"], [37, 80], 3.0),
    "p0_euler_roe_p1_faces": ("tri", P0_BOX, P0_VORTEX + ["--order", "1"], [37, 34, 120, 80], 0.3),
    "p0_euler_roe_p1_both": ("tri", P0_BOX, P0_VORTEX + ["--order", "1"], [37, 34, 120, 80], 0.4),
    "p0_euler_roe_p3_both": ("tri", P0_BOX, P0_VORTEX + ["--order", "3"], [37, 34, 120, 80], 0.2),
}


def run_p0_case(name, kind, margs, dargs, cells, amp):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "p0")
        cmd = [DRIVER, "--mesh", msh, "--p0-rhs", out, "--p0-cells", ",".join(map(str, cells)),
               "--p0-amp", repr(amp)] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        lines = open(out).read().split("\n")
        E, m, Np, nz = map(int, lines[0].split())
        zeroed = np.array(list(map(int, lines[1].split())), dtype=np.int64)
        rows = np.array([list(map(float, ln.split())) for ln in lines[2:2 + 3 * E]])
    state, after = rows[:E].reshape(E, m, Np), rows[E:2 * E].reshape(E, m, Np)
    dropped = np.nonzero((after != state).any(axis=(1, 2)))[0]
    assert len(dropped) > 0, "no cell became non-physical"
    np.savez_compressed(os.path.join(HERE, name + ".npz"), state=state, after=after,
                        rhs=rows[2 * E:].reshape(E, m, Np), zeroed_by_faces=zeroed, dropped=dropped,
                        cells=np.array(cells), amp=amp, args=np.array(dargs))

# Point sensors (DGPointSensor, DGCell::inCell) after a few steps, at seeded
# points inside the domain and one outside it (ref_driver --probe-out):
# ``points``, ``cell`` (-1 outside), ``values`` [point][field] (NaN outside),
# ``state`` the final state.
def probe_points(kind, seed, n):
    rng = np.random.default_rng(seed)
    if kind == "tri":
        p = np.zeros((n + 1, 3))
        p[:n, :2] = rng.uniform(0.3, 9.7, size=(n, 2))
        p[n, :2] = (12.0, 5.0)
    else:
        p = rng.uniform(0.05, 0.95, size=(n + 1, 3))
        p[n] = (1.5, 0.5, 0.5)
    return p


PROBE_CASES = {
    "probes_euler_roe_p2": ("tri", dict(nx=6, ny=6, x0=0.0, x1=10.0, y0=0.0, y1=10.0, seed=2),
                            ["--case", "vortex", "--flux", "roe", "--order", "2"], 3, 16),
    "probes_scalar_tet_p2": ("tet", dict(n=2, seed=3),
                             ["--case", "gauss3d", "--order", "2", "--ax", "1", "--ay", "0.5", "--az", "0.25",
                              "--cx", "0.5", "--cy", "0.5", "--cz", "0.5", "--s", "0.05"], 3, 12),
}


def run_probe_case(name, kind, margs, dargs, steps, npts):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    pts = probe_points(kind, 11, npts)
    with tempfile.TemporaryDirectory() as td:
        out, state = os.path.join(td, "p"), os.path.join(td, "s")
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--state", state,
               "--every", str(steps), "--probe-out", out,
               "--probe-pts", ";".join(",".join(repr(float(v)) for v in p) for p in pts)] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        rows = [list(map(float, ln.split())) for ln in open(out) if ln.strip()]
        blocks = open(state).read().split("step ")[1:]
        st = np.array([list(map(float, ln.split())) for ln in blocks[-1].split("\n")[1:] if ln.strip()])
    m = max(len(r) for r in rows) - 2
    cell = np.array([int(r[1]) for r in rows], dtype=np.int64)
    vals = np.full((len(rows), m), np.nan)
    for i, r in enumerate(rows):
        if r[1] >= 0:
            vals[i] = r[2:]
    assert (cell >= 0).sum() == npts and cell[-1] == -1
    np.savez_compressed(os.path.join(HERE, name + ".npz"), points=pts, cell=cell, values=vals, state=st,
                        args=np.array(dargs), steps=steps)

# The DGError.cc error norms summed as DGAnalysis does (DGPref.cc:249-381)
# after a few steps (ref_driver --norms): ``t``, ``state`` and one entry per
# norm (ExactError, LinfError, densityErrorL2; for the vortex also
# PressureError, entropyErrorL1, pressureErrorL2, entropyErrorL2).
NORM_CASES = {
    "norms_euler_roe_p3": ("tri", dict(nx=8, ny=8, x0=0.0, x1=10.0, y0=0.0, y1=10.0, seed=2),
                           ["--case", "vortex", "--flux", "roe", "--order", "3"], 5),
    "norms_scalar_p2": ("tri", SQUARE, ["--case", "gauss", "--order", "2"], 5),
}


def run_norm_case(name, kind, margs, dargs, steps):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        state, nf = os.path.join(td, "s"), os.path.join(td, "n")
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--state", state,
               "--every", str(steps), "--norms", nf] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        blocks = open(state).read().split("step ")[1:]
        st = np.array([list(map(float, ln.split())) for ln in blocks[-1].split("\n")[1:] if ln.strip()])
        vals = {ln.split()[0]: float(ln.split()[1]) for ln in open(nf) if ln.strip()}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), state=st, args=np.array(dargs), steps=steps, **vals)


def run_size_case(name, kind, margs, dargs, steps):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        conn, rhs, state, log = (os.path.join(td, f) for f in ("c", "r", "s", "l"))
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--conn", conn, "--rhs", rhs,
               "--state", state, "--every", str(steps), "--log", log] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        c = np.loadtxt(conn)
        nf = 5 + (2 if kind == "tri" else 3)
        r = np.loadtxt(rhs, skiprows=1)
        blocks = open(state).read().split("step ")[1:]
        states = np.array([[list(map(float, ln.split())) for ln in b.split("\n")[1:] if ln.strip()]
                           for b in blocks])
        lg = np.loadtxt(log, ndmin=2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), conn=c[:, :nf].astype(np.int64),
                        geom=c[:, nf:], states=states, rhs=np.atleast_2d(r), log=lg,
                        args=np.array(dargs), steps=steps)


def run_l2_case(name, kind, margs, dargs, steps):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        state, l2 = os.path.join(td, "s"), os.path.join(td, "e")
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--state", state,
               "--every", str(steps), "--l2", l2] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        blocks = open(state).read().split("step ")[1:]
        st = np.array([list(map(float, ln.split())) for ln in blocks[-1].split("\n")[1:] if ln.strip()])
        t, total = map(float, open(l2).readline().split())
        cells = np.loadtxt(l2, skiprows=1)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), state=st, t=t, l2=total, l2_cells=cells,
                        args=np.array(dargs), steps=steps)


def run_barth_case(name, kind, margs, dargs, steps):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        state, barth = os.path.join(td, "s"), os.path.join(td, "b")
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--state", state,
               "--every", str(max(steps, 1)), "--barth", barth] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        blocks = open(state).read().split("step ")[1:]
        pre = np.array([list(map(float, ln.split())) for ln in blocks[-1].split("\n")[1:] if ln.strip()])
        E, m, Np = map(int, open(barth).readline().split())
        b = np.loadtxt(barth, skiprows=1, ndmin=2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), pre=pre, post=b[:, :m * Np],
                        slope=b[:, m * Np:], args=np.array(dargs), steps=steps)


# Checkpoint fixture: the data stream of DGAnalysis::write after `steps` steps
# (ref_driver --ckpt-out, the reference's own writeMEntity + DGCell::write at
# 16 digits), stored as <name>.dat, with the same state at 17 digits in
# <name>.npz (``state`` [cell][field*mode], ``t``, ``steps``).
CKPT_CASES = {
    "ckpt_euler_roe_p2": ("tri", VORTEX_BOX, ["--case", "vortex", "--flux", "roe", "--order", "2"], 2),
}


def run_ckpt_case(name, kind, margs, dargs, steps):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    dat = os.path.join(HERE, name + ".dat")
    with tempfile.TemporaryDirectory() as td:
        state, log = os.path.join(td, "s"), os.path.join(td, "l")
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--state", state,
               "--every", str(steps), "--log", log, "--ckpt-out", dat] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        blocks = open(state).read().split("step ")[1:]
        st = np.array([list(map(float, ln.split())) for ln in blocks[-1].split("\n")[1:] if ln.strip()])
        lg = np.loadtxt(log, ndmin=2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), state=st, t=lg[-1, 2], steps=steps,
                        args=np.array(dargs))


# Local time stepping fixtures: oracle/_ref/ref_driver_lts (the reference's
# RungeKuttaTVD2adaptive with the range helpers TimeIntegrator::assembleVolume /
# assembleBoundary(begin, end, t) given the bodies of their whole-mesh versions,
# and the size bins of DGAnalysis::sortCellsBySize) on geometrically graded
# meshes, the mode-5 step (CFL minimum times 2^(bins-1)); stored as ``bins``
# (bin, role per cell), ``states`` (initial + every step) and ``log``.
LTS_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver_lts")
GRADED = dict(nx=16, ny=16, ratio=1.15)
GRADED_BOX = dict(nx=14, ny=14, ratio=1.15, x0=0.0, x1=10.0, y0=0.0, y1=10.0)
LTS_CASES = {
    "lts_scalar_graded_p2": ("graded", GRADED, ["--case", "gauss", "--order", "2"], 3),
    "lts_euler_roe_graded_p2": ("graded", GRADED_BOX, ["--case", "vortex", "--flux", "roe", "--order", "2"], 2),
    "lts_scalar_tet_graded_p2": ("tet_graded", dict(n=6, ratio=1.35),
                                 ["--case", "gauss3d", "--order", "2", "--ax", "1", "--ay", "0.5", "--az", "0.25",
                                  "--cx", "0.5", "--cy", "0.5", "--cz", "0.5", "--s", "0.05"], 2),
}


def run_lts_case(name, kind, margs, dargs, steps):
    mesh = meshgen.tri_graded(**margs) if kind == "graded" else meshgen.tet_graded(**margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        bins, state, log = (os.path.join(td, f) for f in ("b", "s", "l"))
        cmd = [LTS_DRIVER, "--mesh", msh, "--lts", "1", "--steps", str(steps), "--cfl", "0.1",
               "--bins", bins, "--state", state, "--log", log] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        b = np.loadtxt(bins, skiprows=1, dtype=np.int64, ndmin=2)
        nb = int(open(bins).readline().split()[1])
        blocks = open(state).read().split("step ")[1:]
        states = np.array([[list(map(float, ln.split())) for ln in blk.split("\n")[1:] if ln.strip()]
                           for blk in blocks])
        lg = np.loadtxt(log, ndmin=2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), bins=b, nbins=nb, states=states, log=lg,
                        args=np.array(dargs), steps=steps)


def build_mesh(kind, args):
    return meshgen.tri_square(**args) if kind == "tri" else meshgen.tet_cube(**args)


def run_case(name, kind, margs, dargs, steps):
    mesh = build_mesh(kind, margs)
    msh = os.path.join(HERE, name + ".msh")
    meshgen.write_msh_v1(mesh, msh)
    with tempfile.TemporaryDirectory() as td:
        conn, rhs, state, log = (os.path.join(td, f) for f in ("c", "r", "s", "l"))
        cmd = [DRIVER, "--mesh", msh, "--steps", str(steps), "--cfl", "0.1", "--conn", conn,
               "--rhs", rhs, "--state", state, "--log", log] + dargs
        subprocess.run(cmd, check=True, capture_output=True)
        c = np.loadtxt(conn)
        nf = 5 + (2 if kind == "tri" else 3)
        r = np.loadtxt(rhs, skiprows=1)
        blocks = open(state).read().split("step ")[1:]
        states = np.array([[list(map(float, ln.split())) for ln in b.split("\n")[1:] if ln.strip()]
                           for b in blocks])
        lg = np.loadtxt(log, ndmin=2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), conn=c[:, :nf].astype(np.int64),
                        geom=c[:, nf:], states=states, rhs=np.atleast_2d(r), log=lg,
                        args=np.array(dargs), steps=steps)


def main():
    if not os.path.exists(DRIVER):
        sys.exit("build the reference first: make -C oracle ref")
    only = set(sys.argv[1:])  # case names (default: all)
    for name, (kind, margs, dargs, steps) in CASES.items():
        if only and name not in only:
            continue
        run_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps) in LTS_CASES.items():
        if only and name not in only:
            continue
        run_lts_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps) in CKPT_CASES.items():
        if only and name not in only:
            continue
        run_ckpt_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps) in BARTH_CASES.items():
        if only and name not in only:
            continue
        run_barth_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps) in SIZE_CASES.items():
        if only and name not in only:
            continue
        run_size_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps) in L2_CASES.items():
        if only and name not in only:
            continue
        run_l2_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps) in NORM_CASES.items():
        if only and name not in only:
            continue
        run_norm_case(name, kind, margs, dargs, steps)
        print("wrote", name)
    for name, (kind, margs, dargs, steps, npts) in PROBE_CASES.items():
        if only and name not in only:
            continue
        run_probe_case(name, kind, margs, dargs, steps, npts)
        print("wrote", name)
    for name, (kind, margs, dargs, cells, amp) in P0_CASES.items():
        if only and name not in only:
            continue
        run_p0_case(name, kind, margs, dargs, cells, amp)
        print("wrote", name)


if __name__ == "__main__":
    main()
