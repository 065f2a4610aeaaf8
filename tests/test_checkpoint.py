"""Checkpoints in the data format of DGAnalysis::write / read (DGPref.cc:712-766).

The fixture ckpt_euler_roe_p2.dat was written by the reference itself
(oracle/ref_driver --ckpt-out: mMesh::writeMEntity + DGCell::write, 16 digits,
cells in the reference's entity order, no geometric order after the type);
ckpt_euler_roe_p2.npz holds the same state at 17 digits in file order.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import dgp
from cases import GOLDEN, ROOT, VORTEX

NAME = "ckpt_euler_roe_p2"
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def _msh_cells(path):
    """file-order cell vertex ids of a Gmsh v1 triangle mesh (type 2)"""
    lines = open(path).read().split("$ELM")[1].split("$ENDELM")[0].split("\n")[2:]
    cells = []
    for ln in lines:
        t = ln.split()
        if len(t) >= 8 and t[1] == "2":
            cells.append(tuple(sorted(int(v) for v in t[5:8])))
    return cells


def _parse_reference_data(path, m, np_):
    tok = open(path).read().split()
    t, it, dim, ncell, nface = float(tok[0]), int(tok[1]), int(tok[2]), int(tok[3]), int(tok[4])
    p, cells = 5, {}
    for _ in range(ncell):
        typ = int(tok[p])
        assert typ == 2
        vids = tuple(sorted(int(v) for v in tok[p + 1:p + 4]))
        order = int(tok[p + 4])
        vals = np.array([float(v) for v in tok[p + 5:p + 5 + m * np_]])
        cells[vids] = (order, vals)
        p += 5 + m * np_
    return t, it, cells


def test_reference_checkpoint_fixture_matches_its_state():
    d = np.load(os.path.join(GOLDEN, NAME + ".npz"))
    t, it, cells = _parse_reference_data(os.path.join(GOLDEN, NAME + ".dat"), 4, 6)
    assert it == 2 and abs(t - float(d["t"])) <= 1e-15 * float(d["t"])
    order = _msh_cells(os.path.join(GOLDEN, NAME + ".msh"))
    st = np.array([cells[c][1] for c in order])
    assert all(cells[c][0] == 2 for c in order)
    assert np.abs(st - d["state"]).max() <= 1e-15 * np.abs(d["state"]).max()


def _solver():
    mesh = dgp.Mesh.from_msh(os.path.join(GOLDEN, NAME + ".msh"))
    return dgp.Solver(mesh, dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX), 2, dgp.FP64)


@pytest.mark.gpu
def test_gpu_reads_the_reference_checkpoint():
    d = np.load(os.path.join(GOLDEN, NAME + ".npz"))
    s = _solver()
    t, it = s.read_checkpoint(os.path.join(GOLDEN, NAME + ".dat"))
    assert it == 2 and abs(t - float(d["t"])) <= 1e-15 * float(d["t"])
    st = s.get_state().reshape(d["state"].shape)
    assert np.abs(st - d["state"]).max() <= 1e-15 * np.abs(d["state"]).max()
    # the traces follow the loaded state: stepping from it matches a state set
    # from the host
    s2 = _solver()
    s2.set_state(s.get_state())
    assert np.array_equal(s.rhs(t), s2.rhs(t))
    s.close()
    s2.close()


@pytest.mark.gpu
def test_gpu_checkpoint_round_trip_and_reference_reader():
    s = _solver()
    s.run(0.0, 0.0, 0.1, 3)
    u = s.get_state()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "c.dat")
        s.write_checkpoint(path, 0.125, 3)
        s2 = _solver()
        t, it = s2.read_checkpoint(path)
        assert (t, it) == (0.125, 3)
        assert np.array_equal(s2.get_state(), u)
        s2.close()
        if os.path.exists(REF_DRIVER):
            # DG-Parallel's own reader (mMesh::readMEntity + DGCell::read) loads it
            out = os.path.join(td, "s")
            subprocess.run([REF_DRIVER, "--mesh", os.path.join(GOLDEN, NAME + ".msh"), "--case", "vortex",
                            "--flux", "roe", "--order", "2", "--steps", "0", "--ckpt-in", path,
                            "--state", out], check=True, capture_output=True)
            blk = open(out).read().split("step ")[1]
            ref = np.array([list(map(float, ln.split())) for ln in blk.split("\n")[1:] if ln.strip()])
            assert np.array_equal(ref, u.reshape(ref.shape))
    s.close()
