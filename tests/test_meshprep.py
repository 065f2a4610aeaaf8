"""Face matching on the GPU (dgp_mesh_*_ex with gpu_faces): the same faces,
sides, local faces, orientations, classification ids, normals and measures as
the host matching (which the reference connectivity fixtures pin), so solvers
built on either mesh step identically."""
import os
import time

import numpy as np
import pytest

import dgp
from dgp import meshgen
from cases import GOLDEN_CASES, VORTEX, golden


def _by_face(mesh):
    conn = mesh.connectivity()
    geo = mesh.face_geometry()
    return {tuple(r): g for r, g in zip(conn, geo)}


def _same(a, b):
    fa, fb = _by_face(a), _by_face(b)
    assert set(fa) == set(fb)
    for k, g in fa.items():
        assert np.array_equal(g, fb[k]), k


def test_gpu_faces_request_without_device_matches_host():
    # without a device the request falls back to the host matching
    msh, _ = golden("scalar_tri_p2")
    _same(dgp.Mesh.from_msh(msh, gpu_faces=True), dgp.Mesh.from_msh(msh))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_gpu_face_matching_equals_host_on_fixtures(name):
    msh, _ = golden(name)
    _same(dgp.Mesh.from_msh(msh, gpu_faces=True), dgp.Mesh.from_msh(msh))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tri", "tet"])
def test_gpu_face_matching_equals_host_on_larger_meshes(kind):
    if kind == "tri":
        m = meshgen.tri_square(96, 80, 0.0, 3.0, 0.0, 2.0, jitter=0.2, seed=5)
    else:
        m = meshgen.tet_cube(10, 0.0, 1.0, jitter=0.1, seed=4)
    dim = 2 if kind == "tri" else 3
    a = dgp.Mesh.from_arrays(dim, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags, gpu_faces=True)
    b = dgp.Mesh.from_arrays(dim, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags)
    _same(a, b)


@pytest.mark.gpu
def test_gpu_matched_mesh_steps_identically(tmp_path):
    m = meshgen.tri_square(24, 24, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, VORTEX)
    out = []
    for gpu in (True, False):
        mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, 100, m.bfaces, m.btags, gpu_faces=gpu)
        s = dgp.Solver(mesh, law, 2, dgp.FP64)
        s.run(0.0, 0.0, 0.1, 5)
        out.append(s.get_state())
        s.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.gpu
def test_gpu_face_matching_periodic_box():
    m = meshgen.tri_square(9, 7, -1.0, 1.0, -1.0, 1.0, jitter=0.1, seed=7, side_tags=(610, 510, 610, 510))
    a = dgp.Mesh.from_arrays(2, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags, gpu_faces=True)
    b = dgp.Mesh.from_arrays(2, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags)
    _same(a, b)
    law = dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS,
                  dgp.law_params(velocity=(1.0, 0.5, 0.0), center=(0.2, -0.1, 0.0), width=0.1))
    st = []
    for mesh in (a, b):
        s = dgp.Solver(mesh, law, 2, dgp.FP64)
        s.run(0.0, 0.0, 0.1, 10)
        st.append(s.get_state())
        s.close()
    assert np.array_equal(st[0], st[1])
