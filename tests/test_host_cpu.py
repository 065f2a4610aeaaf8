"""CPU checks of the product library: it loads, exports every entry point of
include/dgp.h, and its mesh import / connectivity (host code, no GPU needed)
reproduce DG-Parallel's face table exactly."""
import ctypes
import os
import re

import numpy as np
import pytest

import dgp
from cases import GOLDEN_CASES, ROOT, golden

HEADER = os.path.join(ROOT, "include", "dgp.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(dgp_\w+)\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = dgp.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.dgp_version() == 1


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_connectivity_matches_reference(name):
    msh, g = golden(name)
    m = dgp.Mesh.from_msh(msh)
    conn = m.connectivity()
    assert conn.shape[0] == g["conn"].shape[0]
    assert set(map(tuple, conn)) == set(map(tuple, g["conn"].astype(np.int32)))
    # unit normals (outward from the left cell) and face measures
    geo = m.face_geometry()
    ref = {tuple(r): gg for r, gg in zip(g["conn"].astype(np.int32), g["geom"])}
    for row, gg in zip(conn, geo):
        r = ref[tuple(row)]
        assert np.abs(gg[:3] - r[:3]).max() < 1e-14
        assert abs(gg[3] - r[3]) < 1e-13 * r[3]


def test_mesh_from_arrays_equals_file(tmp_path):
    from dgp import meshgen
    mesh = meshgen.tri_square(5, 3, seed=11)
    path = str(tmp_path / "m.msh")
    meshgen.write_msh_v1(mesh, path)
    a = dgp.Mesh.from_msh(path).connectivity()
    b = dgp.Mesh.from_arrays(2, mesh.vertices, mesh.cells, 100, mesh.bfaces, mesh.btags).connectivity()
    assert set(map(tuple, a)) == set(map(tuple, b))


def test_mesh_import_errors(tmp_path):
    with pytest.raises(dgp.DGPError) as e:
        dgp.Mesh.from_msh(str(tmp_path / "missing.msh"))
    assert e.value.code == -2
    bad = tmp_path / "trunc.msh"
    bad.write_text("$NOD\n3\n1 0 0 0\n2 1 0 0\n")
    with pytest.raises(dgp.DGPError) as e:
        dgp.Mesh.from_msh(str(bad))
    assert e.value.code == -2
    quad = tmp_path / "quad.msh"
    quad.write_text("$NOD\n4\n1 0 0 0\n2 1 0 0\n3 1 1 0\n4 0 1 0\n$ENDNOD\n$ELM\n1\n1 3 100 100 4 1 2 3 4\n$ENDELM\n")
    with pytest.raises(dgp.DGPError) as e:
        dgp.Mesh.from_msh(str(quad))
    assert e.value.code == -3
    with pytest.raises(dgp.DGPError) as e:
        dgp.Mesh.from_arrays(2, np.zeros((3, 3)), np.array([[0, 1, 2]]))
    assert e.value.code == -1  # degenerate cell


def test_tet_mesh_faces_and_orientation():
    from dgp import meshgen
    mesh = meshgen.tet_cube(3, seed=5)
    m = dgp.Mesh.from_arrays(3, mesh.vertices, mesh.cells, 100, mesh.bfaces, mesh.btags)
    conn = m.connectivity()
    n = 3
    nb = int((conn[:, n + 1] < 0).sum())
    assert nb == 6 * 2 * 3 * 3  # two triangles per boundary square
    assert 4 * m.ncells == 2 * (m.nfaces - nb) + nb
    # left-outward normals point away from the left cell centroid
    geo = m.face_geometry()
    cells = mesh.cells
    v = mesh.vertices
    ids = {vid: i for i, vid in enumerate(range(1, len(v) + 1))}
    for row, gg in zip(conn[:50], geo[:50]):
        fc = np.mean([v[ids[x]] for x in row[:3]], axis=0)
        cc = v[cells[row[n]]].mean(axis=0)
        assert np.dot(gg[:3], fc - cc) > 0


def test_law_boundary_settings_are_checked():
    """dgp_law_set_bc (no GPU needed): periodic ids are not boundary
    conditions, the scalar laws have no wall, at most DGP_MAX_BC ids a law."""
    import dgp
    e = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, dgp.law_params())
    e.set_bc(1, dgp.BC_WALL)
    e.set_bc(1, dgp.BC_FARFIELD)  # a second setting of the same id replaces the first
    with pytest.raises(dgp.DGPError) as ei:
        e.set_bc(510, dgp.BC_WALL)
    assert ei.value.code == -1
    with pytest.raises(dgp.DGPError) as ei:
        e.set_bc(2, 7)
    assert ei.value.code == -1
    for bid in range(2, 9):
        e.set_bc(bid, dgp.BC_WALL)
    with pytest.raises(dgp.DGPError) as ei:
        e.set_bc(99, dgp.BC_WALL)
    assert ei.value.code == -1
    s = dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS, dgp.law_params())
    with pytest.raises(dgp.DGPError) as ei:
        s.set_bc(1, dgp.BC_WALL)
    assert ei.value.code == -3
    s.set_bc(1, dgp.BC_FARFIELD)
