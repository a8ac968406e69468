"""Mesh files and per-vertex geometry (host side) against the reference's own
surfaces.py run on the same mesh (tests/golden: a perturbed, decimated
icosphere with obtuse faces and an odd vertex count)."""
import os

import numpy as np
import pytest

from registration_b200 import meshio
from registration_b200 import surfaces as sf


def _mesh(golden):
    return golden["mesh_v"], golden["mesh_f"]


def test_vertex_area_matches_reference(golden):
    v, f = _mesh(golden)
    AV, AF = sf.Surface(FV=[f, v]).computeVertexArea()
    assert AV.shape == golden["mesh_AV"].shape and AF.shape == golden["mesh_AF"].shape
    np.testing.assert_allclose(AF, golden["mesh_AF"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(AV, golden["mesh_AV"], rtol=1e-13, atol=1e-16)
    # the mesh has obtuse faces (both branches are exercised)
    V = v[f]
    x12, x13, x23 = V[:, 1] - V[:, 0], V[:, 2] - V[:, 0], V[:, 2] - V[:, 1]
    obtuse = ((x12 * x13).sum(1) < 0) | ((x12 * x23).sum(1) > 0) | ((x13 * x23).sum(1) < 0)
    assert 0 < obtuse.sum() < len(f)


def test_vertex_normals_and_volume_match_reference(golden):
    v, f = _mesh(golden)
    s = sf.Surface(FV=[f, v])
    np.testing.assert_allclose(s.computeVertexNormals(), golden["mesh_normals"], rtol=1e-13, atol=1e-15)
    assert s.surfVolume() == pytest.approx(float(golden["mesh_volume"]), rel=1e-13)


def test_byu_writer_is_byte_identical_and_reader_matches(golden, tmp_path):
    v, f = _mesh(golden)
    p = str(tmp_path / "m.byu")
    sf.Surface(FV=[f, v]).savebyu(p)
    with open(p) as fh:
        assert fh.read() == str(golden["mesh_byu_text"])
    back = sf.Surface(filename=p)
    np.testing.assert_array_equal(back.vertices, golden["mesh_byu_v"])
    np.testing.assert_array_equal(back.faces, golden["mesh_byu_f"])
    assert back.centers.shape == (len(f), 3)


def test_vtk_writer_is_byte_identical_and_reader_round_trips(golden, tmp_path):
    v, f = _mesh(golden)
    s = sf.Surface(FV=[f, v])
    AV, _ = s.computeVertexArea()
    n = s.computeVertexNormals()
    p = str(tmp_path / "m.vtk")
    s.saveVTK(p, scalars=AV[:, 0], normals=golden["mesh_normals"], vectors=0.5 * golden["mesh_normals"])
    with open(p) as fh:
        assert fh.read() == str(golden["mesh_vtk_text"])
    back = sf.Surface(filename=p)
    np.testing.assert_array_equal(back.faces, f)
    np.testing.assert_allclose(back.vertices, v, rtol=0, atol=5e-7)   # '{0: f}' keeps 6 decimals
    assert n.shape == v.shape


def test_off_reader_matches_reference(golden, tmp_path):
    p = str(tmp_path / "m.off")
    with open(p, "w") as fh:
        fh.write(str(golden["mesh_off_text"]))
    back = sf.Surface(filename=p)
    np.testing.assert_array_equal(back.vertices, golden["mesh_off_v"])
    np.testing.assert_array_equal(back.faces, golden["mesh_off_f"])


def test_obj_reader_and_dispatch(tmp_path):
    v = np.array([[0., 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    p = str(tmp_path / "t.obj")
    with open(p, "w") as fh:
        fh.write("# tetra\n" + "".join("v %.17g %.17g %.17g\n" % tuple(x) for x in v))
        fh.write("f 1 3 2\nf 1/1/1 2/2/2 4/4/4\nf -3 -2 -1\nf 1 4 3 2\n")
    s = sf.Surface(filename=p)
    np.testing.assert_array_equal(s.vertices, v)
    np.testing.assert_array_equal(s.faces, [[0, 2, 1], [0, 1, 3], [1, 2, 3], [0, 3, 2]])
    e = sf.Surface(filename=str(tmp_path / "x.ply"))
    assert e.vertices.size == 0


def test_readers_reject_malformed_files(tmp_path):
    p = str(tmp_path / "q.off")
    with open(p, "w") as fh:
        fh.write("OFF\n4 1 0\n0 0 0\n1 0 0\n1 1 0\n0 1 0\n4 0 1 2 3\n")
    with pytest.raises(ValueError):
        meshio.read_off(p)
    p = str(tmp_path / "t.byu")
    with open(p, "w") as fh:
        fh.write(" 1  3  1  3 0\n1  1\n0 0 0 1 0 0\n")
    with pytest.raises(ValueError):
        meshio.read_byu(p)
    p = str(tmp_path / "b.vtk")
    with open(p, "w") as fh:
        fh.write("# vtk DataFile Version 3.0\nx\nBINARY\nDATASET POLYDATA\n")
    with pytest.raises(ValueError):
        meshio.read_vtk(p)


def test_save_evolution_and_read_multiple(golden, tmp_path):
    v, f = _mesh(golden)
    xt = np.stack([v, 1.1 * v, 1.2 * v])
    base = str(tmp_path / "evo")
    sf.saveEvolution(base, sf.Surface(FV=[f, v]), xt)
    names = sorted(os.listdir(str(tmp_path)))
    assert names == ["evo 0.byu", "evo 1.byu", "evo 2.byu"]   # the reference's '{0: 02d}' names
    got = sf.readMultipleByu(str(tmp_path / "evo*.byu"))
    assert len(got) == 3
    for s in got:
        np.testing.assert_array_equal(s.faces, f)
    assert len(sf.readMultipleByu(str(tmp_path / "evo*.byu"), Nmax=2)) == 2
