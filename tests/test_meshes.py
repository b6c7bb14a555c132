"""Mesh generators and the reference's text mesh format (ReadMeshFromFile.hpp)."""
import numpy as np
import pytest

from baemm_b200 import meshes


@pytest.mark.parametrize("level,nv,nt", [(0, 12, 20), (1, 42, 80), (3, 642, 1280), (5, 10242, 20480)])
def test_icosphere_counts(level, nv, nt):
    c, t = meshes.icosphere(level)
    assert c.shape == (nv, 3) and t.shape == (nt, 3)
    assert np.allclose(np.linalg.norm(c, axis=1), 1.0)
    cen = c[t].mean(axis=1)
    n = np.cross(c[t[:, 1]] - c[t[:, 0]], c[t[:, 2]] - c[t[:, 0]])
    assert np.all((n * cen).sum(axis=1) > 0)   # outward


def test_torus_counts_and_orientation():
    c, t = meshes.torus(1.0, 0.4, 160, 480)
    assert c.shape == (76800, 3) and t.shape == (153600, 3)
    assert c.shape[0] - t.shape[0] // 2 * 3 + t.shape[0] == 0 or True
    # Euler characteristic V - E + F = 0 for a torus (E = 3F/2)
    assert c.shape[0] - 3 * t.shape[0] // 2 + t.shape[0] == 0
    p = c[t]
    area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1).sum()
    assert abs(area - 4 * np.pi ** 2 * 1.0 * 0.4) / (4 * np.pi ** 2 * 0.4) < 1e-3


def test_text_format_roundtrip(tmp_path):
    c, t = meshes.icosphere(1)
    p = tmp_path / "m.txt"
    meshes.write_mesh_txt(p, c, t)
    head = p.read_text().split()[:8]
    assert head == ["dom_dim", "2", "amb_dim", "3", "vertex_count", "42", "simplex_count", "80"]
    c2, t2 = meshes.read_mesh_txt(p)
    assert np.array_equal(t, t2) and np.allclose(c, c2)


def test_text_format_rejects_bad_header(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("dim 2\n")
    with pytest.raises(ValueError):
        meshes.read_mesh_txt(p)


def test_fibonacci_and_sh_perturbation():
    d = meshes.fibonacci_sphere(256)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0)
    assert np.abs(d.mean(axis=0)).max() < 1e-2
    c, t = meshes.sh_perturbed_sphere(3, 8, 0.1, seed=0)
    r = np.linalg.norm(c, axis=1)
    assert abs(np.abs(r - 1).max() - 0.1) < 1e-9


def test_points_off_torus_keep_their_distance():
    p = meshes.points_off_torus(5000, 1.0, 0.4, min_dist=0.05, seed=3)
    assert p.shape == (5000, 3)
    d = np.abs(np.hypot(np.hypot(p[:, 0], p[:, 1]) - 1.0, p[:, 2]) - 0.4)
    assert d.min() >= 0.05
    assert np.all(np.abs(p[:, 2]) <= 0.6) and np.all(np.abs(p[:, :2]) <= 1.6)
    inside = np.hypot(np.hypot(p[:, 0], p[:, 1]) - 1.0, p[:, 2]) < 0.4
    assert 0.1 < inside.mean() < 0.4                      # both sides of the surface
    assert np.array_equal(p, meshes.points_off_torus(5000, 1.0, 0.4, min_dist=0.05, seed=3))


@pytest.mark.parametrize("binary", [True, False])
def test_stl_round_trip_merges_vertices(tmp_path, binary):
    c, t = meshes.icosphere(2)
    p = tmp_path / "s.stl"
    meshes.write_mesh_stl(p, c, t, binary=binary)
    c2, t2 = meshes.read_mesh_stl(p)
    assert c2.shape == c.shape and t2.shape == t.shape        # shared corners merged back to 162 vertices
    assert np.array_equal(c2[t2], c[t].astype(np.float32).astype(np.float64))   # same triangles, same orientation
    assert np.all(np.diff(c2[:, 0]) >= 0)                     # lexicographic vertex order


def test_stl_ascii_with_two_solids(tmp_path):
    c, t = meshes.icosphere(1)
    half = t.shape[0] // 2
    a, b = tmp_path / "a.stl", tmp_path / "b.stl"
    meshes.write_mesh_stl(a, c, t[:half], binary=False, name="first")
    meshes.write_mesh_stl(b, c, t[half:], binary=False, name="second")
    p = tmp_path / "ab.stl"
    p.write_text(a.read_text() + b.read_text())
    c2, t2 = meshes.read_mesh_stl(p)
    assert c2.shape == c.shape and t2.shape == t.shape
    assert np.array_equal(c2[t2], c[t].astype(np.float32).astype(np.float64))


def test_stl_rejects_other_files(tmp_path):
    p = tmp_path / "bad.stl"
    p.write_bytes(b"not a mesh at all")
    with pytest.raises(ValueError):
        meshes.read_mesh_stl(p)


@pytest.fixture(scope="module")
def mesh_reader_exe(tmp_path_factory):
    import os
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path_factory.mktemp("cpp") / "mesh_reader"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
                        os.path.join(root, "tests", "cpp", "mesh_reader.cpp"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


def _cpp_read(exe, kind, path):
    import subprocess
    r = subprocess.run([exe, kind, str(path)], capture_output=True, text=True)
    if r.returncode != 0:
        return None
    lines = r.stdout.split("\n")
    nv, nt = (int(x) for x in lines[0].split())
    c = np.array([[float(x) for x in ln.split()] for ln in lines[1:1 + nv]])
    t = np.array([[int(x) for x in ln.split()] for ln in lines[1 + nv:1 + nv + nt]], dtype=np.int64)
    return c, t


@pytest.mark.parametrize("binary", [True, False])
def test_cpp_stl_reader_matches_python(tmp_path, mesh_reader_exe, binary):
    c, t = meshes.torus(1.0, 0.4, 12, 20)
    p = tmp_path / "t.stl"
    meshes.write_mesh_stl(p, c, t, binary=binary)
    cp, tp = meshes.read_mesh_stl(p)
    cc, tc = _cpp_read(mesh_reader_exe, "stl", p)
    assert np.array_equal(cp, cc) and np.array_equal(tp, tc)


def test_cpp_text_reader_matches_python(tmp_path, mesh_reader_exe):
    c, t = meshes.icosphere(2)
    p = tmp_path / "s.txt"
    meshes.write_mesh_txt(p, c, t)
    cp, tp = meshes.read_mesh_txt(p)
    cc, tc = _cpp_read(mesh_reader_exe, "txt", p)
    assert np.array_equal(cp, cc) and np.array_equal(tp, tc)
    bad = tmp_path / "bad.txt"
    bad.write_text("dom_dim 2\namb_dim 3\nvertex_count 4\nsimplex_count 1\n0 0 0\n")
    assert _cpp_read(mesh_reader_exe, "txt", bad) is None


def test_reference_meshes_read_the_same_in_python_and_cpp(mesh_reader_exe):
    """The reference's own mesh files (Meshes/*.txt of the reference tree, read
    where that tree is present): both readers agree, and the unit spheres have
    their vertices on the sphere."""
    import os

    from oracle import oracle as O
    ref = O.reference_root()
    if ref is None or not os.path.isdir(os.path.join(ref, "Meshes")):
        pytest.skip("reference tree not present (set BAEMM_REFERENCE or build oracle/_ref here)")
    d = os.path.join(ref, "Meshes")
    for name in ("Sphere_00001280T.txt", "TorusMesh_00002400T.txt", "Spot_00005856T.txt"):
        p = os.path.join(d, name)
        cp, tp = meshes.read_mesh_txt(p)
        cc, tc = _cpp_read(mesh_reader_exe, "txt", p)
        assert np.array_equal(cp, cc) and np.array_equal(tp, tc)
        assert tp.shape[0] == int(name.split("_")[1][:-5])
        if name.startswith("Sphere"):
            assert np.allclose(np.linalg.norm(cp, axis=1), 1.0, atol=1e-6)
