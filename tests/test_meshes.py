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
