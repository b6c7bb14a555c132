"""Mesh and direction generators, and the reference's text mesh format.

Host-side data preparation only (numpy); nothing here computes operators.

* ``read_mesh_txt`` / ``write_mesh_txt`` follow the text format read by
  ReadMeshFromFile.hpp:3-102 (``dom_dim``, ``amb_dim``, ``vertex_count``,
  ``simplex_count`` headers, then vertex rows and 0-based simplex rows).
* ``read_mesh_stl`` / ``write_mesh_stl`` read and write STL (ASCII or binary)
  for ReadMeshFromSTL.hpp:5-44, with the vertex merging of the stl_reader
  library the reference calls (restated in include/BAEMM_Meshes.hpp).
* ``icosphere`` builds the unit sphere from an icosahedron subdivided ``level``
  times and projected to radius 1 (level 3: 642 vertices / 1280 triangles).
* ``torus`` builds the parametric torus of the large-block apply workload.
* ``fibonacci_sphere`` gives quasi-uniform unit directions.
* ``sh_perturbed_sphere`` applies a radial spherical-harmonic perturbation.
"""
from __future__ import annotations

import functools
import math
import os

import numpy as np

__all__ = [
    "read_mesh_txt",
    "write_mesh_txt",
    "read_mesh_stl",
    "write_mesh_stl",
    "points_off_torus",
    "icosphere",
    "torus",
    "fibonacci_sphere",
    "real_sph_harm_sum",
    "sh_perturbed_sphere",
]


def read_mesh_txt(path: str | os.PathLike):
    """Read a mesh in the format of ReadMeshFromFile.hpp:30-97.

    Returns ``(coords, simplices)`` as float64 (vertex_count x amb_dim) and
    int64 (simplex_count x (dom_dim+1)) arrays.  Raises ``ValueError`` on a
    malformed header (the reference prints an error and returns false).
    """
    with open(path, "r") as f:
        tokens = f.read().split()
    hdr = {}
    pos = 0
    for key in ("dom_dim", "amb_dim", "vertex_count", "simplex_count"):
        if pos + 1 >= len(tokens) or tokens[pos] != key:
            raise ValueError(f"read_mesh_txt: invalid file {path}: expected '{key}'")
        hdr[key] = int(tokens[pos + 1])
        pos += 2
    nv, amb = hdr["vertex_count"], hdr["amb_dim"]
    ns, ss = hdr["simplex_count"], hdr["dom_dim"] + 1
    need = nv * amb + ns * ss
    if len(tokens) - pos < need:
        raise ValueError(f"read_mesh_txt: file {path} is truncated")
    coords = np.array(tokens[pos:pos + nv * amb], dtype=np.float64).reshape(nv, amb)
    pos += nv * amb
    simp = np.array(tokens[pos:pos + ns * ss], dtype=np.int64).reshape(ns, ss)
    return coords, simp


def write_mesh_txt(path: str | os.PathLike, coords: np.ndarray, simplices: np.ndarray) -> None:
    coords = np.asarray(coords, dtype=np.float64)
    simplices = np.asarray(simplices, dtype=np.int64)
    with open(path, "w") as f:
        f.write(f"dom_dim {simplices.shape[1] - 1}\n")
        f.write(f"amb_dim {coords.shape[1]}\n")
        f.write(f"vertex_count {coords.shape[0]}\n")
        f.write(f"simplex_count {simplices.shape[0]}\n")
        for row in coords:
            f.write(" ".join(repr(float(x)) for x in row) + "\n")
        for row in simplices:
            f.write(" ".join(str(int(x)) for x in row) + "\n")


def read_mesh_stl(path: str | os.PathLike):
    """Read an STL file (ASCII or binary) as ``(coords, triangles)``, float64
    n x 3 and int64 m x 3 (ReadMeshFromSTL.hpp:5-44).

    Vertices with bit-identical float32 coordinates are merged and numbered in
    lexicographic (x, y, z) order; triangles keep their file order.  Raises
    ``ValueError`` on a file that is neither form (the reference prints the
    reader's exception and returns false).
    """
    data = open(path, "rb").read()
    raw = None
    if len(data) >= 84:
        count = int(np.frombuffer(data[80:84], dtype="<u4")[0])
        if len(data) == 84 + 50 * count:
            rec = np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("attr", "<u2")])
            raw = np.frombuffer(data, dtype=rec, count=count, offset=84)["v"].reshape(-1, 3)
    if raw is None:
        tokens = data.decode("ascii", errors="replace").split()
        if not tokens or tokens[0] != "solid":
            raise ValueError(f"read_mesh_stl: {path} is neither binary STL nor ASCII STL")
        vals = []
        for k, t in enumerate(tokens):
            if t == "vertex":
                if k + 3 >= len(tokens):
                    raise ValueError(f"read_mesh_stl: {path}: malformed vertex")
                vals.extend(tokens[k + 1:k + 4])
        raw = np.array(vals, dtype=np.float32).reshape(-1, 3)
        if raw.shape[0] % 3:
            raise ValueError(f"read_mesh_stl: {path}: vertex count is not a multiple of 3")
    uniq, inv = np.unique(np.ascontiguousarray(raw, np.float32), axis=0, return_inverse=True)
    return uniq.astype(np.float64), inv.reshape(-1, 3).astype(np.int64)


def write_mesh_stl(path: str | os.PathLike, coords: np.ndarray, triangles: np.ndarray, binary: bool = True,
                   name: str = "baemm") -> None:
    """Write a triangle mesh as STL (float32 coordinates, facet normals from
    the vertex order)."""
    p = np.asarray(coords, np.float64)[np.asarray(triangles, np.int64)]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-300)
    if binary:
        rec = np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("attr", "<u2")])
        out = np.zeros(p.shape[0], dtype=rec)
        out["n"] = n
        out["v"] = p.reshape(-1, 9)
        with open(path, "wb") as f:
            f.write(name.encode("ascii")[:80].ljust(80, b" "))
            f.write(np.array([p.shape[0]], "<u4").tobytes())
            f.write(out.tobytes())
        return
    p32, n32 = p.astype(np.float32), n.astype(np.float32)
    with open(path, "w") as f:
        f.write(f"solid {name}\n")
        for t in range(p.shape[0]):
            f.write("  facet normal {:.9e} {:.9e} {:.9e}\n    outer loop\n".format(*n32[t]))
            for q in range(3):
                f.write("      vertex {:.9e} {:.9e} {:.9e}\n".format(*p32[t, q]))
            f.write("    endloop\n  endfacet\n")
        f.write(f"endsolid {name}\n")


def icosphere(level: int):
    """Unit icosphere: an icosahedron subdivided ``level`` times, projected to
    radius 1 and oriented outward; float64 coordinates and int64 triangles
    (level 3: 642 vertices / 1280 triangles).  The subdivision is cached per
    level; the arrays returned are fresh copies."""
    coords, tris = _icosphere_cached(int(level))
    return coords.copy(), tris.copy()


@functools.lru_cache(maxsize=8)
def _icosphere_cached(level: int):
    return _icosphere_build(level)


def _icosphere_build(level: int):
    """Unit icosphere: icosahedron, ``level`` midpoint subdivisions, projected.

    Outward-oriented triangles.  V = 10*4^level + 2, T = 20*4^level.
    """
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
         (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
         (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
         (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            idx = cache.get(key)
            if idx is None:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                idx = len(verts) - 1
                cache[key] = idx
            return idx

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    coords = np.array(verts)
    tris = np.array(faces, dtype=np.int64)
    # orient outward
    cen = coords[tris].mean(axis=1)
    nrm = np.cross(coords[tris[:, 1]] - coords[tris[:, 0]], coords[tris[:, 2]] - coords[tris[:, 0]])
    flip = (nrm * cen).sum(axis=1) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return coords, tris


def torus(major: float = 1.0, minor: float = 0.4, n_minor: int = 160, n_major: int = 480):
    """Parametric torus, ``n_minor`` x ``n_major`` grid, 2 triangles per quad.

    Vertex (a, b) with a over the tube circle and b around the major circle.
    V = n_minor * n_major, T = 2 V.  Outward-oriented triangles.
    """
    a = 2.0 * np.pi * np.arange(n_minor) / n_minor
    b = 2.0 * np.pi * np.arange(n_major) / n_major
    A, Bm = np.meshgrid(a, b, indexing="ij")
    x = (major + minor * np.cos(A)) * np.cos(Bm)
    y = (major + minor * np.cos(A)) * np.sin(Bm)
    z = minor * np.sin(A)
    coords = np.stack([x, y, z], axis=-1).reshape(-1, 3)
    ia = np.arange(n_minor)
    ib = np.arange(n_major)
    I, J = np.meshgrid(ia, ib, indexing="ij")
    v00 = (I * n_major + J).ravel()
    v10 = (((I + 1) % n_minor) * n_major + J).ravel()
    v01 = (I * n_major + (J + 1) % n_major).ravel()
    v11 = (((I + 1) % n_minor) * n_major + (J + 1) % n_major).ravel()
    tris = np.empty((2 * v00.size, 3), dtype=np.int64)
    tris[0::2] = np.stack([v00, v01, v11], axis=1)
    tris[1::2] = np.stack([v00, v11, v10], axis=1)
    # orient outward: normal should point away from the tube centre line
    p = coords[tris]
    cen = p.mean(axis=1)
    nrm = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    phi = np.arctan2(cen[:, 1], cen[:, 0])
    core = np.stack([major * np.cos(phi), major * np.sin(phi), np.zeros_like(phi)], axis=1)
    flip = ((cen - core) * nrm).sum(axis=1) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return coords, tris


def points_off_torus(n: int, major: float = 1.0, minor: float = 0.4, min_dist: float = 0.05, seed: int = 0,
                     box=((-1.6, 1.6), (-1.6, 1.6), (-0.6, 0.6))) -> np.ndarray:
    """``n`` seeded points, uniform in ``box``, whose distance to the torus
    surface is at least ``min_dist`` (inside the tube and outside), float64 n x 3.

    Evaluation points for near-field potentials: closer to the surface the
    rounding of z = y - x in single precision is amplified by 1 / r^3.
    """
    rng = np.random.default_rng(seed)
    lo = np.array([b[0] for b in box])
    hi = np.array([b[1] for b in box])
    out = []
    have = 0
    while have < n:
        p = lo + (hi - lo) * rng.random((2 * (n - have) + 64, 3))
        rho = np.hypot(p[:, 0], p[:, 1])
        d = np.abs(np.hypot(rho - major, p[:, 2]) - minor)
        p = p[d >= min_dist]
        out.append(p)
        have += p.shape[0]
    return np.concatenate(out)[:n]


def fibonacci_sphere(n: int) -> np.ndarray:
    """``n`` quasi-uniform unit vectors (golden-angle spiral), float64 n x 3."""
    i = np.arange(n, dtype=np.float64) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = np.pi * (3.0 - np.sqrt(5.0)) * i
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def real_sph_harm_sum(xyz: np.ndarray, coeffs: np.ndarray, degree: int) -> np.ndarray:
    """Sum of real spherical harmonics of degree <= ``degree`` at unit points.

    ``coeffs`` has (degree+1)^2 entries ordered (l, m) with m = -l..l.
    Associated Legendre functions by the standard three-term recurrence.
    """
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    theta = np.arccos(np.clip(z, -1.0, 1.0))
    phi = np.arctan2(y, x)
    ct, st = np.cos(theta), np.sin(theta)
    L = degree
    P = np.zeros((L + 1, L + 1, xyz.shape[0]))
    P[0, 0] = 1.0
    for m in range(1, L + 1):
        P[m, m] = -(2 * m - 1) * st * P[m - 1, m - 1]
    for m in range(0, L):
        P[m + 1, m] = (2 * m + 1) * ct * P[m, m]
    for m in range(0, L + 1):
        for l in range(m + 2, L + 1):
            P[l, m] = ((2 * l - 1) * ct * P[l - 1, m] - (l + m - 1) * P[l - 2, m]) / (l - m)
    out = np.zeros(xyz.shape[0])
    idx = 0
    for l in range(L + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                Y = norm * P[l, 0]
            elif m > 0:
                Y = math.sqrt(2.0) * norm * P[l, am] * np.cos(am * phi)
            else:
                Y = math.sqrt(2.0) * norm * P[l, am] * np.sin(am * phi)
            out += coeffs[idx] * Y
            idx += 1
    return out


def sh_perturbed_sphere(level: int, degree: int, amplitude: float, seed: int):
    """Icosphere radially scaled by 1 + amplitude * S / max|S|, S a random
    real spherical-harmonic sum of degree <= ``degree`` with N(0,1) coefficients."""
    coords, tris = icosphere(level)
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((degree + 1) ** 2)
    s = real_sph_harm_sum(coords, c, degree)
    s = s / np.max(np.abs(s))
    return coords * (1.0 + amplitude * s)[:, None], tris
