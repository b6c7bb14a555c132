import numpy as np


def relerr(a, b):
    a = np.asarray(a); b = np.asarray(b)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def crandn(rng, *shape, dtype=np.complex128):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def tiny_meshes():
    """Meshes of 1, 2, 4 and 17 triangles (a single partly filled tile)."""
    tri1 = (np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0.2]]), np.array([[0, 1, 2]]))
    quad2 = (np.array([[0.0, 0, 0], [1, 0, 0], [1, 1, 0.3], [0, 1, 0]]), np.array([[0, 1, 2], [0, 2, 3]]))
    tetra = (np.array([[1.0, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]]),
             np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]]))
    # a strip of 17 triangles over 10 lower and 9 upper vertices (all used)
    xs = np.arange(10, dtype=float)
    strip_v = np.concatenate([np.stack([xs, 0 * xs, 0 * xs], 1), np.stack([xs[:9], 1 + 0 * xs[:9], 0.1 * xs[:9]], 1)])
    strip_t = [[i, i + 1, 10 + i] for i in range(9)] + [[i + 1, 11 + i, 10 + i] for i in range(8)]
    return {"tri1": tri1, "quad2": quad2, "tetra": tetra, "strip17": (strip_v, np.array(strip_t))}


def oracle_apply_at_vertices(orc, tris, B, kappa, coeff, wave_count, wave_chunk_size, verts):
    """The oracle's ApplyBoundaryOperators_PL (alpha 1, beta 0, no mass term) at
    the vertices `verts` only, for meshes too large for the full O(N^2) oracle:
    B_tri = AvOp B, the dense kernel on the triangles incident to `verts`
    (orc.boundary_kernel_tri_index), the single-layer diagonal
    c1 (diag_i + i kappa) B_tri[i] (ApplySingleLayerDiagonal.hpp:29-61) and
    AvOp^T restricted to `verts`, in the oracle's precision and geometry."""
    tris = np.asarray(tris)
    _, _, area, diag = orc.geometry()
    a3 = area / 3.0
    Btri = a3[:, None] * np.asarray(B, np.complex128)[tris].sum(axis=1)
    inc = [np.nonzero((tris == v).any(axis=1))[0] for v in verts]
    rows = np.unique(np.concatenate(inc))
    Ct = orc.boundary_kernel_tri_index(Btri, kappa, coeff, wave_count, wave_chunk_size, rows)
    pos = {int(r): k for k, r in enumerate(rows)}
    scale = 1.0 / (4.0 * np.pi)
    c1 = np.asarray(coeff, np.complex128).reshape(-1, 4)[:, 1] * scale
    kap = np.asarray(kappa, np.float64)
    nch = wave_count // wave_chunk_size
    fac = np.repeat(c1[None, :nch] * (diag[rows][:, None] + 1j * kap[None, :nch]), wave_chunk_size, axis=1)
    Ct = Ct + fac * Btri[rows]
    out = np.zeros((len(verts), wave_count), np.complex128)
    for q, tri_list in enumerate(inc):
        for i in tri_list:
            out[q] += a3[i] * Ct[pos[int(i)]]
    return out
