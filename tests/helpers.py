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
