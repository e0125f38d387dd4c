"""Synthetic tetrahedral sphere meshes in gmsh 2.2 ``.vmsh`` format.

The cube [-1,1]^3 is cut into n^3 cells; each cell is split into 6 tetrahedra
around its (+,+,+) main diagonal (the Kuhn split, which is conforming across
cells).  Every vertex is then mapped radially, x -> R * x * |x|_inf / |x|_2,
which sends the cube surface onto the sphere of radius R and keeps the origin
fixed.  Tetrahedra are emitted with positive signed volume, because the
material Gram blocks depend on that sign (the weights 6V and the SWG prefactor
A/3V both carry the signed volume, see libbuff ``SWGVolume.cc:50-85`` and
``VIEMatrix.cc:200-316``).

Counts: NV=(n+1)^3 vertices, NT=6n^3 tetrahedra, N=12n^3-6n^2 interior faces
(= SWG basis functions).

The files are read by the reference-compatible gmsh reader
(``ReadGMSHFile.cc:66-261`` semantics: ``$Nodes`` / ``$Elements``, element
type 4 = tetrahedron).
"""
from __future__ import annotations

import itertools
import os

import numpy as np


def sphere_arrays(n: int, radius: float = 1.0, jitter: float = 0.0,
                  seed: int = 0, center=(0.0, 0.0, 0.0)):
    """Return (vertices[NV,3] float64, tets[NT,4] int32, 0-based)."""
    g = np.linspace(-1.0, 1.0, n + 1)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def vid(i, j, k):
        return (i * (n + 1) + j) * (n + 1) + k

    tets = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                base = np.array([i, j, k])
                for perm in itertools.permutations(range(3)):
                    c = base.copy()
                    vs = [vid(*c)]
                    for ax in perm:
                        c = c.copy()
                        c[ax] += 1
                        vs.append(vid(*c))
                    tets.append(vs)
    tets = np.asarray(tets, dtype=np.int64)

    # radial map of the cube onto the sphere
    ninf = np.max(np.abs(P), axis=1)
    n2 = np.linalg.norm(P, axis=1)
    scale = np.where(n2 > 0, ninf / np.where(n2 > 0, n2, 1.0), 0.0)
    V = radius * P * scale[:, None]

    if jitter > 0.0:
        h = 2.0 * radius / n
        rng = np.random.default_rng(seed)
        V = V + rng.uniform(-jitter * h, jitter * h, size=V.shape)

    V = V + np.asarray(center, dtype=np.float64)[None, :]
    tets = orient_positive(V, tets)
    return V, tets.astype(np.int32)


def signed_volumes(V, tets):
    a = V[tets[:, 1]] - V[tets[:, 0]]
    b = V[tets[:, 2]] - V[tets[:, 0]]
    c = V[tets[:, 3]] - V[tets[:, 0]]
    return np.einsum("ij,ij->i", a, np.cross(b, c)) / 6.0


def orient_positive(V, tets):
    tets = np.array(tets, copy=True)
    vol = signed_volumes(V, tets)
    neg = vol < 0
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    vol = signed_volumes(V, tets)
    if np.any(vol <= 0):
        raise ValueError("degenerate tetrahedron in generated mesh")
    return tets


def write_vmsh(path: str, V, tets) -> str:
    """Write a gmsh 2.2 ASCII mesh holding only tetrahedra (1-based ids)."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
        f.write(f"{len(V)}\n")
        for i, (x, y, z) in enumerate(V):
            f.write(f"{i + 1} {x:.17g} {y:.17g} {z:.17g}\n")
        f.write("$EndNodes\n$Elements\n")
        f.write(f"{len(tets)}\n")
        for i, t in enumerate(tets):
            f.write(f"{i + 1} 4 2 0 1 {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}\n")
        f.write("$EndElements\n")
    return path


def sphere_vmsh(path: str, n: int, radius: float = 1.0, jitter: float = 0.0,
                seed: int = 0, center=(0.0, 0.0, 0.0)) -> str:
    V, T = sphere_arrays(n, radius, jitter, seed, center)
    return write_vmsh(path, V, T)


def num_bfs(n: int) -> int:
    return 12 * n ** 3 - 6 * n ** 2


def cached_sphere(directory: str, n: int, radius: float = 1.0,
                  jitter: float = 0.0, seed: int = 0) -> str:
    """Generate (once) a sphere mesh file under ``directory`` and return its path."""
    os.makedirs(directory, exist_ok=True)
    tag = f"sphere_n{n}_R{radius:g}" + (f"_j{jitter:g}_s{seed}" if jitter > 0 else "")
    path = os.path.join(directory, tag + ".vmsh")
    if not os.path.exists(path):
        tmp = path + f".tmp{os.getpid()}"
        sphere_vmsh(tmp, n, radius, jitter, seed)
        os.replace(tmp, path)
    return path


if __name__ == "__main__":
    import sys
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 5
    out = sys.argv[2] if len(sys.argv) > 2 else f"sphere_n{n}.vmsh"
    sphere_vmsh(out, n)
    print(out, "N =", num_bfs(n))
