"""Mesh sources: icospheres, spherical-harmonic perturbations, OBJ files.

The reference loads meshes with pywavefront and normalises them
(src/managers/mesh_manager.py:479-494); the benchmark configurations use
generated unit icospheres (subdivision 3/4/5 -> 1280/5120/20480 panels).
"""
from __future__ import annotations

import math

import numpy as np


def icosphere(subdiv: int):
    """Unit icosphere: the icosahedron with every triangle split into four
    `subdiv` times and the new vertices projected onto the unit sphere.
    Returns (vertices [nv,3] float64, panels [nt,3] int32), outward-oriented."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(int(subdiv)):
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
    return np.array(verts, dtype=np.float64), np.array(faces, dtype=np.int32)


def real_sph_harm_matrix(lmax: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Real orthonormal spherical harmonics Y_lm (l <= lmax, m = -l..l) at
    colatitude theta / longitude phi, via the associated Legendre recurrence.
    Returns [(lmax+1)^2, npts]."""
    x = np.cos(theta)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    P = {}
    P[(0, 0)] = np.ones_like(x)
    for m in range(1, lmax + 1):
        P[(m, m)] = -(2 * m - 1) * s * P[(m - 1, m - 1)]
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * x * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * x * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    rows = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                rows.append(norm * P[(l, 0)])
            elif m > 0:
                rows.append(math.sqrt(2) * norm * P[(l, am)] * np.cos(am * phi))
            else:
                rows.append(math.sqrt(2) * norm * P[(l, am)] * np.sin(am * phi))
    return np.array(rows)


def perturbed_sphere(subdiv: int, lmax: int = 6, amplitude: float = 0.05, seed: int = 0):
    """Icosphere radially perturbed by seeded real spherical harmonics of
    degree <= lmax: r = 1 + delta, delta = sum c_lm Y_lm with c_lm ~ N(0,1),
    scaled so that max|delta| = amplitude."""
    v, f = icosphere(subdiv)
    theta = np.arccos(np.clip(v[:, 2], -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    Y = real_sph_harm_matrix(lmax, theta, phi)
    rng = np.random.default_rng(seed)
    c = rng.standard_normal(Y.shape[0])
    delta = c @ Y
    delta *= amplitude / np.abs(delta).max()
    return v * (1.0 + delta)[:, None], f


def load_obj(path: str, normalise: bool = True):
    """Read `v`/`f` records (polygons fan-triangulated, 1-based or negative
    relative indices, `a/b/c` forms accepted).  With normalise=True the mesh
    is centred on the vertex mean and scaled by 1/max|coordinate| as the
    reference's MeshManager.load_asset does (mesh_manager.py:479-494)."""
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v":
                verts.append([float(p) for p in parts[1:4]])
            elif parts[0] == "f":
                # 1-based, or negative: relative to the vertices read so far
                idx = [int(p.split("/")[0]) for p in parts[1:]]
                idx = [i - 1 if i > 0 else len(verts) + i for i in idx]
                for t in range(1, len(idx) - 1):
                    faces.append([idx[0], idx[t], idx[t + 1]])
    v = np.array(verts, dtype=np.float64)
    if normalise:
        v = v - v.mean(axis=0, keepdims=True)
        v = v * (1.0 / np.abs(v).max())
    return v, np.array(faces, dtype=np.int32)


def analytical_sphere(r: float = 1.0, rows: int = 17, cols: int = 17):
    """Latitude-longitude sphere of MeshManager.load_analytical_sphere
    (src/managers/mesh_manager.py:496-518), same vertex and panel order: the
    south pole (0, -r, 0); rings i = 1..rows-1 at polar angle pi i / rows,
    each of `cols` vertices at azimuth 2 pi j / cols; the north pole last.
    Panels: a fan from the south pole to ring 1, then two triangles per
    (ring, column) quad, then a fan from the last ring to the north pole.
    Returns (vertices [nv,3] float64, panels [nt,3] int32)."""
    verts = [(0.0, -r, 0.0)]
    panels = []
    for i in range(1, rows):
        theta = math.pi * i / rows
        below, ring = 1 + (i - 2) * cols, 1 + (i - 1) * cols  # first vertex of rings i-1 and i
        for j in range(cols):
            phi = 2.0 * math.pi * j / cols
            verts.append((r * math.cos(phi) * math.sin(theta), -r * math.cos(theta), r * math.sin(phi) * math.sin(theta)))
            jn = (j + 1) % cols
            if i == 1:
                panels.append((0, ring + jn, ring + j))
            else:
                panels.append((below + j, below + jn, ring + j))
                panels.append((below + jn, ring + jn, ring + j))
    verts.append((0.0, r, 0.0))
    last, north = 1 + (rows - 2) * cols, 1 + (rows - 1) * cols
    for j in range(cols):
        panels.append((last + j, last + (j + 1) % cols, north))
    return np.array(verts, dtype=np.float64), np.array(panels, dtype=np.int32)


def analytical_disk(r: float = 1.0, N: int = 256):
    """Boundary of the disk of radius r as N segments, counter-clockwise
    (MeshManager.load_analytical_disk, src/managers/mesh_manager.py:520-536):
    vertex i at angle 2 pi i / N, segment i from vertex i to vertex (i+1) % N.
    Returns (vertices [N,2] float64, panels [N,2] int32)."""
    ang = [2.0 * math.pi * i / N for i in range(N)]
    v = np.array([[r * math.cos(a) for a in ang], [r * math.sin(a) for a in ang]], dtype=np.float64).T
    f = np.array([[i, (i + 1) % N] for i in range(N)], dtype=np.int32)
    return np.ascontiguousarray(v), f
