"""Seeded synthetic geometries of the benchmark systems (Angstrom).

The reference generates lattices with its ``geom`` submodule (invoked from
python/input_/geom_interface.py:361-370), which is not part of the reference
tree; these generators build the same kinds of clusters from the lattice
definitions: a bcc or fcc lattice carved to a sphere, and two triangular
prisms facing each other tip to tip (bow-tie).  Every generator takes a seed
and applies a uniform positional jitter, so a configuration is reproducible
from (shape, size, lattice constant, jitter, seed).
"""
import math

import numpy as np


def _lattice(kind, a, extent):
    n = int(math.ceil(extent / a)) + 1
    r = np.arange(-n, n + 1, dtype=np.float64)
    base = np.stack(np.meshgrid(r, r, r, indexing='ij'), axis=-1).reshape(-1, 3)
    if kind == 'bcc':
        basis = np.array([[0, 0, 0], [0.5, 0.5, 0.5]])
    elif kind == 'fcc':
        basis = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]])
    else:
        raise ValueError(kind)
    pts = (base[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    return pts


def sphere(kind, a, radius, jitter=0.0, seed=0):
    """Lattice sites with |r| <= radius, ordered by (x, y, z), plus uniform jitter in [-j, j]."""
    pts = _lattice(kind, a, radius)
    pts = pts[np.einsum('ij,ij->i', pts, pts) <= radius * radius + 1e-9]
    pts = pts[np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))]
    if jitter:
        rng = np.random.default_rng(seed)
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    return pts


def rod(kind, a, length, radius, jitter=0.0, seed=0):
    """Lattice sites inside a cylinder of the given radius along z with hemispherical
    caps, total length `length` (Angstrom), ordered by (x, y, z), plus uniform jitter."""
    half = max(length / 2.0 - radius, 0.0)
    pts = _lattice(kind, a, length / 2.0 + a)
    z = np.clip(pts[:, 2], -half, half)
    d2 = pts[:, 0] ** 2 + pts[:, 1] ** 2 + (pts[:, 2] - z) ** 2
    pts = pts[d2 <= radius * radius + 1e-9]
    pts = pts[np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))]
    if jitter:
        rng = np.random.default_rng(seed)
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    return pts


def prism(a, edge, thickness, kind='fcc'):
    """Equilateral triangular prism in the xy plane, one tip at the origin pointing to -x,
    the opposite side at x = edge * sqrt(3)/2, thickness along z centred on 0."""
    h = edge * math.sqrt(3.0) / 2.0
    pts = _lattice(kind, a, max(edge, thickness) + a)
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    inside = (x >= -1e-9) & (x <= h + 1e-9) & (np.abs(y) <= x / math.sqrt(3.0) + 1e-9) & \
        (np.abs(z) <= thickness / 2.0 + 1e-9)
    return pts[inside]


def bowtie(a, edge, thickness, gap, jitter=0.0, seed=0):
    """Two prisms tip to tip along x with the given gap (Angstrom).

    Returns (coords, species) with species 0 for the left prism and 1 for the
    right one (e.g. Ag and Au)."""
    p = prism(a, edge, thickness)
    h = edge * math.sqrt(3.0) / 2.0
    left = p.copy()
    left[:, 0] = -(left[:, 0]) - gap / 2.0           # tip at -gap/2 pointing +x
    right = p.copy()
    right[:, 0] = right[:, 0] + gap / 2.0            # tip at +gap/2 pointing -x
    pts = np.concatenate([left, right])
    species = np.concatenate([np.zeros(len(left), np.int32), np.ones(len(right), np.int32)])
    order = np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))
    pts, species = pts[order], species[order]
    if jitter:
        rng = np.random.default_rng(seed)
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    del h
    return pts, species
