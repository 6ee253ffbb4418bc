"""Cell geometry and the phase-0 cell list (src/cell.jl).

Matrices are 3x3 numpy arrays with the lattice vectors as columns (a along x, b in the xy plane).
"""
import math

import numpy as np

from .errors import ArgumentError


def _cosd(x):
    r = math.fmod(x, 360.0)
    exact = {0.0: 1.0, 90.0: 0.0, 180.0: -1.0, 270.0: 0.0, -90.0: 0.0, -180.0: -1.0, -270.0: 0.0}
    return exact.get(r, math.cos(math.radians(x)))


def _sind(x):
    r = math.fmod(x, 360.0)
    exact = {0.0: 0.0, 90.0: 1.0, 180.0: 0.0, 270.0: -1.0, -90.0: -1.0, -180.0: 0.0, -270.0: 1.0}
    return exact.get(r, math.sin(math.radians(x)))


def cell_matrix(a, b, c, alpha, beta, gamma):
    """Upper-triangular cell matrix from lengths and angles in degrees (src/cell.jl:2-12)."""
    if not (a > 0 and b > 0 and c > 0):
        raise ArgumentError(f"cell lengths must be positive, got a={a}, b={b}, c={c}")
    ca, cb, cg, sg = _cosd(alpha), _cosd(beta), _cosd(gamma), _sind(gamma)
    if sg == 0:
        raise ArgumentError(f"cell angle γ={gamma} is degenerate: sin(γ) is zero")
    cy = (ca - cb * cg) / sg
    radicand = 1.0 - cb**2 - cy**2
    if not radicand > 0:
        raise ArgumentError(f"cell angles α={alpha}, β={beta}, γ={gamma} describe a degenerate cell")
    cz = math.sqrt(radicand)
    return np.array([[a, b * cg, c * cb], [0.0, b * sg, c * cy], [0.0, 0.0, c * cz]])


def det3(A):
    """Cofactor expansion along the first row (exact for diagonal and triangular cells, unlike
    an LU-based determinant)."""
    return float(A[0, 0] * (A[1, 1] * A[2, 2] - A[1, 2] * A[2, 1]) - A[0, 1] * (A[1, 0] * A[2, 2] - A[1, 2] * A[2, 0])
                 + A[0, 2] * (A[1, 0] * A[2, 1] - A[1, 1] * A[2, 0]))


def volume(A):
    return abs(det3(A))


def perpendicular_lengths(A):
    """Distances between opposite faces (src/cell.jl:16-20)."""
    V = volume(A)
    a, b, c = A[:, 0], A[:, 1], A[:, 2]
    return np.array([V / np.linalg.norm(np.cross(b, c)), V / np.linalg.norm(np.cross(a, c)),
                     V / np.linalg.norm(np.cross(a, b))])


def min_multiplicity(A, cutoff):
    """Smallest replication with 2*cutoff between opposite faces (src/cell.jl:24-27)."""
    L = perpendicular_lengths(A)
    return tuple(int(math.ceil(2 * cutoff / L[i])) for i in range(3))


def reciprocal_basis(A):
    return 2 * math.pi * np.linalg.inv(A).T


def minimum_image(A, invA, d):
    """d - A round(invA d), round half to even (src/cell.jl:34-37); d may be (..., 3)."""
    d = np.asarray(d, dtype=np.float64)
    f = d @ invA.T
    return d - np.rint(f) @ A.T


def grid_dims(L, w):
    return np.array([max(1, int(math.floor(L[i] / w))) for i in range(3)], dtype=np.int32)


def stencil_reaches(L, n, reach):
    return np.array([int(math.ceil(reach * int(n[i]) / L[i])) for i in range(3)], dtype=np.int32)


def cell_coord(frac, n):
    """0-based cell coordinates of fractional coordinates wrapped into [0, 1) (src/cell.jl:149-152)."""
    f = np.asarray(frac, dtype=np.float64)
    fw = f - np.floor(f)
    c = np.floor(fw * n).astype(np.int64)
    return np.minimum(c, np.asarray(n, dtype=np.int64) - 1)


def cell_linear(ijk, n):
    ijk = np.asarray(ijk)
    return ijk[..., 0] + int(n[0]) * (ijk[..., 1] + int(n[1]) * ijk[..., 2])


def cell_sort(frac, n):
    """Stable counting sort of atoms by cell: (permutation, prod(n)+1 local offsets) (src/cell.jl:96-118)."""
    ncell = int(n[0]) * int(n[1]) * int(n[2])
    if len(frac) == 0:
        return np.zeros(0, dtype=np.int64), np.zeros(ncell + 1, dtype=np.int32)
    c = cell_linear(cell_coord(frac, n), n)
    perm = np.argsort(c, kind="stable")
    counts = np.bincount(c, minlength=ncell)
    offsets = np.zeros(ncell + 1, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)
    return perm, offsets
