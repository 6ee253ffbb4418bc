"""Ewald parameters, k-vectors and structure factors (src/ewald.jl, src/reference.jl:10-16)."""
import math
from dataclasses import dataclass

import numpy as np

from .cell import reciprocal_basis, volume
from .errors import ArgumentError

# The screened-Coulomb pair term is only evaluated for alpha*r in [0, PAIR_ERFC_XMAX]
# (src/ewald.jl:88); FrameworkBatch enforces alpha*ewald_cutoff <= PAIR_ERFC_XMAX.
PAIR_ERFC_XMAX = 4.0


@dataclass(frozen=True)
class EwaldParams:
    """Real-space cutoff (A) and target relative precision (src/ewald.jl:8-18)."""

    cutoff: float
    precision: float = 1.0e-6


def ewald_alpha(cutoff, precision):
    """alpha with erfc(alpha*rc) = rc*precision/2, by bisection (src/ewald.jl:21-32)."""
    target = cutoff * precision / 2
    lo, hi = 0.0, 20.0
    if not math.erfc(hi) - target < 0:
        raise ArgumentError(f"cannot reach precision {precision} with cutoff {cutoff}")
    for _ in range(200):
        mid = (lo + hi) / 2
        if math.erfc(mid) - target > 0:
            lo = mid
        else:
            hi = mid
        if hi - lo < 1.0e-12:
            break
    return (lo + hi) / 2 / cutoff


def ewald_kmax(alpha, precision):
    return 2 * alpha * math.sqrt(-math.log(precision / 2))


def pk(k2, alpha, V):
    """Reciprocal-space prefactor 2 pi / V exp(-k^2/4 alpha^2) / k^2 (src/ewald.jl:36-39)."""
    return 2 * math.pi / V * np.exp(-np.asarray(k2) / (4 * alpha**2)) / np.asarray(k2)


def kvector_bounds(A, kmax):
    """|n_i| <= kmax |a_i| / 2 pi for the half-space enumeration (src/ewald.jl:143)."""
    return np.array([int(math.ceil(kmax * np.linalg.norm(A[:, i]) / (2 * math.pi))) for i in range(3)], dtype=np.int32)


def kvectors(A, kmax):
    """Half-space k-vectors within kmax: n1 >= 0, weight 2 when n1 > 0, in the order n1, n2, n3
    (n3 fastest). Returns (ks (nk,3), weights, integer coefficients (nk,3)) (src/ewald.jl:142-157).
    k = (n1 B[:,0] + n2 B[:,1]) + n3 B[:,2] and |k| = sqrt((kx^2 + ky^2) + kz^2), in that operation
    order (pa_kvectors forms them the same way on the device)."""
    B = reciprocal_basis(A)
    n = kvector_bounds(A, kmax)
    n1, n2, n3 = np.meshgrid(np.arange(0, n[0] + 1), np.arange(-n[1], n[1] + 1), np.arange(-n[2], n[2] + 1),
                             indexing="ij")
    c = np.stack([n1.ravel(), n2.ravel(), n3.ravel()], axis=1)
    c = c[np.any(c != 0, axis=1)]
    cf = c.astype(np.float64)
    k = (cf[:, 0:1] * B[:, 0] + cf[:, 1:2] * B[:, 1]) + cf[:, 2:3] * B[:, 2]
    keep = np.sqrt(k2_of(k)) <= kmax
    c, k = c[keep], k[keep]
    w = np.where(c[:, 0] == 0, 1.0, 2.0)
    return k, w, c.astype(np.int32)


def k2_of(k):
    """|k|^2 = (kx^2 + ky^2) + kz^2 per row."""
    k = np.asarray(k, dtype=np.float64).reshape(-1, 3)
    return (k[:, 0] * k[:, 0] + k[:, 1] * k[:, 1]) + k[:, 2] * k[:, 2]


def structure_factor(ks, positions, charges, chunk_elems=1 << 22):
    """S(k) = sum_j q_j exp(i k.r_j), FP64 on the host (src/ewald.jl:159-170)."""
    ks = np.asarray(ks, dtype=np.float64).reshape(-1, 3)
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    q = np.asarray(charges, dtype=np.float64)
    S = np.zeros(len(ks), dtype=np.complex128)
    if len(ks) == 0 or len(pos) == 0:
        return S
    step = max(1, chunk_elems // max(1, len(pos)))
    for i0 in range(0, len(ks), step):
        ph = ks[i0:i0 + step] @ pos.T
        S[i0:i0 + step] = np.cos(ph) @ q + 1j * (np.sin(ph) @ q)
    return S


def full_ktables(A, positions, charges, alpha, kmax, sk=None, kv=None):
    """Every k-vector kvectors enumerates with its prefactor, host structure factor and integer
    coefficients (src/reference.jl:10-16). `sk`, if given, computes the structure factor
    (ks, positions, charges) -> complex array (e.g. on the device); `kv`, if given, the k-vectors
    and prefactors (B, nmax, kmax, alpha, V) -> (ks, weights, kpref, coefficients) (e.g. on the
    device, Context.kvectors)."""
    V = volume(A)
    if kv is not None:
        ks, w, kpref, coeffs = kv(reciprocal_basis(A), kvector_bounds(A, kmax), kmax, alpha, V)
    else:
        ks, w, coeffs = kvectors(A, kmax)
        kpref = w * pk(k2_of(ks), alpha, V) if len(ks) else np.zeros(0)
    S = (sk or structure_factor)(ks, positions, charges)
    return ks, kpref, S, coeffs
