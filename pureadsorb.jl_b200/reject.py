"""Hard-core rejection bounds (src/reject.jl), evaluated on the host in FP64.

The pair erfc here is scipy's, the function the reference's pair_erfc_dev approximates."""
import math

import numpy as np
from scipy.special import erfc

from .constants import KE
from .errors import ArgumentError

MAX_BISECT_ITERS = 200
EPS64 = float(np.finfo(np.float64).eps)


def theta_F(T=np.float64):
    """Smallest theta of type T with exp(-theta) == 0, by bisection on the float grid
    (src/reject.jl:11-19)."""
    T = np.dtype(T).type
    lo, hi = T(0), T(2000)
    with np.errstate(under="ignore"):
        if np.exp(-hi) != 0:
            raise ArgumentError(f"theta_F({T}): {hi} is too small for exp(-θ) to underflow to zero")
        while np.nextafter(lo, hi) != hi:
            mid = T(lo + (hi - lo) / T(2))
            if np.exp(-mid) == 0:
                hi = mid
            else:
                lo = mid
    return hi


def lj_pair_energy(r2, s, e):
    x = (s * s / r2) ** 3
    return 4 * e * (x * x - x)


def pair_energy(r, s, e, K, alpha):
    """LJ plus screened Coulomb of one pair at separation r (src/reject.jl:23)."""
    return lj_pair_energy(r * r, s, e) + K * erfc(alpha * r) / r


def find_r0(s, e, K, alpha, r_lj):
    """Zero of the attractive pair energy below the LJ minimum, clamped to r_lj
    (src/reject.jl:46-69). Vectorised over numpy arrays of equal shape."""
    s, e, K = (np.asarray(x, dtype=np.float64) for x in (s, e, K))
    if np.any(~(e > 0)):
        raise ArgumentError(f"find_r0: ε={e[~(e > 0)].ravel()[0]} must be positive (no Lennard-Jones well to bracket a root against)")
    if np.any(~(K < 0)):
        raise ArgumentError(f"find_r0: K={K[~(K < 0)].ravel()[0]} must be negative (attractive pair)")
    hi = s * 2.0 ** (1.0 / 6)
    if np.any(~(pair_energy(hi, s, e, K, alpha) < 0)):
        raise ArgumentError("find_r0: pair_energy at σ·2^(1/6) is not negative")
    lo = hi.copy()
    act = pair_energy(lo, s, e, K, alpha) <= 0
    it = 0
    while np.any(act):
        lo = np.where(act, lo / 2, lo)
        act = act & (pair_energy(lo, s, e, K, alpha) <= 0)
        it += 1
        if it > MAX_BISECT_ITERS:
            raise ArgumentError(f"find_r0: lower bracket search exceeded {MAX_BISECT_ITERS} halvings")
    act = hi - lo > 4 * EPS64 * hi
    it = 0
    while np.any(act):
        mid = (lo + hi) / 2
        pos = pair_energy(mid, s, e, K, alpha) > 0
        lo = np.where(act & pos, mid, lo)
        hi = np.where(act & ~pos, mid, hi)
        act = hi - lo > 4 * EPS64 * hi
        it += 1
        if it > MAX_BISECT_ITERS:
            raise ArgumentError(f"find_r0: bisection exceeded {MAX_BISECT_ITERS} iterations")
    return np.minimum((lo + hi) / 2, r_lj)


def hardcore_bound(guest_types, guest_charges, sigma, epsilon, types, charges, r_lj, alpha, kprefactor, Shost):
    """B_s: lower-magnitude bound on every pair's energy plus the reciprocal cross-term bound,
    Inf when a pair is attractive with no LJ wall (src/reject.jl:95-124). Types are 1-based
    indices into sigma/epsilon."""
    ht = np.asarray(types, dtype=np.int64) - 1
    q = np.asarray(charges, dtype=np.float64)
    # per site: the attractive pairs' (sigma, eps, K) triples; sigma and eps depend only on the
    # host type, so the distinct triples are (type, distinct K). One bisection per distinct triple
    # (as the reference memoises), all of a framework's triples in one vectorised call.
    sites, groups, ss, es, ks = [], [], [], [], []
    for a in range(len(guest_types)):
        gt = int(guest_types[a]) - 1
        ep = epsilon[gt, ht]
        K = KE * float(guest_charges[a]) * q
        att = K < 0
        if np.any(att & (ep == 0)):
            return math.inf
        sites.append((ep, att))
        for t in np.unique(ht[att]):
            sel = att & (ht == t)
            uk, inv = np.unique(K[sel], return_inverse=True)
            groups.append((a, sel, inv.reshape(-1), sum(len(x) for x in ks), len(uk), float(epsilon[gt, t])))
            ss.append(np.full(len(uk), float(sigma[gt, t])))
            es.append(np.full(len(uk), float(epsilon[gt, t])))
            ks.append(uk)
    bound = None
    if ks:
        uk_all = np.concatenate(ks)
        r0 = find_r0(np.concatenate(ss), np.concatenate(es), uk_all, alpha, r_lj)
        bound = np.concatenate(es) + np.abs(uk_all) * erfc(alpha * r0) / r0
    acc = 0.0
    for a, (ep, att) in enumerate(sites):
        terms = ep.copy()
        for ga, sel, inv, o, n, e_t in groups:
            if ga == a:
                terms[sel] = bound[o:o + n][inv]
        # sequential sum in atom order (builtin sum() of floats compensates, so accumulate)
        acc = float(np.add.accumulate(np.concatenate(([acc], terms)))[-1])
    Rs = 0.0
    for i in range(len(kprefactor)):
        Rs += float(kprefactor[i]) * abs(complex(Shost[i]))
    return acc + 2 * KE * float(np.sum(np.abs(guest_charges))) * Rs


def kmin_table(guest_charges, types, charges, ntypes):
    """K_min[a, t]: most negative KE q_a q_h over host atoms of type t, or 0 (src/reject.jl:134-145)."""
    N = len(guest_charges)
    kmin = np.zeros((N, ntypes))
    ht = np.asarray(types, dtype=np.int64) - 1
    for a in range(N):
        K = KE * float(guest_charges[a]) * np.asarray(charges, dtype=np.float64)
        np.minimum.at(kmin[a], ht, K)
    return kmin


def find_rho2(s, e, kmin, margin, r_lj):
    """Squared rejection radius: first root of LJ(r) - |kmin|/r = margin, clamped to r_lj; 0 for
    an infinite margin or a zero epsilon (src/reject.jl:168-209). Vectorised over s, e, kmin."""
    s, e, kmin = (np.atleast_1d(np.asarray(x, dtype=np.float64)) for x in (s, e, kmin))
    if not margin > 0:
        raise ArgumentError(f"find_rho2: margin={margin} must be positive (sigma={s[0]}, epsilon={e[0]}, kmin={kmin[0]})")
    out = np.zeros(s.shape)
    if math.isinf(margin):
        return out
    live = e != 0
    if not np.any(live):
        return out
    s, e, kmin = s[live], e[live], kmin[live]

    def f(r):
        return lj_pair_energy(r * r, s, e) - np.abs(kmin) / r - margin

    hi = s.copy()
    act = f(hi) >= 0
    it = 0
    while np.any(act):
        hi = np.where(act, hi * 2, hi)
        act = act & (f(hi) >= 0)
        it += 1
        if it > MAX_BISECT_ITERS:
            raise ArgumentError(f"find_rho2: upper bracket search exceeded {MAX_BISECT_ITERS} doublings")
    lo = hi.copy()
    act = f(lo) < 0
    it = 0
    while np.any(act):
        lo = np.where(act, lo / 2, lo)
        act = act & (f(lo) < 0)
        it += 1
        if it > MAX_BISECT_ITERS:
            raise ArgumentError(f"find_rho2: lower bracket search exceeded {MAX_BISECT_ITERS} halvings")
    act = hi - lo > 4 * EPS64 * hi
    it = 0
    while np.any(act):
        mid = (lo + hi) / 2
        pos = f(mid) > 0
        lo = np.where(act & pos, mid, lo)
        hi = np.where(act & ~pos, mid, hi)
        act = hi - lo > 4 * EPS64 * hi
        it += 1
        if it > MAX_BISECT_ITERS:
            raise ArgumentError(f"find_rho2: bisection exceeded {MAX_BISECT_ITERS} iterations")
    out[live] = np.minimum((lo + hi) / 2, r_lj) ** 2
    return out
