"""Force field and rigid guest (src/forcefield.jl)."""
import math
from dataclasses import dataclass, field

import numpy as np
import yaml

from .errors import ArgumentError, DimensionMismatch


class ForceField:
    """Lennard-Jones pair tables from per-type sigma (A) and epsilon (eV) with Lorentz-Berthelot
    mixing, LJ `cutoff` (A) and the analytic `tail` correction switch (src/forcefield.jl:8-39)."""

    def __init__(self, names, sigma, epsilon, cutoff, tail=True):
        s = np.asarray(sigma, dtype=np.float64).reshape(-1)
        e = np.asarray(epsilon, dtype=np.float64).reshape(-1)
        if not (len(names) == len(s) == len(e)):
            raise DimensionMismatch("names, sigma and epsilon must have the same length")
        self.names = [str(x) for x in names]
        self.sigma = (s[:, None] + s[None, :]) / 2
        self.epsilon = np.sqrt(e[:, None] * e[None, :])
        self.cutoff = float(cutoff)
        self.tail = bool(tail)

    def typeindex(self, name):
        """1-based index of a type name (src/forcefield.jl:41-45); the first of equal names."""
        index = self.__dict__.get("_index")
        if index is None:
            index = {}
            for i, n in enumerate(self.names):
                index.setdefault(n, i + 1)
            self._index = index
        i = index.get(name)
        if i is None:
            raise ArgumentError(f"unknown LJ type {name}; force field defines {self.names}")
        return i


def read_forcefield(path, T=np.float64):
    """kUPS-style YAML force field (src/forcefield.jl:54-61)."""
    with open(path) as fh:
        d = yaml.safe_load(fh)
    params = d["parameters"]
    names = list(params.keys())
    sig = [1.0 if params[n][0] is None else float(params[n][0]) for n in names]
    eps = [0.0 if params[n][1] is None else float(params[n][1]) for n in names]
    return ForceField(names, sig, eps, cutoff=float(d["cutoff"]), tail=d.get("tail_correction", True))


@dataclass(eq=False)
class Guest:
    """A rigid guest: site positions (A, body frame), 1-based force-field `types`, partial
    `charges` (e), critical temperature/pressure and acentric factor (src/forcefield.jl:76-83)."""

    sites: np.ndarray
    types: np.ndarray
    charges: np.ndarray
    tc: float = 1.0
    pc: float = 1.0
    omega: float = 0.0

    def __post_init__(self):
        self.sites = np.asarray(self.sites, dtype=np.float64).reshape(-1, 3)
        self.types = np.asarray(self.types, dtype=np.int64).reshape(-1)
        self.charges = np.asarray(self.charges, dtype=np.float64).reshape(-1)

    def same_as(self, other):
        return (np.array_equal(self.types, other.types) and np.array_equal(self.sites, other.sites)
                and np.array_equal(self.charges, other.charges))


def _number(x):
    return float(str(x).replace("_", "")) if isinstance(x, str) else float(x)


def read_guest(path, ff, T=np.float64):
    """kUPS-style YAML guest (src/forcefield.jl:91-101)."""
    with open(path) as fh:
        d = yaml.safe_load(fh)
    return Guest(np.array(d["positions"], dtype=np.float64), [ff.typeindex(s) for s in d["symbols"]],
                 np.array(d["charges"], dtype=np.float64), _number(d["critical_temperature"]),
                 _number(d["critical_pressure"]), _number(d["acentric_factor"]))


def tail_coefficient(ff, i, j):
    eps = ff.epsilon[i, j]
    if eps == 0:
        return 0.0
    s = ff.sigma[i, j]
    x = s / ff.cutoff
    return eps * s**3 * (x**9 / 3 - x**3)


def tail_delta(ff, counts, guest_counts, V):
    """Change of the analytic LJ tail correction on adding the guest (src/forcefield.jl:113-124)."""
    if not ff.tail:
        return 0.0
    n = ff.sigma.shape[0]
    if len(counts) != n or len(guest_counts) != n:
        raise DimensionMismatch(f"counts must have one entry per LJ type ({n}), got {len(counts)}")
    acc = 0.0
    # every term carries a factor guest_counts[b]; types absent from both host and guest add zero
    rows = [a for a in range(n) if counts[a] or guest_counts[a]]
    cols = [b for b in range(n) if guest_counts[b]]
    for a in rows:
        for b in cols:
            c = tail_coefficient(ff, a, b)
            acc += 2 * counts[a] * guest_counts[b] * c + guest_counts[a] * guest_counts[b] * c
    return 8 * math.pi / 3 / V * acc


def type_parameters(ff):
    """Per-type (sigma, epsilon) of a Lorentz-Berthelot force field: the diagonals of its tables
    (src/forcefield.jl:22-39 builds sigma_ii = sigma_i, epsilon_ii = epsilon_i)."""
    return np.diag(ff.sigma).copy(), np.diag(ff.epsilon).copy()


def pair_to_type_grad(ff, d_sigma_pair, d_epsilon_pair):
    """Chain rule through Lorentz-Berthelot mixing: derivatives with respect to the pair tables
    (d/dsigma_ij, d/depsilon_ij, full ntypes x ntypes matrices indexed like ff.sigma) to
    derivatives with respect to the per-type parameters. sigma_ij = (sigma_i + sigma_j)/2 gives
    d/dsigma_t = sum_ij d/dsigma_ij (delta_it + delta_jt)/2; epsilon_ij = sqrt(epsilon_i epsilon_j)
    gives d/depsilon_t = sum_ij d/depsilon_ij epsilon_ij (delta_it + delta_jt)/(2 epsilon_t)
    (unbounded at epsilon_t = 0 when another factor is nonzero)."""
    dS = np.asarray(d_sigma_pair, dtype=np.float64)
    dE = np.asarray(d_epsilon_pair, dtype=np.float64)
    _, eps_t = type_parameters(ff)
    g_sig = 0.5 * (dS.sum(axis=1) + dS.sum(axis=0))
    wE = dE * ff.epsilon
    with np.errstate(divide="ignore", invalid="ignore"):
        g_eps = (wE.sum(axis=1) + wE.sum(axis=0)) / (2 * eps_t)
    return g_sig, g_eps


def tail_delta_pair_grad(ff, counts, guest_counts, V):
    """Derivatives of tail_delta with respect to the pair tables (d/dsigma_ij, d/depsilon_ij) for
    c_ij = epsilon_ij (s^12/(3 rc^9) - s^6/rc^3), s = sigma_ij, weighted like tail_delta by
    2 counts_i guest_counts_j + guest_counts_i guest_counts_j (src/forcefield.jl:103-124)."""
    n = ff.sigma.shape[0]
    if not ff.tail:
        return np.zeros((n, n)), np.zeros((n, n))
    counts = np.asarray(counts, dtype=np.float64)
    gc = np.asarray(guest_counts, dtype=np.float64)
    M = 2 * counts[:, None] * gc[None, :] + gc[:, None] * gc[None, :]
    s, e, rc = ff.sigma, ff.epsilon, ff.cutoff
    f = 8 * math.pi / 3 / V
    dE = f * M * (s**12 / (3 * rc**9) - s**6 / rc**3)
    dS = f * M * e * (4 * s**11 / rc**9 - 6 * s**5 / rc**3)
    return dS, dE
