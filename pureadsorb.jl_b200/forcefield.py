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
        """1-based index of a type name (src/forcefield.jl:41-45)."""
        try:
            return self.names.index(name) + 1
        except ValueError:
            raise ArgumentError(f"unknown LJ type {name}; force field defines {self.names}") from None


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
