"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference measures on RUBTAK 3x3x3 + CO2; the benchmark configurations here are synthetic
frameworks generated deterministically from numpy's PCG64 (numpy.random.default_rng(seed)):

- lj_ch4:   cubic P1, a = 25.832 A, 424 atoms of 4 types (round-robin A..D), uniform positions
            with 1.2 A minimum-image separation (seed 1), no charges, united-atom CH4 guest,
            LJ cutoff 12.8 A, truncated without tail correction.
- co2:      monoclinic a=12.4, b=14.1, c=16.3 A, beta=104.7 deg, 216 atoms of 5 types
            (round-robin), eps/kB U(20,70) K, sigma U(2.4,3.5) A, 1.2 A minimum separation,
            charges N(0, 0.4 e) shifted to zero net charge, replicated 3x3x3 (5,832 atoms); rigid
            3-site CO2 (C-O 1.16 A); LJ and Ewald cutoffs 12 A, Ewald precision 1e-6, tail on.
- batched:  nfw triclinic frameworks (seed 7): lengths U(8,30) A, angles U(60,120) deg (redrawn
            when degenerate), log-uniform 50..2000 atoms per unit cell, 3..6 own types each with
            eps/kB U(15,80) K and sigma U(2.3,3.6) A, zero-sum N(0, 0.5 e) charges, uniform
            positions, replicated until every perpendicular width reaches 2 (rc + r_guest).
- fitting:  nfw frameworks (seed 11) drawn like `batched` but typed from one shared 4-type palette,
            plus 8 hidden scale factors U(0.9, 1.1) of the palette's (epsilon, sigma).
"""
import math

import numpy as np

from .cell import cell_matrix, min_multiplicity, minimum_image
from .constants import KB
from .errors import ArgumentError
from .ewald import EwaldParams
from .forcefield import ForceField, Guest
from .structure import Framework, replicate


def _uniform_min_dist(rng, A, n, dmin, max_tries=2_000_000):
    invA = np.linalg.inv(A)
    pts = np.zeros((0, 3))
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms with the requested minimum separation")
        f = rng.random(3)
        if len(pts):
            d = minimum_image(A, invA, (f - pts) @ A.T)
            if np.min(np.einsum("ij,ij->i", d, d)) < dmin * dmin:
                continue
        pts = np.vstack([pts, f])
    return pts


def co2_guest(ff):
    return Guest(np.array([[0.0, 0, 0], [-1.16, 0, 0], [1.16, 0, 0]]),
                 [ff.typeindex("C_co2"), ff.typeindex("O_co2"), ff.typeindex("O_co2")],
                 np.array([0.70, -0.35, -0.35]), 304.13, 7.3773e6, 0.22394)


CO2_TYPES = [("C_co2", 2.80, 27.0), ("O_co2", 3.05, 79.0)]


def lj_ch4(T=np.float64):
    """The LJ-only CH4 workload. Returns (frameworks, ff, guest, ewald, run parameters)."""
    rng = np.random.default_rng(1)
    a = 25.832
    A = cell_matrix(a, a, a, 90.0, 90.0, 90.0)
    frac = _uniform_min_dist(rng, A, 424, 1.2)
    params = [("A", 2.46, 62.4), ("B", 3.12, 48.2), ("C", 3.47, 47.9), ("D", 2.57, 22.1)]
    symbols = [params[i % 4][0] for i in range(424)]
    fw = Framework(A, frac, symbols, symbols, np.zeros(424), (1, 1, 1), T)
    names = [p[0] + "_" for p in params] + ["CH4"]
    ff = ForceField(names, [p[1] for p in params] + [3.73], [p[2] * KB for p in params] + [148.0 * KB],
                    cutoff=12.8, tail=False)
    guest = Guest(np.zeros((1, 3)), [ff.typeindex("CH4")], np.zeros(1), 190.564, 4.5992e6, 0.01142)
    return [fw], ff, guest, EwaldParams(cutoff=12.8, precision=1.0e-6), dict(T=298.15, ninsert=100_000, seed=42,
                                                                            nblocks=10)


def co2(T=np.float64, seed=42, replication=(3, 3, 3)):
    """The charged rigid-CO2 workload (5,832 atoms)."""
    rng = np.random.default_rng(seed)
    A = cell_matrix(12.4, 14.1, 16.3, 90.0, 104.7, 90.0)
    frac = _uniform_min_dist(rng, A, 216, 1.2)
    eps = rng.uniform(20.0, 70.0, 5)
    sig = rng.uniform(2.4, 3.5, 5)
    q = rng.normal(0.0, 0.4, 216)
    q -= q.mean()
    symbols = ["ABCDE"[i % 5] for i in range(216)]
    unit = Framework(A, frac, symbols, symbols, q, (1, 1, 1), T)
    fw = replicate(unit, replication)
    names = [c + "_" for c in "ABCDE"] + [t[0] for t in CO2_TYPES]
    ff = ForceField(names, list(sig) + [t[1] for t in CO2_TYPES], list(eps * KB) + [t[2] * KB for t in CO2_TYPES],
                    cutoff=12.0, tail=True)
    return [fw], ff, co2_guest(ff), EwaldParams(cutoff=12.0, precision=1.0e-6), dict(T=298.15, ninsert=1_000_000,
                                                                                     seed=42, nblocks=10)


def _geometry(rng, max_unit_atoms):
    """One framework's cell and atom count as the batched workload draws them."""
    while True:
        L = rng.uniform(8.0, 30.0, 3)
        ang = rng.uniform(60.0, 120.0, 3)
        try:
            A = cell_matrix(L[0], L[1], L[2], ang[0], ang[1], ang[2])
            break
        except ArgumentError:
            continue
    na = int(round(math.exp(rng.uniform(math.log(50), math.log(max_unit_atoms)))))
    return A, na


def batched(nfw=64, seed=7, T=np.float64, max_unit_atoms=2000):
    """The batched uneven-framework workload: nfw distinct frameworks."""
    rng = np.random.default_rng(seed)
    rc, r_guest = 12.0, 1.16
    fws, names, sig, eps = [], [], [], []
    for n in range(nfw):
        A, na = _geometry(rng, max_unit_atoms)
        nt = int(rng.integers(3, 7))
        tnames = [f"F{n}T{t}" for t in range(nt)]
        names += [x + "_" for x in tnames]
        eps += list(rng.uniform(15.0, 80.0, nt) * KB)
        sig += list(rng.uniform(2.3, 3.6, nt))
        frac = rng.random((na, 3))
        q = rng.normal(0.0, 0.5, na)
        q -= q.mean()
        symbols = [tnames[i % nt] for i in range(na)]
        unit = Framework(A, frac, symbols, symbols, q, (1, 1, 1), T)
        fws.append(replicate(unit, min_multiplicity(A, rc + r_guest)))
    names += [t[0] for t in CO2_TYPES]
    sig += [t[1] for t in CO2_TYPES]
    eps += [t[2] * KB for t in CO2_TYPES]
    ff = ForceField(names, sig, eps, cutoff=rc, tail=True)
    return fws, ff, co2_guest(ff), EwaldParams(cutoff=rc, precision=1.0e-6), dict(T=298.15, ninsert=nfw * 2**20,
                                                                                  seed=7, nblocks=10)


PALETTE = ("P0", "P1", "P2", "P3")


def fitting(nfw=128, seed=11, T=np.float64, max_unit_atoms=2000):
    """The force-field fitting workload: nfw frameworks drawn like the batched workload (cells,
    atom counts, uniform positions, zero-sum N(0, 0.5 e) charges, replication) whose atoms share
    one 4-type host palette P0..P3 (round-robin), so that the fitted parameters are the palette's
    4 x (epsilon, sigma). The palette's eps/kB U(15,80) K and sigma U(2.3,3.6) A come first from
    the seeded stream; after the frameworks, 8 hidden scale factors U(0.9, 1.1) (epsilon of P0..P3,
    then sigma of P0..P3) define the parameters the targets are computed at."""
    rng = np.random.default_rng(seed)
    rc, r_guest = 12.0, 1.16
    pal_eps = rng.uniform(15.0, 80.0, 4) * KB
    pal_sig = rng.uniform(2.3, 3.6, 4)
    fws = []
    for n in range(nfw):
        A, na = _geometry(rng, max_unit_atoms)
        frac = rng.random((na, 3))
        q = rng.normal(0.0, 0.5, na)
        q -= q.mean()
        symbols = [PALETTE[i % 4] for i in range(na)]
        unit = Framework(A, frac, symbols, symbols, q, (1, 1, 1), T)
        fws.append(replicate(unit, min_multiplicity(A, rc + r_guest)))
    hidden = rng.uniform(0.9, 1.1, 8)
    names = [p + "_" for p in PALETTE] + [t[0] for t in CO2_TYPES]
    ff = ForceField(names, list(pal_sig) + [t[1] for t in CO2_TYPES], list(pal_eps) + [t[2] * KB for t in CO2_TYPES],
                    cutoff=rc, tail=True)
    return fws, ff, co2_guest(ff), EwaldParams(cutoff=rc, precision=1.0e-6), dict(
        T=298.15, ninsert_per_framework=2**18, seed=seed, nblocks=10, steps=200, lr=1e-2, hidden=hidden,
        fitted_types=[p + "_" for p in PALETTE])
