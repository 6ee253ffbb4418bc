"""Frameworks: the periodic host structures (src/structure.jl)."""
from dataclasses import dataclass, field

import numpy as np

from .cell import cell_matrix
from .errors import ArgumentError


@dataclass(eq=False)
class Framework:
    """A periodic host: `cell` (lattice vectors as columns), fractional coordinates `frac`,
    `labels`, element `symbols`, partial `charges` (e) and `replication`, the supercell factors
    already folded into cell/frac. `T` is the float type the caller works in (numpy.float64 or
    numpy.float32); it selects the kernel precision of a FrameworkBatch built from it
    (src/structure.jl:14-24)."""

    cell: np.ndarray
    frac: np.ndarray
    labels: list
    symbols: list
    charges: np.ndarray
    replication: tuple = (1, 1, 1)
    T: type = field(default=np.float64)

    def __post_init__(self):
        self.cell = np.asarray(self.cell, dtype=np.float64).reshape(3, 3)
        self.frac = np.asarray(self.frac, dtype=np.float64).reshape(-1, 3)
        self.charges = np.asarray(self.charges, dtype=np.float64).reshape(-1)
        self.replication = tuple(int(x) for x in self.replication)
        self.labels = list(self.labels)
        self.symbols = list(self.symbols)


def natoms(fw):
    return len(fw.frac)


def total_charge(fw):
    return float(np.sum(fw.charges))


def cartesian(fw):
    """Cartesian positions A*f (src/structure.jl:28)."""
    return fw.frac @ fw.cell.T


def read_cif(path, T=np.float64):
    """Minimal P1 CIF reader: one _atom_site loop with fractional coordinates and a required
    _atom_site_charge column (src/structure.jl:37-69)."""
    with open(path) as fh:
        lines = [l.strip() for l in fh.read().splitlines()]

    def getval(key):
        for l in lines:
            if l.startswith(key + " ") or l.startswith(key + "\t"):
                return l[len(key):].strip()
        raise ArgumentError(f"CIF is missing {key}")

    sg = getval("_symmetry_space_group_name_H-M").strip("'\"")
    if sg.replace(" ", "") != "P1":
        raise ArgumentError(f"only P1 CIF files are supported, got space group {sg}")
    keys = ("_cell_length_a", "_cell_length_b", "_cell_length_c", "_cell_angle_alpha", "_cell_angle_beta",
            "_cell_angle_gamma")
    cell = cell_matrix(*[float(getval(k)) for k in keys])
    try:
        h = lines.index("_atom_site_label")
    except ValueError:
        raise ArgumentError("CIF has no _atom_site_label loop") from None
    cols = []
    i = h
    while i < len(lines) and lines[i].startswith("_atom_site_"):
        cols.append(lines[i])
        i += 1
    if "_atom_site_charge" not in cols:
        raise ArgumentError("CIF has no _atom_site_charge column; partial charges are required")
    need = ("_atom_site_fract_x", "_atom_site_fract_y", "_atom_site_fract_z", "_atom_site_label",
            "_atom_site_type_symbol")
    if any(c not in cols for c in need):
        raise ArgumentError("CIF atom_site loop lacks label, type_symbol or fractional coordinates")
    cx, cy, cz = (cols.index(c) for c in need[:3])
    cl, cs, cq = cols.index("_atom_site_label"), cols.index("_atom_site_type_symbol"), cols.index("_atom_site_charge")
    frac, labels, symbols, charges = [], [], [], []
    while i < len(lines) and lines[i] and not lines[i].startswith("_") and not lines[i].startswith("loop_"):
        f = lines[i].split()
        if len(f) != len(cols):
            raise ArgumentError(f"CIF atom row has {len(f)} fields, header has {len(cols)}")
        frac.append([float(f[cx]), float(f[cy]), float(f[cz])])
        labels.append(f[cl])
        symbols.append(f[cs])
        charges.append(float(f[cq]))
        i += 1
    return Framework(cell, np.array(frac).reshape(-1, 3), labels, symbols, np.array(charges), (1, 1, 1), T)


def replicate(fw, n):
    """n[0] x n[1] x n[2] supercell; loop order k, j, i, atom (src/structure.jl:79-92)."""
    n = tuple(int(x) for x in n)
    if not all(x >= 1 for x in n):
        raise ArgumentError(f"replication factors must be ≥ 1, got {n}")
    na = natoms(fw)
    k, j, i = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    shifts = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)  # (N, 3), k slowest
    frac = ((fw.frac[None, :, :] + shifts[:, None, :]) / np.array(n, dtype=np.float64)).reshape(-1, 3)
    N = int(np.prod(n))
    return Framework(fw.cell @ np.diag(np.array(n, dtype=np.float64)), frac, fw.labels * N, fw.symbols * N,
                     np.tile(fw.charges, N), tuple(a * b for a, b in zip(fw.replication, n)), fw.T)
