"""FrameworkBatch: the structure-of-arrays batch of framework systems (src/batch.jl).

Built on the host in FP64 whatever the precision tag `T`: `T` (numpy.float32 or numpy.float64,
taken from the frameworks) selects the device kernels - the FP32 pair/Ewald path with FP64
constants and accumulation, or the plain FP64 path - as the reference's float type does.
Index conventions follow the reference exactly: offsets are 0-based, LJ types, guest types and
framework indices 1-based.
"""
import copy
import math

import numpy as np

from . import _lib
from .cell import cell_sort, grid_dims, min_multiplicity, perpendicular_lengths, volume
from .constants import KB, KE
from .errors import ArgumentError, DimensionMismatch
from .ewald import PAIR_ERFC_XMAX, ewald_alpha, ewald_kmax, full_ktables
from .forcefield import tail_delta
from .reject import hardcore_bound, kmin_table
from .structure import cartesian

# Guard on the orientation dependence of the guest self term (src/batch.jl:160-162).
SELF_TERM_TOLERANCE = 1.0e-3
SELF_TERM_GUARD_FACTOR = 2
KT_REF = KB * 300
# The 64 fixed guest orientations of the self-term average: quaternions of the pose stream with
# seed 0x5e1f, system 0 (no real system uses index 0), insertions 1..64. The reference draws them
# from Julia's Xoshiro(0x5e1f) (src/batch.jl:302-303), which has no counterpart outside Julia.
SELF_TERM_SEED = 0x5E1F
SELF_TERM_NORIENT = 64


def self_term_quaternions():
    return np.array([_lib.pose_host(_lib.PA_PRECISION_F64, SELF_TERM_SEED, 0, o)[1]
                     for o in range(1, SELF_TERM_NORIENT + 1)])


def _rotate(q, v):
    u = np.asarray(q[:3], dtype=np.float64)
    w = float(q[3])
    v = np.asarray(v, dtype=np.float64)
    return v + 2 * np.cross(u, np.cross(u, v) + w * v)


def verify_replication(n, fw, kv_full, coeffs, Sh_full):
    """Host structure factor negligible on a strided sample of up to 32 uncoupled k-vectors, or
    the claimed replication is false (src/batch.jl:173-195)."""
    rep = np.array(fw.replication)
    uncoupled = np.nonzero(np.any(np.mod(coeffs, rep) != 0, axis=1))[0]
    if len(uncoupled) == 0:
        return
    stride = max(1, -(-len(uncoupled) // 32))
    sample = uncoupled[::stride][:32]
    mags = np.abs(Sh_full[sample])
    i = int(np.argmax(mags))
    maxS = float(mags[i])
    threshold = max(1.0e-8, 100 * float(np.finfo(np.float64).eps)) * float(np.sum(np.abs(fw.charges)))
    if maxS > threshold:
        raise ArgumentError(
            f"framework {n} claims replication {fw.replication}, but its host structure factor at "
            f"k={kv_full[sample[i]]} (not coupled to that replication) is {maxS}, exceeding threshold "
            f"{threshold} = max(1e-8, 100·eps)·Σ|q_host|; this replication does not describe the atoms")


class FrameworkBatch:
    """Batch of `nsys` framework systems sharing one force field, guest and Ewald parameters
    (src/batch.jl:1-104, 237-432). Arrays are stored once per distinct framework;
    `framework_of[n]` (1-based) names system n's framework.

    `sk`, if given, computes host structure factors (ks, positions, charges) -> complex array;
    the default evaluates them on the host in FP64 like the reference, and
    `sk=Context.structure_factor` runs the library's FP64 device kernel instead. `self_term`,
    likewise, computes the guest self term's per-orientation sums (ks, kpref, sites, charges) ->
    array (without KE); `self_term=Context.self_term` runs them on the device. `bounds`, likewise,
    computes the hard-core bounds B_s from the finished batch (batch -> array of one per
    framework); `bounds=Context.batch_bounds` evaluates them on the device (FP64, equal to the
    host's to rounding) through the batch's upload to that context, which later calls reuse.
    `kv`, `kmin` and `cellsort` take the k-vector enumeration with its prefactors, the kmin table and
    the phase-0 cell sort (signatures of `Context.kvectors`, `Context.kmin_table` and
    `Context.cell_sort`); `device=Context` sets sk, self_term, kv, kmin and cellsort to that
    context's device versions at once (the tables equal the host's bit for bit, the structure
    factors, self terms and prefactors to rounding).
    """

    def __init__(self, fws, ff, guest, ewald, cellwidth=2, fullk=False, T=None, sk=None, self_term=None,
                 bounds=None, kv=None, kmin=None, cellsort=None, device=None):
        if device is not None:
            sk = sk or device.structure_factor
            self_term = self_term or device.self_term
            kv = kv or device.kvectors
            kmin = kmin or device.kmin_table
            cellsort = cellsort or device.cell_sort
        fws = list(fws)
        if not fws:
            raise ArgumentError("FrameworkBatch needs at least one framework")
        self.T = np.dtype(T if T is not None else fws[0].T).type
        if self.T not in (np.float32, np.float64):
            raise ArgumentError(f"float type must be float32 or float64, got {self.T}")
        N = len(guest.sites)
        if N > _lib.PA_MAX_GUEST_SITES:
            raise ArgumentError(f"guest has {N} sites; at most {_lib.PA_MAX_GUEST_SITES} are supported")
        rc = max(ff.cutoff, ewald.cutoff)
        r_guest = float(np.max(np.linalg.norm(guest.sites, axis=1))) if N else 0.0
        rc_guard = rc + r_guest
        w = float(cellwidth)

        # dedup by value: cell, replication, fractional coordinates, symbols, charges (src/batch.jl:252-265)
        index = {}
        framework_of = []
        unique = []
        for fw in fws:
            key = (fw.cell.tobytes(), fw.replication, fw.frac.tobytes(), tuple(fw.symbols), fw.charges.tobytes())
            if key not in index:
                unique.append(fw)
                index[key] = len(unique)
            framework_of.append(index[key])

        alpha = ewald_alpha(ewald.cutoff, ewald.precision)
        if alpha * ewald.cutoff > PAIR_ERFC_XMAX:
            raise ArgumentError(
                f"α·ewald_cutoff = {alpha * ewald.cutoff} exceeds PAIR_ERFC_XMAX = {PAIR_ERFC_XMAX}: "
                "insertion_energy's screened-Coulomb series is only fitted up to that bound; "
                f"loosen ewald.precision or shorten ewald.cutoff to bring α·ewald_cutoff back under {PAIR_ERFC_XMAX}")
        kmax = ewald_kmax(alpha, ewald.precision)
        neutral = bool(np.all(guest.charges == 0))
        self_quats = self_term_quaternions() if not neutral else None
        # the guest's site offsets at every self-term orientation (the same for every framework)
        self_sites = (np.array([[_rotate(q, s) for s in guest.sites] for q in self_quats]) if not neutral
                      else None)

        # compact LJ types: framework atoms' types union the guest's (src/batch.jl:309-317)
        ty_orig = []
        for fw in unique:  # one lookup per distinct symbol, then a gather over the atoms
            syms, inv = np.unique(np.asarray(fw.symbols, dtype=str), return_inverse=True)
            idx = np.array([ff.typeindex(s + "_") for s in syms], dtype=np.int64)
            ty_orig.append(idx[inv.reshape(-1)] if len(syms) else np.zeros(0, np.int64))
        allt = np.concatenate(ty_orig + [np.asarray(guest.types, dtype=np.int64)])
        compact_to_orig = np.unique(allt).astype(np.int32)
        o2c = {int(t): i + 1 for i, t in enumerate(compact_to_orig)}
        o2c_arr = np.zeros(int(compact_to_orig.max(initial=0)) + 1, dtype=np.int32)
        o2c_arr[compact_to_orig] = np.arange(1, len(compact_to_orig) + 1, dtype=np.int32)
        ci = compact_to_orig - 1
        sigma = ff.sigma[np.ix_(ci, ci)].copy()
        epsilon = ff.epsilon[np.ix_(ci, ci)].copy()
        ntypes = len(compact_to_orig)
        guest_types = np.array([o2c[int(t)] for t in guest.types], dtype=np.int32)
        nff = len(ff.names)
        gcounts = np.bincount(np.asarray(guest.types, dtype=np.int64) - 1, minlength=nff)

        positions, types, charges, perms = [], [], [], []
        atom_offsets = [0]
        cells, invcells, volumes, alphas = [], [], [], []
        ks, kpref, Shost, kcoeffs = [], [], [], []
        k_offsets = [0]
        constant_offset, halfranges = [], []
        ncells, cell_offsets, cellgrid_offsets = [], [], [0]
        kmin_list = []
        offset_parts = []  # per framework: (KE (self + excl + net), self-term mean, type counts, V)
        natoms_total = 0
        for n, fw in enumerate(unique, start=1):
            m = min_multiplicity(fw.cell, rc_guard)
            if m != (1, 1, 1):
                raise ArgumentError(f"framework {n} is too small for cutoff {rc} plus guest reach {r_guest} = "
                                    f"{rc_guard}; replicate it by {m} first")
            A = fw.cell
            L = perpendicular_lengths(A)
            n_grid = grid_dims(L, w)
            pos = cartesian(fw)
            ty = o2c_arr[ty_orig[n - 1]]
            perm, local = (cellsort or cell_sort)(fw.frac, n_grid)
            positions.append(pos[perm])
            types.append(ty[perm])
            charges.append(fw.charges[perm])
            perms.append(perm.astype(np.int32))
            natoms_total += len(perm)
            atom_offsets.append(natoms_total)
            cell_offsets.append(local)
            cellgrid_offsets.append(cellgrid_offsets[-1] + len(local))
            ncells.append(n_grid)
            V = volume(A)
            cells.append(A)
            invcells.append(np.linalg.inv(A))
            volumes.append(V)
            alphas.append(alpha)
            if not neutral or fw.replication != (1, 1, 1):
                kv_full, kpref_full, Sh_full, coeffs = full_ktables(A, pos, fw.charges, alpha, kmax, sk, kv)
                if fw.replication != (1, 1, 1):
                    verify_replication(n, fw, kv_full, coeffs, Sh_full)
            self_mean = 0.0
            if not neutral:
                coupled = np.all(np.mod(coeffs, np.array(fw.replication)) == 0, axis=1)
                sel = np.ones(len(coeffs), dtype=bool) if fullk else coupled
                ks.append(kv_full[sel])
                kpref.append(kpref_full[sel])
                Shost.append(Sh_full[sel])
                kcoeffs.append(coeffs[sel])
                if self_term is not None:
                    samples = KE * np.asarray(self_term(kv_full, kpref_full, self_sites, guest.charges))
                else:
                    samples = np.empty(SELF_TERM_NORIENT)
                    for o in range(SELF_TERM_NORIENT):
                        gs = self_sites[o]
                        ph = kv_full @ gs.T
                        Sg = np.cos(ph) @ guest.charges + 1j * (np.sin(ph) @ guest.charges)
                        samples[o] = KE * float(np.sum(kpref_full * np.abs(Sg) ** 2))
                self_mean = float(np.sum(samples)) / len(samples)
                half = (float(np.max(samples)) - float(np.min(samples))) / 2
                halfranges.append(half)
                if SELF_TERM_GUARD_FACTOR * half / KT_REF > SELF_TERM_TOLERANCE:
                    raise ArgumentError(
                        f"guest self-term half-range estimate {half} eV (guard factor {SELF_TERM_GUARD_FACTOR}) for "
                        f"guest with charges {guest.charges} at framework {n}: {SELF_TERM_GUARD_FACTOR}·{half} exceeds "
                        f"{SELF_TERM_TOLERANCE}·KB·300K = {SELF_TERM_TOLERANCE * KT_REF} eV; this guest/cell "
                        "combination needs the per-insertion reciprocal sum")
            else:
                halfranges.append(0.0)
            k_offsets.append(k_offsets[-1] + (len(ks[-1]) if (not neutral) else 0))
            kmin_list.append((kmin or kmin_table)(guest.charges, types[-1], charges[-1], ntypes).reshape(-1))
            counts = np.bincount(ty_orig[n - 1] - 1, minlength=nff)
            self_e = -alpha / math.sqrt(math.pi) * float(np.sum(guest.charges ** 2))
            excl = 0.0
            for a in range(N):
                for c in range(a + 1, N):
                    r = float(np.linalg.norm(guest.sites[a] - guest.sites[c]))
                    excl -= guest.charges[a] * guest.charges[c] * (1 - math.erfc(alpha * r)) / r
            Qh = float(np.sum(fw.charges))
            Qg = float(np.sum(guest.charges))
            net = -math.pi / (2 * V * alpha**2) * ((Qh + Qg) ** 2 - Qh**2)
            constant_offset.append(tail_delta(ff, counts, gcounts, V) + KE * (self_e + excl + net) + self_mean)
            offset_parts.append((KE * (self_e + excl + net), self_mean, counts, V))

        self.positions = np.ascontiguousarray(np.concatenate(positions) if natoms_total else np.zeros((0, 3)))
        self.types = np.ascontiguousarray(np.concatenate(types) if natoms_total else np.zeros(0, np.int32), dtype=np.int32)
        self.charges = np.ascontiguousarray(np.concatenate(charges) if natoms_total else np.zeros(0))
        self.atom_offsets = np.array(atom_offsets, dtype=np.int32)
        self.cells = np.array(cells)
        self.invcells = np.array(invcells)
        self.volumes = np.array(volumes)
        self.alphas = np.array(alphas)
        nk = k_offsets[-1]
        self.ks = np.concatenate(ks) if nk else np.zeros((0, 3))
        self.kprefactor = np.concatenate(kpref) if nk else np.zeros(0)
        self.Shost = np.concatenate(Shost) if nk else np.zeros(0, dtype=np.complex128)
        self.kcoeffs = np.concatenate(kcoeffs).astype(np.int32) if nk else np.zeros((0, 3), np.int32)
        self.k_offsets = np.array(k_offsets, dtype=np.int32)
        self.constant_offset = np.array(constant_offset)
        self.self_term_halfrange = np.array(halfranges)
        self.ncells = np.array(ncells, dtype=np.int32).reshape(-1, 3)
        self.cell_offsets = np.concatenate(cell_offsets).astype(np.int32)
        self.cellgrid_offsets = np.array(cellgrid_offsets, dtype=np.int32)
        self.sigma, self.epsilon = sigma, epsilon
        self.compact_to_orig = compact_to_orig
        self.guest_types = guest_types
        self.guest_types_orig = np.asarray(guest.types, dtype=np.int64).copy()
        self.guest_sites_orig = guest.sites.copy()
        self.guest_charges_orig = guest.charges.copy()
        self.kmin = np.concatenate(kmin_list) if kmin_list else np.zeros(0)
        self.cutoff = float(ff.cutoff)
        self.ewald_cutoff = float(ewald.cutoff)
        self.fullk = bool(fullk)
        self.nsys = len(fws)
        self.framework_of = np.array(framework_of, dtype=np.int32)
        self.perm = np.concatenate(perms) if perms else np.zeros(0, np.int32)
        self._ff_names = list(ff.names)
        self._gcounts = gcounts
        self._offset_parts = offset_parts
        self._device = {}
        self._desc = None      # desc() result; a FrameworkBatch is not modified after construction
        self._rejection = {}   # rejection tables per (kT, eps)
        self.bs = (np.asarray(bounds(self), dtype=np.float64).reshape(-1) if bounds is not None
                   else self._hardcore_bounds())

    def _hardcore_bounds(self):
        """B_s per framework (src/batch.jl:409-423)."""
        bs = np.empty(self.nframeworks())
        for n in range(len(bs)):
            a0, a1 = self.atom_offsets[n], self.atom_offsets[n + 1]
            k0, k1 = self.k_offsets[n], self.k_offsets[n + 1]
            bs[n] = hardcore_bound(self.guest_types, self.guest_charges_orig, self.sigma, self.epsilon,
                                   self.types[a0:a1], self.charges[a0:a1], self.cutoff, float(self.alphas[n]),
                                   self.kprefactor[k0:k1], self.Shost[k0:k1])
        return bs

    def with_forcefield(self, ff, move_device=False, device_bounds=False):
        """The same frameworks, guest and Ewald tables under another force field with the same type
        names, cutoff and tail setting (a fitting loop changes only LJ parameters). Recomputes what
        depends on them: the compact pair tables, each framework's constant offset (its tail
        correction) and hard-core bound; the rest is shared with this batch. The result equals a
        fresh FrameworkBatch(fws, ff, guest, ewald) field for field. With move_device=True the new
        batch takes over this batch's device uploads, whose pair tables and constant offsets are
        replaced in place (pa_batch_set_pair_tables), and this batch loses them. With
        device_bounds=True as well, the hard-core bounds come from the device
        (pa_batch_hardcore_bounds; equal to the host's to rounding) instead of the host loop."""
        if list(ff.names) != self._ff_names:
            raise ArgumentError("with_forcefield needs a force field with the same type names")
        if float(ff.cutoff) != self.cutoff:
            raise ArgumentError(f"with_forcefield needs the same LJ cutoff ({self.cutoff}), got {ff.cutoff}")
        new = copy.copy(self)
        ci = np.asarray(self.compact_to_orig, dtype=np.int64) - 1
        new.sigma = ff.sigma[np.ix_(ci, ci)].copy()
        new.epsilon = ff.epsilon[np.ix_(ci, ci)].copy()
        new.constant_offset = np.array([tail_delta(ff, counts, self._gcounts, V) + ke + sm
                                        for ke, sm, counts, V in self._offset_parts])
        new._device = {}
        new._desc = None
        new._rejection = {}
        if move_device:
            for key, dev in self._device.items():
                dev.set_pair_tables(new.sigma, new.epsilon, new.constant_offset)
                new._device[key] = dev
            self._device = {}
        if device_bounds and new._device:
            new.bs = next(iter(new._device.values())).hardcore_bounds(new.nframeworks())
        else:
            new.bs = new._hardcore_bounds()
        return new

    def nframeworks(self):
        return len(self.cells)

    def check_axes(self):
        """The array-consistency checks widom makes before using a batch (src/widom.jl:331-364)."""
        if not (len(self.positions) == len(self.types) == len(self.charges)):
            raise DimensionMismatch(f"batch positions/types/charges must share axes: {len(self.positions)} vs "
                                    f"{len(self.types)} vs {len(self.charges)}")
        if not (len(self.ks) == len(self.kprefactor) == len(self.Shost)):
            raise DimensionMismatch(f"batch ks/kprefactor/Shost must share axes: {len(self.ks)} vs "
                                    f"{len(self.kprefactor)} vs {len(self.Shost)}")
        nfw = self.nframeworks()
        if len(self.ncells) != nfw:
            raise DimensionMismatch(f"batch ncells must have one entry per framework (nframeworks={nfw}): {len(self.ncells)}")
        if len(self.cellgrid_offsets) != nfw + 1:
            raise DimensionMismatch(f"batch cellgrid_offsets must have nframeworks+1={nfw + 1} entries, got "
                                    f"{len(self.cellgrid_offsets)}")
        if self.cellgrid_offsets[-1] != len(self.cell_offsets):
            raise DimensionMismatch(f"batch cellgrid_offsets[end]={self.cellgrid_offsets[-1]} must equal "
                                    f"length(cell_offsets)={len(self.cell_offsets)}")
        for fw in range(nfw):
            g1 = self.cellgrid_offsets[fw + 1]
            nat = self.atom_offsets[fw + 1] - self.atom_offsets[fw]
            if self.cell_offsets[g1 - 1] != nat:
                raise DimensionMismatch(f"framework {fw + 1}: last cell_offsets entry {self.cell_offsets[g1 - 1]} "
                                        f"must equal its atom count {nat}")

    def desc(self):
        """(pa_batch_desc, arrays it points into): the C-ABI view of this batch, built once."""
        if getattr(self, "_desc", None) is None:
            self._desc = self._make_desc()
        return self._desc

    def _make_desc(self):
        col = lambda M: np.ascontiguousarray(np.transpose(M, (0, 2, 1)).reshape(-1))  # column-major per matrix
        arr = {
            "positions": np.ascontiguousarray(self.positions.reshape(-1), dtype=np.float64),
            "types": np.ascontiguousarray(self.types, dtype=np.int32),
            "charges": np.ascontiguousarray(self.charges, dtype=np.float64),
            "atom_offsets": np.ascontiguousarray(self.atom_offsets, dtype=np.int32),
            "cells": col(self.cells), "invcells": col(self.invcells),
            "volumes": np.ascontiguousarray(self.volumes), "alphas": np.ascontiguousarray(self.alphas),
            "ks": np.ascontiguousarray(self.ks.reshape(-1), dtype=np.float64),
            "kprefactor": np.ascontiguousarray(self.kprefactor, dtype=np.float64),
            "Shost": np.ascontiguousarray(np.stack([self.Shost.real, self.Shost.imag], axis=1).reshape(-1)),
            "kcoeffs": np.ascontiguousarray(self.kcoeffs.reshape(-1), dtype=np.int32),
            "k_offsets": np.ascontiguousarray(self.k_offsets, dtype=np.int32),
            "constant_offset": np.ascontiguousarray(self.constant_offset, dtype=np.float64),
            "ncells": np.ascontiguousarray(self.ncells.reshape(-1), dtype=np.int32),
            "cell_offsets": np.ascontiguousarray(self.cell_offsets, dtype=np.int32),
            "cellgrid_offsets": np.ascontiguousarray(self.cellgrid_offsets, dtype=np.int32),
            "sigma": np.ascontiguousarray(self.sigma.T.reshape(-1)),
            "epsilon": np.ascontiguousarray(self.epsilon.T.reshape(-1)),
            "guest_types": np.ascontiguousarray(self.guest_types, dtype=np.int32),
            "guest_sites": np.ascontiguousarray(self.guest_sites_orig.reshape(-1), dtype=np.float64),
            "guest_charges": np.ascontiguousarray(self.guest_charges_orig, dtype=np.float64),
            "framework_of": np.ascontiguousarray(self.framework_of, dtype=np.int32),
        }
        d = _lib.BatchDesc()
        d.nsys, d.nfw, d.ntypes, d.nguest = self.nsys, self.nframeworks(), len(self.sigma), len(self.guest_types)
        for k, v in arr.items():
            setattr(d, k, _lib.ptr(v) if v.size else None)
        d.cutoff, d.ewald_cutoff = self.cutoff, self.ewald_cutoff
        return d, arr

    def device(self, ctx):
        """This batch uploaded to `ctx` for its precision (cached per context)."""
        key = id(ctx)
        dev = self._device.get(key)
        if dev is None or dev.ctx is not ctx:
            d, keep = self.desc()
            prec = _lib.PA_PRECISION_F32 if self.T == np.float32 else _lib.PA_PRECISION_F64
            dev = _lib.DeviceBatch(ctx, d, keep, prec)
            self._device[key] = dev
        return dev

    def drop_device(self):
        for dev in self._device.values():
            dev.free()
        self._device.clear()

    def drop_host_caches(self):
        """Forgets the cached C-ABI descriptor and the per-(kT, eps) rejection tables, so the next
        call rebuilds both as a reference widom call does (src/widom.jl:382)."""
        self._desc = None
        self._rejection = {}


def nframeworks(batch):
    return batch.nframeworks()
