"""Widom insertion into a loaded configuration: the test-particle step of PureAdsorb.jl's NVT
chain (`widom_chain_kernel!`, src/nvt.jl:85-124, driven per production cycle by `run_nvt!`,
src/nvt.jl:200-358).

A configuration is what `SystemState` (src/state.jl:5-446) holds for the test particle: each
system's live guests (reference points and orientations) and its running structure factor
S(k) = S_host(k) + sum over guests, over the system's full k table (the batch must be built with
fullk=True: a guest's own S(k) is nonzero at every k, not only the host-coupled subset). A test
insertion's energy is then

    ΔU = host-guest real space + KE 2 Re(conj(S_sys) S_test) over the k table
         + guest-guest real space (each site pair its own minimum image, src/guest.jl:51-75)
         + insertion_constant_term(system, N_g)    (src/nvt.jl:45-66)

with no hard-core rejection (single-phase). On the device this is the FP32 path with three
per-call inputs (pa_chain_args): the systems' S(k) in place of the host's, their constant terms
in place of the frameworks' constant offsets, and the live guests' site positions for the
guest-guest kernel (k_guest32). Tiles of the FP32 path never mix systems, so a batch whose
systems share a framework (the usual NVT/isotherm set-up, src/isotherm.jl:118) is expanded to one
framework per system before upload (`system_batch`).

The Monte Carlo moves that evolve the configuration between cycles (src/moves.jl, src/state.jl's
bookkeeping, src/audit.jl) are a different path and are not part of this package: a caller passes
the configuration of each cycle. `widom_along_chain` then reduces the cycles' insertions with
WidomResult's reduction, one block per cycle, as `run_nvt!` does (src/nvt.jl:336-345).
"""
import copy
import math

import numpy as np

from . import _lib
from .batch import _rotate
from .constants import KB, KE
from .errors import ArgumentError, DimensionMismatch
from .forcefield import tail_delta
from .widom import _reduce, block_sums, build_rejection_tables, default_backend


class SystemState:
    """The configuration of every system of a batch that a test insertion sees (the Widom subset
    of src/state.jl:5-126): guest_offsets (nsys+1, each system's reserved slot range),
    occupancy (nsys, live guests, a prefix of the slots), refpoints (nslots x 3, Cartesian, Å),
    orientations (nslots x 4, unit quaternions (x, y, z, w)), k_offsets (nsys+1) and Sk (complex,
    each system's running structure factor over its framework's k table, host plus live guests).
    Slots beyond a system's occupancy hold the sentinel pose (origin, identity)."""

    def __init__(self, batch, guest, refpoints, orientations, guest_offsets, occupancy):
        _check_guest(batch, guest, "SystemState")
        if not batch.fullk:
            raise ArgumentError("SystemState needs a FrameworkBatch built with fullk=true: a guest's structure factor "
                                "is nonzero at every k-vector, not only the host-coupled subset the sparse "
                                "(Milestone A) path keeps")
        nsys = batch.nsys
        go = np.asarray(guest_offsets, dtype=np.int64)
        occ = np.asarray(occupancy, dtype=np.int64)
        if len(go) != nsys + 1 or len(occ) != nsys:
            raise DimensionMismatch(f"guest_offsets must have nsys+1={nsys + 1} entries and occupancy nsys={nsys}, got "
                                    f"{len(go)} and {len(occ)}")
        if go[0] != 0 or np.any(np.diff(go) < 0):
            raise ArgumentError("guest_offsets must start at 0 and be nondecreasing")
        if np.any(occ < 0) or np.any(occ > np.diff(go)):
            raise ArgumentError(f"occupancy must be within each system's capacity: occupancy={occ.tolist()}, "
                                f"capacities={np.diff(go).tolist()}")
        rp = np.asarray(refpoints, dtype=np.float64).reshape(-1, 3)
        qt = np.asarray(orientations, dtype=np.float64).reshape(-1, 4)
        if len(rp) != go[-1] or len(qt) != go[-1]:
            raise DimensionMismatch(f"refpoints and orientations must have one row per slot ({go[-1]}), got {len(rp)} "
                                    f"and {len(qt)}")
        self.nsys = nsys
        self.guest_offsets = go
        self.occupancy = occ
        self.refpoints = rp.copy()
        self.orientations = qt.copy()
        fw = np.asarray(batch.framework_of, dtype=np.int64) - 1
        ko = np.asarray(batch.k_offsets, dtype=np.int64)
        nk = ko[fw + 1] - ko[fw]
        self.k_offsets = np.concatenate([[0], np.cumsum(nk)]).astype(np.int64)
        # S(k) = S_host(k) + Σ_guests Σ_sites q e^{i k·r}, FP64 (src/state.jl:404-413)
        self.Sk = np.zeros(int(self.k_offsets[-1]), dtype=np.complex128)
        q = np.asarray(guest.charges, dtype=np.float64)
        for s in range(nsys):
            ks = batch.ks[ko[fw[s]]:ko[fw[s] + 1]]
            S = np.array(batch.Shost[ko[fw[s]]:ko[fw[s] + 1]], dtype=np.complex128)
            sites = self.live_sites(guest, s).reshape(-1, 3)
            if len(sites) and len(ks):
                qs = np.tile(q, len(sites) // len(q))
                S = S + np.exp(1j * (sites @ ks.T)).T @ qs
            self.Sk[self.k_offsets[s]:self.k_offsets[s + 1]] = S

    def nguests(self, s):
        """Live guests of system s (0-based)."""
        return int(self.occupancy[s])

    def live_sites(self, guest, s):
        """Absolute site positions of system s's live guests, (nguests, N, 3) (guest_sites_at,
        src/guest.jl:78): refpoint + v + 2 u x (u x v + w v) per site (src/energy.jl:13-16)."""
        j0 = int(self.guest_offsets[s])
        n = int(self.occupancy[s])
        q = self.orientations[j0:j0 + n]
        u, w = q[:, None, :3], q[:, None, 3:4]
        v = np.asarray(guest.sites, dtype=np.float64)[None, :, :]
        c = np.cross(u, v) + w * v
        return self.refpoints[j0:j0 + n, None, :] + v + 2 * np.cross(u, c)

    def chain_inputs(self, guest):
        """The per-call tables of a device call (cached: a SystemState is not modified after
        construction): S(k) as (re, im) pairs, live-guest offsets and their site positions."""
        cached = self.__dict__.get("_chain_inputs")
        if cached is not None:
            return cached
        Sk = np.ascontiguousarray(np.stack([self.Sk.real, self.Sk.imag], axis=1).reshape(-1))
        live = [self.live_sites(guest, s) for s in range(self.nsys)]
        goff = np.concatenate([[0], np.cumsum([len(x) for x in live])]).astype(np.int32)
        sites = np.ascontiguousarray(np.concatenate([x.reshape(-1) for x in live]) if goff[-1] else np.zeros(3))
        self._chain_inputs = (Sk, goff, sites)
        return self._chain_inputs

    @classmethod
    def placed(cls, batch, guest, ncounts, *, T, seed=0, capacities=None, max_draws=100_000):
        """A configuration with ncounts[s] guests in system s, each drawn uniformly (position in the
        cell, orientation on SO(3)) and redrawn until it clears widom's hard-core test against the
        host at temperature T (src/state.jl:304-343, `initial_poses`); guest-guest overlap is not
        checked. The draws are the pose stream keyed by (seed, system, draw index), so a Widom seed
        equal to `seed` would insert exactly onto the placed guests: pass another one."""
        nsys = batch.nsys
        ncounts = np.asarray(ncounts, dtype=np.int64)
        caps = ncounts if capacities is None else np.asarray(capacities, dtype=np.int64)
        if len(ncounts) != nsys:
            raise DimensionMismatch(f"ncounts must have one entry per system (nsys={nsys}), got {len(ncounts)}")
        if len(caps) != nsys:
            raise DimensionMismatch(f"capacities must have one entry per system (nsys={nsys}), got {len(caps)}")
        if np.any(ncounts < 0):
            raise ArgumentError(f"ncounts must be non-negative, got {ncounts.tolist()}")
        if np.any(ncounts > caps):
            raise ArgumentError(f"capacities must be >= ncounts in every system: ncounts={ncounts.tolist()}, "
                                f"capacities={caps.tolist()}")
        go = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
        rp = np.zeros((int(go[-1]), 3))
        qt = np.tile([0.0, 0.0, 0.0, 1.0], (int(go[-1]), 1))
        kT = float(batch.T(KB * float(T)))
        rho2, _ = build_rejection_tables(batch, kT)
        N, nt = len(batch.guest_types), len(batch.sigma)
        prec = _lib.PA_PRECISION_F32 if batch.T == np.float32 else _lib.PA_PRECISION_F64
        for s in range(nsys):
            fw = int(batch.framework_of[s]) - 1
            A, iA = batch.cells[fw], batch.invcells[fw]
            a0, a1 = int(batch.atom_offsets[fw]), int(batch.atom_offsets[fw + 1])
            hpos = batch.positions[a0:a1]
            r2max = np.asarray(rho2, dtype=np.float64).reshape(nsys, N, nt)[s][:, np.asarray(batch.types[a0:a1]) - 1]
            k = 0
            for j in range(int(ncounts[s])):
                while True:
                    k += 1
                    if k > max_draws:
                        raise ArgumentError(f"system {s + 1}: no pose clearing the hard-core test in {max_draws} draws")
                    rpos, quat = _lib.pose_host(prec, seed, s + 1, k)
                    pos = A @ rpos
                    ok = True
                    for a, site in enumerate(guest.sites):
                        d = pos + _rotate(quat, site) - hpos
                        d = d - (np.rint(d @ iA.T) @ A.T)
                        if np.any(np.einsum("ij,ij->i", d, d) < r2max[a]):
                            ok = False
                            break
                    if ok:
                        break
                rp[go[s] + j] = pos
                qt[go[s] + j] = quat
        return cls(batch, guest, rp, qt, go, ncounts)


def _check_guest(batch, guest, who):
    if not (np.array_equal(guest.types, batch.guest_types_orig) and np.array_equal(guest.sites, batch.guest_sites_orig)
            and np.array_equal(guest.charges, batch.guest_charges_orig)):
        raise ArgumentError(f"guest passed to {who} does not match the guest FrameworkBatch was built with")


def insertion_constant_term(ff, batch, guest, s, Ng):
    """The pose-independent part of a test insertion's ΔU in system s (0-based) holding Ng guests
    (src/nvt.jl:45-66): the tail-correction and net-charge-correction changes from adding one more
    guest, plus the guest's own self energy, exclusion and orientation-averaged reciprocal self
    term. At Ng = 0 it is the framework's constant offset itself."""
    fw = int(batch.framework_of[s]) - 1
    if Ng == 0:
        return float(batch.constant_offset[fw])
    a0, a1 = int(batch.atom_offsets[fw]), int(batch.atom_offsets[fw + 1])
    V, alpha = float(batch.volumes[fw]), float(batch.alphas[fw])
    nff = len(ff.names)
    c2o = np.asarray(batch.compact_to_orig, dtype=np.int64) - 1
    gcounts = np.bincount(np.asarray(batch.guest_types_orig, dtype=np.int64) - 1, minlength=nff)
    host = np.bincount(c2o[np.asarray(batch.types[a0:a1], dtype=np.int64) - 1], minlength=nff)
    Qh = float(np.sum(batch.charges[a0:a1]))
    Qg = float(np.sum(guest.charges))

    def net_at(m):
        return -KE * math.pi / (2 * V * alpha**2) * ((Qh + m * Qg) ** 2 - Qh**2)

    def tail_at(m):  # guest_tail_correction (src/guest.jl:17)
        return tail_delta(ff, host, m * gcounts, V)

    base = float(batch.constant_offset[fw]) - tail_at(1) - net_at(1)
    return base + tail_at(Ng + 1) - tail_at(Ng) + net_at(Ng + 1) - net_at(Ng)


def system_batch(batch):
    """The batch with one framework per system (framework_of = 1..nsys): each system's framework
    tables copied, so that the FP32 path's spatial bins and tiles never mix systems. The batch
    itself when it already has that form. Cached on the batch."""
    fwo = np.asarray(batch.framework_of, dtype=np.int64) - 1
    if batch.nframeworks() == batch.nsys and np.array_equal(fwo, np.arange(batch.nsys)):
        return batch
    cached = getattr(batch, "_system_batch", None)
    if cached is not None:
        return cached
    new = copy.copy(batch)
    ao = np.asarray(batch.atom_offsets, dtype=np.int64)
    ko = np.asarray(batch.k_offsets, dtype=np.int64)
    cgo = np.asarray(batch.cellgrid_offsets, dtype=np.int64)
    N, nt = len(batch.guest_types), len(batch.sigma)

    def ragged(x, off):
        return np.concatenate([x[off[f]:off[f + 1]] for f in fwo]) if len(fwo) else x[:0]

    def offsets(off):
        return np.concatenate([[0], np.cumsum([off[f + 1] - off[f] for f in fwo])])

    new.positions = np.ascontiguousarray(ragged(batch.positions, ao))
    new.types = ragged(np.asarray(batch.types), ao)
    new.charges = ragged(np.asarray(batch.charges), ao)
    new.perm = ragged(np.asarray(batch.perm), ao)
    new.atom_offsets = offsets(ao).astype(batch.atom_offsets.dtype)
    new.ks = ragged(batch.ks, ko)
    new.kprefactor = ragged(batch.kprefactor, ko)
    new.Shost = ragged(batch.Shost, ko)
    new.kcoeffs = ragged(batch.kcoeffs, ko)
    new.k_offsets = offsets(ko).astype(batch.k_offsets.dtype)
    new.cell_offsets = ragged(np.asarray(batch.cell_offsets), cgo)
    new.cellgrid_offsets = offsets(cgo).astype(batch.cellgrid_offsets.dtype)
    for name in ("cells", "invcells", "volumes", "alphas", "constant_offset", "self_term_halfrange", "bs", "ncells"):
        setattr(new, name, np.asarray(getattr(batch, name))[fwo].copy())
    new.kmin = np.asarray(batch.kmin).reshape(-1, N * nt)[fwo].reshape(-1).copy()
    new.framework_of = np.arange(1, batch.nsys + 1, dtype=batch.framework_of.dtype)
    new._device = {}
    new._desc = None
    new._rejection = {}
    new._system_batch = None
    batch._system_batch = new
    return new


def widom_chain(batch, state, guest, ff, *, T, n_widom_per_cycle, seed=0, cycle=0, backend=None, insertions=None):
    """One cycle of test insertions into `state`'s configuration (widom_chain_kernel!,
    src/nvt.jl:85-124): n_widom_per_cycle insertions per system, assigned round-robin
    (run = 1, src/nvt.jl:228-233), no hard-core rejection. The poses are the counter-based stream
    keyed by (seed, system, k) with k continuing across cycles (cycle c takes
    k = c n_widom_per_cycle + 1, ...), so with no guests anywhere the cycles together are exactly
    widom_singlephase(batch, guest; ninsert = nsys n_widom_per_cycle n_cycles, run = 1) on the
    same batch. Returns per system (Σ W, Σ ΔU W, count) of the cycle, FP64; `insertions` (a dict)
    receives per-insertion dU and poses in system-major order."""
    if not int(n_widom_per_cycle) >= 1:
        raise ArgumentError(f"n_widom_per_cycle={n_widom_per_cycle} must be >= 1")
    if not int(cycle) >= 0:
        raise ArgumentError(f"cycle={cycle} must be >= 0")
    _check_guest(batch, guest, "widom_chain")
    if not batch.fullk:
        raise ArgumentError("widom_chain needs a FrameworkBatch built with fullk=true")
    if batch.T != np.float32:
        raise ArgumentError("widom_chain runs the FP32 path: build the batch from Float32 frameworks")
    if state.nsys != batch.nsys:
        raise DimensionMismatch(f"state has {state.nsys} systems, batch {batch.nsys}")
    nsys = batch.nsys
    nper = int(n_widom_per_cycle)
    T = float(T.magnitude) if hasattr(T, "magnitude") else float(T)
    kT = float(batch.T(KB * T))
    sb = system_batch(batch)
    backend = backend or default_backend()
    ctx = backend.ctx
    dev = sb.device(ctx)
    const = np.array([insertion_constant_term(ff, batch, guest, s, state.nguests(s)) for s in range(nsys)])
    Sk, goff, sites = state.chain_inputs(guest)
    chain = _lib.ChainArgs(_lib.ptr(Sk) if Sk.size else None, _lib.ptr(const), _lib.ptr(goff), _lib.ptr(sites),
                           int(cycle) * nper)
    n = nsys * nper
    args = _lib.WidomArgs()
    args.kT, args.ninsert, args.seed = kT, n, int(seed) & (2**64 - 1)
    args.nblocks, args.run, args.reject = 1, 1, 0
    args.rho2, args.reach0 = None, None
    args.segment_begin, args.segment_end = 0, 0
    args.chain = _lib.ctypes.pointer(chain)
    lse, sw, suw = np.zeros(nsys), np.zeros(nsys), np.zeros(nsys)
    cnt = np.zeros(nsys, dtype=np.int64)
    sums = _lib.BlockSums(_lib.ptr(lse), _lib.ptr(sw), _lib.ptr(suw), _lib.ptr(cnt), None)
    out = None
    if insertions is not None:
        insertions["dU"] = np.full(n, np.nan)
        insertions["flags"] = np.zeros(n, dtype=np.uint8)
        insertions["poses"] = np.zeros((n, 7))
        out = _lib.InsertionOut(_lib.ptr(insertions["dU"]), _lib.ptr(insertions["flags"]), _lib.ptr(insertions["poses"]))
    ctx.check(_lib.lib().pa_widom(ctx.handle, dev.handle, args, sums, out), "pa_widom (loaded configuration)")
    W, UW = block_sums(lse, sw, suw)
    return W, UW, cnt


def widom_along_chain(batch, states, guest, ff, *, T, n_widom_per_cycle, seed=0, backend=None):
    """Widom statistics along a chain: for each cycle's configuration in `states` (in order),
    n_widom_per_cycle insertions per system (widom_chain), then WidomResult's reduction per system
    with one block per cycle (src/nvt.jl:336-345: successive cycles are correlated, so cycles, not
    insertions, are the blocks). Needs at least two cycles."""
    states = list(states)
    if len(states) < 2:
        raise ArgumentError(f"{len(states)} cycles: at least two are needed for a standard error")
    T = float(T.magnitude) if hasattr(T, "magnitude") else float(T)
    kT = float(batch.T(KB * T))
    nsys = batch.nsys
    sW = np.zeros((nsys, len(states)))
    sUW = np.zeros((nsys, len(states)))
    n = np.zeros((nsys, len(states)), dtype=np.int64)
    for c, st in enumerate(states):
        W, UW, cnt = widom_chain(batch, st, guest, ff, T=T, n_widom_per_cycle=n_widom_per_cycle, seed=seed, cycle=c,
                                 backend=backend)
        sW[:, c], sUW[:, c], n[:, c] = W, UW, cnt
    Vf = batch.volumes.astype(batch.T).astype(np.float64)
    return [_reduce(sW[s], sUW[s], n[s], kT, Vf[int(batch.framework_of[s]) - 1], s + 1) for s in range(nsys)]
