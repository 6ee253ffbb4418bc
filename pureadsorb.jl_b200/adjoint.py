"""Gradients of ln K_H: the adjoint of widom over the force field and the framework charges.

PureAdsorb.jl has no gradients (no AD, no rrule). This module adds them behind the same
FrameworkBatch/widom API. With W_i = exp(-ΔU_i/kT) over the call's insertions,

    d ln K_H / dθ = d ln <W> / dθ = -<W ∂ΔU/∂θ> / (kT <W>),

the derivative of the estimator itself at fixed poses (the counter-based stream makes the poses
independent of θ), so it equals a central finite difference of ln K_H with common random numbers
up to O(h^2). The library (pa_widom_grad) returns the weighted numerator sums with respect to
the batch's inputs: the (site type, host type) pair tables and the stored charges. This module
adds what lives in the framework's constant offset (the analytic tail correction,
src/forcefield.jl:103-124, and the net-charge term, src/batch.jl:404-406), maps the pair tables
onto per-type Lorentz-Berthelot parameters and the stored atoms back to each framework's own atom
order. `lnKH_function` wraps everything as a torch.autograd.Function, the Python analogue of a
ChainRulesCore rrule.
"""
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .constants import KB, KE
from .forcefield import type_parameters
from .widom import _results, _widom, default_backend, lnkh_from_sums


@dataclass
class WidomGrad:
    """d ln K_H / dθ of one system. epsilon and sigma: per force-field type (ff.names order,
    1/eV and 1/Å), from every survivor's LJ sums kept by the forward pass; charges: per atom of
    the system's framework in the framework's own atom order (1/e), None when the charge
    derivatives were not asked for; recomputed: insertions the charge pass recomputed (0 without
    charges); sum_w and xmax: the weight sums."""

    epsilon: np.ndarray
    sigma: np.ndarray
    charges: np.ndarray
    recomputed: int
    sum_w: float
    xmax: float


def system_offsets(batch):
    """Per-system atom and k-vector counts (the layout of pa_grad_sums' per-atom and per-k arrays)."""
    fw = np.asarray(batch.framework_of, dtype=np.int64) - 1
    ao, ko = np.asarray(batch.atom_offsets, dtype=np.int64), np.asarray(batch.k_offsets, dtype=np.int64)
    return ao[fw + 1] - ao[fw], ko[fw + 1] - ko[fw]


def _lj_grads(batch, ff, systems, sums, kT):
    """The ε and σ parts of d ln K_H / dθ for the given systems (0-based) at once, from their
    adjoint sums: the device's (site, compact type) sums mapped onto the force field's pair tables,
    plus the tail correction's pair-table derivatives, then Lorentz-Berthelot's chain rule.
    Returns (g_epsilon, g_sigma, W), the first two of shape (len(systems), ntypes)."""
    beta = 1.0 / float(kT)
    systems = np.asarray(systems, dtype=np.int64)
    ns = len(systems)
    W = np.array([float(p["sum_w"]) for p in sums])
    nff = len(ff.names)
    c2o = np.asarray(batch.compact_to_orig, dtype=np.int64) - 1
    gt = np.asarray(batch.guest_types, dtype=np.int64) - 1
    fws = np.asarray(batch.framework_of, dtype=np.int64)[systems] - 1
    V = np.asarray(batch.volumes, dtype=np.float64)[fws]
    # <∂ΔU/∂(pair table entry)> on the force field's full tables
    dS = np.zeros((ns, nff, nff))
    dE = np.zeros((ns, nff, nff))
    d_eps = np.stack([np.asarray(p["d_epsilon"], dtype=np.float64).reshape(len(gt), -1) for p in sums])
    d_sig = np.stack([np.asarray(p["d_sigma"], dtype=np.float64).reshape(len(gt), -1) for p in sums])
    with np.errstate(divide="ignore", invalid="ignore"):
        for a in range(len(gt)):
            i = c2o[gt[a]]
            dE[:, i, c2o] += d_eps[:, a, :] / W[:, None]
            dS[:, i, c2o] += d_sig[:, a, :] / W[:, None]
    # the tail correction shifts every insertion's ΔU by the same amount
    if ff.tail:
        ao = np.asarray(batch.atom_offsets, dtype=np.int64)
        types = np.asarray(batch.types, dtype=np.int64) - 1
        cnt = {f: np.bincount(c2o[types[ao[f]:ao[f + 1]]], minlength=nff).astype(np.float64) for f in set(fws.tolist())}
        counts = np.stack([cnt[f] for f in fws.tolist()])
        gc = np.bincount(np.asarray(batch.guest_types_orig, dtype=np.int64) - 1, minlength=nff).astype(np.float64)
        M = 2 * counts[:, :, None] * gc[None, None, :] + (gc[:, None] * gc[None, :])[None]
        sg, ep, rc = ff.sigma, ff.epsilon, ff.cutoff
        f = (8 * math.pi / 3 / V)[:, None, None]
        dE = dE + f * M * (sg**12 / (3 * rc**9) - sg**6 / rc**3)
        dS = dS + f * M * ep * (4 * sg**11 / rc**9 - 6 * sg**5 / rc**3)
    # Lorentz-Berthelot (pair_to_type_grad over every system at once)
    _, eps_t = type_parameters(ff)
    g_sig = 0.5 * (dS.sum(axis=2) + dS.sum(axis=1))
    wE = dE * ff.epsilon
    with np.errstate(divide="ignore", invalid="ignore"):
        g_eps = (wE.sum(axis=2) + wE.sum(axis=1)) / (2 * eps_t)
    return -beta * g_eps, -beta * g_sig, W


def _charge_grad(batch, s, sums, W, kT):
    """The charge part of d ln K_H / dθ of system s: real-space and reciprocal parts from the
    device, plus the net-charge term of the constant offset, KE * (-pi/(2 V alpha^2)) *
    ((Qh + Qg)^2 - Qh^2), whose derivative is KE * (-pi Qg / (V alpha^2)) for every host atom;
    in the framework's own atom order."""
    fw = int(batch.framework_of[s]) - 1
    a0, a1 = int(batch.atom_offsets[fw]), int(batch.atom_offsets[fw + 1])
    V, alpha = float(batch.volumes[fw]), float(batch.alphas[fw])
    Qg = float(np.sum(batch.guest_charges_orig))
    with np.errstate(divide="ignore", invalid="ignore"):
        dq = np.asarray(sums["d_charge"], dtype=np.float64) / W + KE * (-math.pi * Qg / (V * alpha**2))
    g_q = np.empty(a1 - a0)
    g_q[np.asarray(batch.perm[a0:a1], dtype=np.int64)] = -(1.0 / float(kT)) * dq
    return g_q


def assemble_all(batch, ff, sums, kT, systems=None):
    """d ln K_H / dθ of every system (or of `systems`, 0-based) from its adjoint sums (xmax, sum_w,
    d_epsilon and d_sigma per (site, compact type), d_charge per stored atom or None): the host
    half of the adjoint, the LJ part vectorised over the systems."""
    systems = list(range(batch.nsys)) if systems is None else list(systems)
    g_eps, g_sig, W = _lj_grads(batch, ff, systems, sums, kT)
    out = []
    for r, (s, p) in enumerate(zip(systems, sums)):
        g_q = None if p.get("d_charge") is None else _charge_grad(batch, s, p, W[r], kT)
        out.append(WidomGrad(g_eps[r], g_sig[r], g_q, int(p.get("recomputed", 0)), float(W[r]), float(p["xmax"])))
    return out


def assemble(batch, ff, s, sums, kT):
    """d ln K_H / dθ of system s (0-based) from its adjoint sums (xmax, sum_w, d_epsilon and
    d_sigma per (site, compact type), d_charge per stored atom or None): the host half of the
    adjoint."""
    return assemble_all(batch, ff, [sums], kT, systems=[s])[0]


def fold_replicas(g, natoms_unit):
    """Gradient with respect to the charges of a unit cell from the gradient with respect to the
    charges of its replication (`replicate` orders atoms replica-major, src/structure.jl:79-92):
    every replica of unit atom u carries the same charge q_u."""
    g = np.asarray(g, dtype=np.float64)
    return g.reshape(-1, natoms_unit).sum(axis=0)


def grad_sums(batch, guest, *, T, ninsert, backend=None, seed=0, chunk=2**16, nblocks=10, run=None, window=0.0,
              segment_range=(0, 0), segments_out=None, charges=True):
    """One pa_widom_grad call. Returns (kT, (lse, sw, suw, cnt), sums): the call's raw block sums
    and, per system, a dict of its adjoint sums (xmax, sum_w, d_epsilon and d_sigma per (site,
    compact type), d_charge per stored atom or None with charges=False, recomputed).
    segment_range restricts the call to a shard of the job (see combine_sums). charges=False
    skips the charge derivatives on the device (the per-pair charge terms and G_k)."""
    nsys = batch.nsys
    N = len(batch.guest_types)
    nt = len(batch.sigma)
    nat, nkv = system_offsets(batch)
    buf = dict(xmax=np.zeros(nsys), sum_w=np.zeros(nsys), d_epsilon=np.zeros(nsys * N * nt),
               d_sigma=np.zeros(nsys * N * nt), d_charge=np.zeros(max(1, int(nat.sum()))))
    gs = _lib.GradSums(_lib.ptr(buf["xmax"]), _lib.ptr(buf["sum_w"]), _lib.ptr(buf["d_epsilon"]),
                       _lib.ptr(buf["d_sigma"]), _lib.ptr(buf["d_charge"]), None, float(window), 0,
                       0 if charges else 1)
    T = float(T.magnitude) if hasattr(T, "magnitude") else float(T)
    kT = float(batch.T(KB * T))
    raw = _widom(batch, guest, reject=True, T=T, ninsert=ninsert, backend=backend, seed=seed, chunk=chunk,
                 nblocks=nblocks, run=run, segment_range=segment_range, segments_out=segments_out, grad_sums=gs)
    aoff = np.concatenate([[0], np.cumsum(nat)]).astype(np.int64)
    sums = [dict(xmax=buf["xmax"][s], sum_w=buf["sum_w"][s], d_epsilon=buf["d_epsilon"].reshape(nsys, N, nt)[s],
                 d_sigma=buf["d_sigma"].reshape(nsys, N, nt)[s],
                 d_charge=buf["d_charge"][aoff[s]:aoff[s + 1]] if charges else None,
                 recomputed=gs.recomputed) for s in range(nsys)]
    return kT, raw, sums


def combine_sums(shards):
    """One system's adjoint sums of a whole job from the sums of disjoint shards of it (several
    GPUs, each with its own segment range and so its own shift xmax): every shard is rescaled to
    the largest shift and the shards are added in the given order."""
    xm = max(float(p["xmax"]) for p in shards)
    out = dict(xmax=xm, recomputed=sum(int(p.get("recomputed", 0)) for p in shards))
    for k in ("sum_w", "d_epsilon", "d_sigma", "d_charge"):
        if any(p.get(k) is None for p in shards):
            out[k] = None
            continue
        acc = None
        for p in shards:
            f = math.exp(float(p["xmax"]) - xm) if np.isfinite(p["xmax"]) else 0.0
            v = f * np.asarray(p[k], dtype=np.float64)
            acc = v if acc is None else acc + v
        out[k] = acc
    return out


def widom_grad(batch, guest, ff, *, T, ninsert, backend=None, seed=0, chunk=2**16, nblocks=10, run=None,
               window=0.0, reduce=True, charges=True):
    """widom plus d ln K_H / dθ for every system: returns (results, grads), grads[s] a WidomGrad.
    θ: the per-type LJ ε and σ of `ff` (which must be the force field the batch was built from)
    and the charges of each framework's atoms. The batch must be FP32 (the adjoint walks the FP32
    path's neighbour lists). Insertions whose weight is below exp(-window) times their system's
    largest are left out of the sums (0 selects 50). With reduce=False the first element is
    ln K_H per system from the raw sums instead of the WidomResults (-inf, and NaN gradients,
    for a system without accessible volume, where the reduction throws). With charges=False only
    the ε and σ derivatives are formed (WidomGrad.charges is None), which skips the per-pair
    charge terms of the adjoint pass."""
    kT, (lse, sw, suw, cnt), sums = grad_sums(batch, guest, T=T, ninsert=ninsert, backend=backend, seed=seed,
                                              chunk=chunk, nblocks=nblocks, run=run, window=window, charges=charges)
    results = _results(batch, kT, nblocks, lse, sw, suw, cnt) if reduce else \
        lnkh_from_sums(batch, kT, nblocks, lse, sw, suw, cnt)
    return results, assemble_all(batch, ff, sums, kT)
