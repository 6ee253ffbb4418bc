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
from .forcefield import pair_to_type_grad, tail_delta_pair_grad
from .widom import _results, _widom, default_backend, lnkh_from_sums


@dataclass
class WidomGrad:
    """d ln K_H / dθ of one system. epsilon and sigma: per force-field type (ff.names order,
    1/eV and 1/Å); charges: per atom of the system's framework in the framework's own atom order
    (1/e); recomputed: insertions the adjoint pass recomputed; sum_w and xmax: the weight sums."""

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


def assemble(batch, ff, s, sums, kT):
    """d ln K_H / dθ of system s (0-based) from its adjoint sums (xmax, sum_w, d_epsilon and
    d_sigma per (site, compact type), d_charge per stored atom): the host half of the adjoint."""
    beta = 1.0 / float(kT)
    W = float(sums["sum_w"])
    nff = len(ff.names)
    c2o = np.asarray(batch.compact_to_orig, dtype=np.int64) - 1
    gt = np.asarray(batch.guest_types, dtype=np.int64) - 1
    fw = int(batch.framework_of[s]) - 1
    a0, a1 = int(batch.atom_offsets[fw]), int(batch.atom_offsets[fw + 1])
    V, alpha = float(batch.volumes[fw]), float(batch.alphas[fw])
    # <∂ΔU/∂(pair table entry)> on the force field's full tables
    dS = np.zeros((nff, nff))
    dE = np.zeros((nff, nff))
    d_eps = np.asarray(sums["d_epsilon"], dtype=np.float64).reshape(len(gt), -1)
    d_sig = np.asarray(sums["d_sigma"], dtype=np.float64).reshape(len(gt), -1)
    with np.errstate(divide="ignore", invalid="ignore"):
        for a in range(len(gt)):
            i = c2o[gt[a]]
            np.add.at(dE, (i, c2o), d_eps[a] / W)
            np.add.at(dS, (i, c2o), d_sig[a] / W)
    # the tail correction shifts every insertion's ΔU by the same amount
    counts = np.bincount(c2o[np.asarray(batch.types[a0:a1], dtype=np.int64) - 1], minlength=nff)
    gcounts = np.bincount(np.asarray(batch.guest_types_orig, dtype=np.int64) - 1, minlength=nff)
    tS, tE = tail_delta_pair_grad(ff, counts, gcounts, V)
    g_sig, g_eps = pair_to_type_grad(ff, dS + tS, dE + tE)
    # charges: real-space and reciprocal parts from the device, plus the net-charge term of the
    # constant offset, KE * (-pi/(2 V alpha^2)) * ((Qh + Qg)^2 - Qh^2), whose derivative is
    # KE * (-pi Qg / (V alpha^2)) for every host atom
    Qg = float(np.sum(batch.guest_charges_orig))
    with np.errstate(divide="ignore", invalid="ignore"):
        dq = np.asarray(sums["d_charge"], dtype=np.float64) / W + KE * (-math.pi * Qg / (V * alpha**2))
    g_q = np.empty(a1 - a0)
    g_q[np.asarray(batch.perm[a0:a1], dtype=np.int64)] = -beta * dq
    return WidomGrad(-beta * g_eps, -beta * g_sig, g_q, int(sums.get("recomputed", 0)), W, float(sums["xmax"]))


def fold_replicas(g, natoms_unit):
    """Gradient with respect to the charges of a unit cell from the gradient with respect to the
    charges of its replication (`replicate` orders atoms replica-major, src/structure.jl:79-92):
    every replica of unit atom u carries the same charge q_u."""
    g = np.asarray(g, dtype=np.float64)
    return g.reshape(-1, natoms_unit).sum(axis=0)


def grad_sums(batch, guest, *, T, ninsert, backend=None, seed=0, chunk=2**16, nblocks=10, run=None, window=0.0,
              segment_range=(0, 0), segments_out=None):
    """One pa_widom_grad call. Returns (kT, (lse, sw, suw, cnt), sums): the call's raw block sums
    and, per system, a dict of its adjoint sums (xmax, sum_w, d_epsilon and d_sigma per (site,
    compact type), d_charge per stored atom, recomputed). segment_range restricts the call to a
    shard of the job (see combine_sums)."""
    nsys = batch.nsys
    N = len(batch.guest_types)
    nt = len(batch.sigma)
    nat, nkv = system_offsets(batch)
    buf = dict(xmax=np.zeros(nsys), sum_w=np.zeros(nsys), d_epsilon=np.zeros(nsys * N * nt),
               d_sigma=np.zeros(nsys * N * nt), d_charge=np.zeros(max(1, int(nat.sum()))))
    gs = _lib.GradSums(_lib.ptr(buf["xmax"]), _lib.ptr(buf["sum_w"]), _lib.ptr(buf["d_epsilon"]),
                       _lib.ptr(buf["d_sigma"]), _lib.ptr(buf["d_charge"]), None, float(window), 0)
    T = float(T.magnitude) if hasattr(T, "magnitude") else float(T)
    kT = float(batch.T(KB * T))
    raw = _widom(batch, guest, reject=True, T=T, ninsert=ninsert, backend=backend, seed=seed, chunk=chunk,
                 nblocks=nblocks, run=run, segment_range=segment_range, segments_out=segments_out, grad_sums=gs)
    aoff = np.concatenate([[0], np.cumsum(nat)]).astype(np.int64)
    sums = [dict(xmax=buf["xmax"][s], sum_w=buf["sum_w"][s], d_epsilon=buf["d_epsilon"].reshape(nsys, N, nt)[s],
                 d_sigma=buf["d_sigma"].reshape(nsys, N, nt)[s], d_charge=buf["d_charge"][aoff[s]:aoff[s + 1]],
                 recomputed=gs.recomputed) for s in range(nsys)]
    return kT, raw, sums


def combine_sums(shards):
    """One system's adjoint sums of a whole job from the sums of disjoint shards of it (several
    GPUs, each with its own segment range and so its own shift xmax): every shard is rescaled to
    the largest shift and the shards are added in the given order."""
    xm = max(float(p["xmax"]) for p in shards)
    out = dict(xmax=xm, recomputed=sum(int(p.get("recomputed", 0)) for p in shards))
    for k in ("sum_w", "d_epsilon", "d_sigma", "d_charge"):
        acc = None
        for p in shards:
            f = math.exp(float(p["xmax"]) - xm) if np.isfinite(p["xmax"]) else 0.0
            v = f * np.asarray(p[k], dtype=np.float64)
            acc = v if acc is None else acc + v
        out[k] = acc
    return out


def widom_grad(batch, guest, ff, *, T, ninsert, backend=None, seed=0, chunk=2**16, nblocks=10, run=None,
               window=0.0, reduce=True):
    """widom plus d ln K_H / dθ for every system: returns (results, grads), grads[s] a WidomGrad.
    θ: the per-type LJ ε and σ of `ff` (which must be the force field the batch was built from)
    and the charges of each framework's atoms. The batch must be FP32 (the adjoint walks the FP32
    path's neighbour lists). Insertions whose weight is below exp(-window) times their system's
    largest are left out of the sums (0 selects 50). With reduce=False the first element is
    ln K_H per system from the raw sums instead of the WidomResults (-inf, and NaN gradients,
    for a system without accessible volume, where the reduction throws)."""
    kT, (lse, sw, suw, cnt), sums = grad_sums(batch, guest, T=T, ninsert=ninsert, backend=backend, seed=seed,
                                              chunk=chunk, nblocks=nblocks, run=run, window=window)
    results = _results(batch, kT, nblocks, lse, sw, suw, cnt) if reduce else \
        lnkh_from_sums(batch, kT, nblocks, lse, sw, suw, cnt)
    return results, [assemble(batch, ff, s, sums[s], kT) for s in range(batch.nsys)]
