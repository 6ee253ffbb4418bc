"""widom: Widom test-particle insertion on the B200 (src/widom.jl).

The host keeps the reference's validation, rejection tables and block reduction; the library
(libpureadsorb_b200.so) runs the whole insertion loop on the device.
"""
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .constants import KB
from .errors import ArgumentError
from .reject import theta_F


@dataclass(frozen=True)
class WidomResult:
    """Per-system result, every field FP64 (src/widom.jl:19-28): mu_ex (eV), K_H (A^3/eV) and
    q_st = kT - <dU W>/<W> (eV) with their block standard errors."""

    mu_ex: float
    mu_ex_err: float
    K_H: float
    K_H_err: float
    q_st: float
    q_st_err: float
    nsamples: int
    nblocks: int


def sys_of_index(g, run, nsys):
    """1-based system of 1-based global insertion index g (src/widom.jl:34)."""
    return ((g - 1) // run) % nsys + 1


def default_run(ninsert, nsys):
    """clamp((ninsert ÷ nsys) ÷ 4, 1, 256) (src/widom.jl:39)."""
    return min(max((ninsert // nsys) // 4, 1), 256)


def system_counts(ninsert, nsys, run):
    """Exact per-system insertion counts under the run-length assignment (src/widom.jl:44-53)."""
    q, rem = divmod(ninsert, run)
    full, hi = divmod(q, nsys)
    ns = [full * run] * nsys
    for r in range(hi):
        ns[r] += run
    if rem > 0:
        ns[q % nsys] += rem
    return ns


def boltzmann_weight(dU, kT):
    """(W, dU*W) in FP64, dU*W forced to 0 when W underflows (src/widom.jl:80-84)."""
    dU64, kT64 = float(dU), float(kT)
    w = math.exp(-dU64 / kT64) if -dU64 / kT64 < 709.782712893384 else math.inf
    return w, (0.0 if w == 0 else dU64 * w)


def build_rejection_tables(batch, kT, ctx=None):
    """Rejection radii rho2 (nsys*N*ntypes) and phase-0 stencil half-widths reach0 (nsys x 3) for
    one call (src/widom.jl:202-253), computed by the library's host code (pa_rejection_tables),
    or, given a context, with the root searches on the device through the batch's upload to it
    (pa_batch_rejection_tables; the same values bit for bit). The summation-error term uses eps of
    the batch's float type; theta is theta_F(Float64) because weights accumulate in FP64. Cached
    on the batch per (kT, eps)."""
    key = (float(kT), float(np.finfo(batch.T).eps))
    cache = getattr(batch, "_rejection", None)
    if cache is not None and key in cache:
        return cache[key]
    N = len(batch.guest_types)
    nt = len(batch.sigma)
    bs = np.ascontiguousarray(batch.bs, dtype=np.float64)
    kmin = np.ascontiguousarray(batch.kmin, dtype=np.float64)
    eps_F = float(np.finfo(batch.T).eps)
    if ctx is not None:
        rho2, reach0, bad_s = batch.device(ctx).rejection_tables(bs, kmin, kT, eps_F, batch.nsys, N, nt)
        st = _lib.PA_OK if bad_s == 0 else _lib.PA_ERR_ARG
    else:
        d, keep = batch.desc()
        rho2 = np.zeros(batch.nsys * N * nt)
        reach0 = np.zeros((batch.nsys, 3), dtype=np.int32)
        bad = _lib.ctypes.c_int32(0)
        st = _lib.lib().pa_rejection_tables(_lib.ctypes.byref(d), _lib.ptr(bs), _lib.ptr(kmin), float(kT), eps_F,
                                            _lib.ptr(rho2), _lib.ptr(reach0), _lib.ctypes.byref(bad))
        bad_s = bad.value
    if st != _lib.PA_OK:
        s = bad_s
        raise ArgumentError(f"build_rejection_tables: system {s} has no valid rejection radius (margin <= 0 or a "
                            f"root search failed; kT={kT}, theta_F={float(theta_F(np.float64))})")
    rho2.flags.writeable = False
    reach0.flags.writeable = False
    if cache is not None:
        cache[key] = (rho2, reach0)
    return rho2, reach0


def _reduce(sW, sUW, n, kT, V, s):
    """Block means, delta-method errors -> WidomResult; throws on non-finite sums or mu_ex/q_st
    (src/widom.jl:451-492). s is the 1-based system index used in messages."""
    return _reduce_rows(np.asarray(sW, dtype=np.float64)[None, :], np.asarray(sUW, dtype=np.float64)[None, :],
                        np.asarray(n)[None, :], kT, np.array([float(V)]), first=s)[0]


def _div(a, b):
    """a / b on Python floats with IEEE semantics for b == 0 (inf or nan instead of an exception)."""
    if b != 0:
        return a / b
    if a == 0 or math.isnan(a):
        return math.nan
    return math.copysign(math.inf, a) * math.copysign(1.0, b)


def _reduce_rows(sW, sUW, n, kT, V, first=1):
    """_reduce for every row (system) of the nsys x nblocks block sums at once: the block
    statistics as array operations over all systems, then the checks and the result of each
    system in order (the first failing system raises, as a loop of _reduce would)."""
    nsys, nb = sW.shape
    kT64 = float(kT)
    ntot = n.sum(axis=1)
    with np.errstate(all="ignore"):
        mW = sW / n
        mUW = sUW / n
        W = sW.sum(axis=1) / ntot
        UW = sUW.sum(axis=1) / ntot
        dW = mW - W[:, None]
        dUW = mUW - UW[:, None]
        varW = (dW * dW).sum(axis=1) / (nb - 1)
        varUW = (dUW * dUW).sum(axis=1) / (nb - 1)
        cov = (dW * dUW).sum(axis=1) / (nb - 1)
        semW = np.sqrt(varW / nb)
    empty = (n <= 0).any(axis=1).tolist()
    W, UW, varW, varUW, cov, semW = W.tolist(), UW.tolist(), varW.tolist(), varUW.tolist(), cov.tolist(), semW.tolist()
    ntot, V = ntot.tolist(), np.asarray(V, dtype=np.float64).tolist()
    out = []
    for r in range(nsys):
        s = first + r
        if empty[r]:
            raise ArgumentError(f"block {int(np.argmin(n[r] > 0)) + 1} of {nb} has zero samples")
        w, uw = W[r], UW[r]
        if not (math.isfinite(w) and math.isfinite(uw)):
            raise ArgumentError(f"system {s}: Boltzmann accumulation overflowed Float64 (W={w}, UW={uw}); an "
                                "insertion energy below about -709·kT was sampled")
        ratio = uw / w if w != 0 else (math.nan if uw == 0 else math.copysign(math.inf, uw))
        var_ratio = 0.0 if uw == 0 else ratio * ratio * (_div(varUW[r], uw * uw) + _div(varW[r], w * w) -
                                                          2 * _div(cov[r], uw * w)) / nb
        mu_ex = -kT64 * math.log(w) if w > 0 else math.inf
        q_st = kT64 - ratio
        for name, v in (("mu_ex", mu_ex), ("q_st", q_st)):
            if not math.isfinite(v):
                raise ArgumentError(f"system {s}: {name} = {v} is not finite")
        mu_err = kT64 * semW[r] / w if w != 0 else math.inf
        out.append(WidomResult(mu_ex, mu_err, V[r] * w / kT64, V[r] * semW[r] / kT64, q_st,
                               math.sqrt(max(var_ratio, 0.0)) if not math.isnan(var_ratio) else math.nan,
                               int(ntot[r]), nb))
    return out


class B200Backend:
    """The device `backend` of widom: one CUDA device context of the library. Plays the role of
    the KernelAbstractions backend object the reference takes (src/widom.jl:298-301). With
    device_tables=True each call's rejection radii are computed on the device
    (pa_batch_rejection_tables, equal to the host's), which pays off for batches of many systems."""

    def __init__(self, device=0, device_tables=False):
        self.device = device
        self.device_tables = bool(device_tables)
        self._ctx = None

    @property
    def ctx(self):
        if self._ctx is None:
            self._ctx = _lib.Context(self.device)
        return self._ctx


_default_backend = None


def default_backend():
    global _default_backend
    if _default_backend is None:
        _default_backend = B200Backend(0)
    return _default_backend


def _validate(batch, guest, ninsert, chunk, nblocks, run):
    if not nblocks >= 2:
        raise ArgumentError(f"nblocks={nblocks}: at least two blocks are needed for a standard error")
    if not chunk >= 1:
        raise ArgumentError(f"chunk={chunk} must be ≥ 1")
    if not (np.array_equal(guest.types, batch.guest_types_orig) and np.array_equal(guest.sites, batch.guest_sites_orig)
            and np.array_equal(guest.charges, batch.guest_charges_orig)):
        raise ArgumentError(
            "guest passed to widom does not match the guest FrameworkBatch was built with: "
            f"passed types={list(guest.types)}, sites={guest.sites.tolist()}, charges={list(guest.charges)}; "
            f"batch types={list(batch.guest_types_orig)}, sites={batch.guest_sites_orig.tolist()}, "
            f"charges={list(batch.guest_charges_orig)}; build a new FrameworkBatch for a different guest")
    nsys = batch.nsys
    per = ninsert // nsys
    if run is None:
        runlen = default_run(ninsert, nsys)
    else:
        if not run >= 1:
            raise ArgumentError(f"run={run} must be ≥ 1")
        if not run <= per:
            raise ArgumentError(f"run={run} must be ≤ per={per} (= ninsert ÷ nsys)")
        runlen = int(run)
    ns = system_counts(ninsert, nsys, runlen)
    if min(ns) < 2 * nblocks:
        raise ArgumentError(f"ninsert={ninsert}, nsys={nsys}, run={runlen}: system {int(np.argmin(ns)) + 1} gets only "
                            f"{min(ns)} samples, need at least 2·nblocks = {2 * nblocks} per system")
    batch.check_axes()
    return runlen, ns


def _widom(batch, guest, *, reject, T, ninsert, backend=None, seed=0, chunk=2**16, nblocks=10, run=None,
           insertions=None, segment_range=None, segments_out=None, grad_sums=None):
    """The widom call with optional extras: `insertions` (a dict) receives per-insertion dU,
    flags and poses in system-major sample order; `segment_range` (begin, end) restricts the call
    to a contiguous range of PA_SEGMENT-insertion segments (a shard of a multi-GPU job), whose
    segment triplets go into `segments_out` (an array of 3 per job segment); `grad_sums` (a
    _lib.GradSums over caller-owned arrays) makes the call pa_widom_grad, which also fills it."""
    ninsert = int(ninsert)
    runlen, ns = _validate(batch, guest, ninsert, chunk, nblocks, run)
    T = float(T.magnitude) if hasattr(T, "magnitude") else float(T)
    kT = float(batch.T(KB * T))
    backend = backend or default_backend()
    ctx = backend.ctx
    dev = batch.device(ctx)
    rho2, reach0 = (build_rejection_tables(batch, kT, ctx if getattr(backend, "device_tables", False) else None)
                    if reject else (None, None))
    rho2c = None if rho2 is None else np.ascontiguousarray(rho2)
    reach0c = None if reach0 is None else np.ascontiguousarray(reach0.reshape(-1))
    args = _lib.WidomArgs()
    args.kT, args.ninsert, args.seed = kT, ninsert, int(seed) & (2**64 - 1)
    args.nblocks, args.run, args.reject = int(nblocks), runlen, 1 if reject else 0
    args.rho2, args.reach0 = _lib.ptr(rho2c), _lib.ptr(reach0c)
    args.segment_begin, args.segment_end = (0, 0) if segment_range is None else segment_range
    nsys = batch.nsys
    lse = np.zeros(nsys * nblocks)
    sw = np.zeros(nsys * nblocks)
    suw = np.zeros(nsys * nblocks)
    cnt = np.zeros(nsys * nblocks, dtype=np.int64)
    sums = _lib.BlockSums(_lib.ptr(lse), _lib.ptr(sw), _lib.ptr(suw), _lib.ptr(cnt), _lib.ptr(segments_out))
    out = None
    if insertions is not None:
        insertions["dU"] = np.full(ninsert, np.nan)
        insertions["flags"] = np.zeros(ninsert, dtype=np.uint8)
        insertions["poses"] = np.zeros((ninsert, 7))
        out = _lib.InsertionOut(_lib.ptr(insertions["dU"]), _lib.ptr(insertions["flags"]),
                                _lib.ptr(insertions["poses"]))
    if grad_sums is not None:
        ctx.check(_lib.lib().pa_widom_grad(ctx.handle, dev.handle, args, sums, grad_sums, out), "pa_widom_grad")
    else:
        ctx.check(_lib.lib().pa_widom(ctx.handle, dev.handle, args, sums, out), "pa_widom")
    if segment_range is not None:
        return lse, sw, suw, cnt
    return _results(batch, kT, nblocks, lse, sw, suw, cnt)


def block_sums(lse, sw, suw):
    """Σ W and Σ dU W per block from the library's (max, scaled sums) representation."""
    neg = np.isneginf(lse)
    with np.errstate(over="ignore", invalid="ignore"):
        scale = np.exp(lse) if not neg.any() else np.where(neg, 0.0, np.exp(np.where(neg, 0.0, lse)))
        return scale * sw, scale * suw


def lnkh_from_sums(batch, kT, nblocks, lse, sw, suw, cnt):
    """ln K_H = ln(V <W> / kT) of every system from a call's raw block sums, -inf for a system
    whose every weight is zero (no accessible volume), where widom's reduction throws."""
    sW, _ = block_sums(lse, sw, suw)
    W = sW.reshape(batch.nsys, nblocks).sum(axis=1) / np.asarray(cnt).reshape(batch.nsys, nblocks).sum(axis=1)
    Vf = batch.volumes.astype(batch.T).astype(np.float64)[np.asarray(batch.framework_of, dtype=np.int64) - 1]
    with np.errstate(divide="ignore"):
        return np.log(Vf) + np.log(W) - math.log(float(kT))


def _results(batch, kT, nblocks, lse, sw, suw, cnt):
    sW, sUW = block_sums(lse, sw, suw)
    Vf = batch.volumes.astype(batch.T).astype(np.float64)[np.asarray(batch.framework_of, dtype=np.int64) - 1]
    return _reduce_rows(sW.reshape(batch.nsys, nblocks), sUW.reshape(batch.nsys, nblocks),
                        np.asarray(cnt).reshape(batch.nsys, nblocks), kT, Vf)


def widom(batch, guest, *, T, ninsert, backend=None, seed=0, chunk=2**16, nblocks=10, run=None):
    """Widom test-particle insertion at temperature T (K): ninsert random poses over the batch's
    systems give <exp(-dU/kT)> split into nblocks blocks, reduced to one WidomResult per system
    (src/widom.jl:255-290). Insertion g goes to system mod1((g-1)÷run+1, nsys); run defaults to
    clamp((ninsert÷nsys)÷4, 1, 256). Poses are drawn on the device from the counter-based stream
    keyed by (seed, system, per-system index), so results do not depend on `chunk` (accepted and
    validated for signature compatibility: the device path stages no poses through the host).
    Hard-core rejection (phase 0) removes only insertions whose FP64 weight is provably zero."""
    return _widom(batch, guest, reject=True, T=T, ninsert=ninsert, backend=backend, seed=seed, chunk=chunk,
                  nblocks=nblocks, run=run)


def widom_singlephase(batch, guest, **kwargs):
    """widom without hard-core rejection: every insertion's energy is computed (src/widom.jl:296)."""
    return _widom(batch, guest, reject=False, **kwargs)
