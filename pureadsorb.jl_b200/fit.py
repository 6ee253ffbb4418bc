"""Force-field fitting with the adjoint: Adam on per-type LJ scale factors (no counterpart in the
reference, which has no gradients).

The parameters are scale factors x on the epsilon and sigma of chosen force-field types
(epsilon_t = x_t epsilon0_t, sigma_t = x_{k+t} sigma0_t). The objective is the mean squared error
of ln K_H over the batch's systems against target values,

    L(x) = mean_s (ln K_H(s; x) - target_s)^2,   dL/dx = mean_s 2 (ln K_H(s) - target_s) d ln K_H(s)/dx,

with d ln K_H / d(epsilon_t, sigma_t) from widom_grad. Every step uses the same seed, so every
step samples the same poses (common random numbers) and L is a deterministic function of x. Each
step updates only the LJ tables of the uploaded batch and recomputes the hard-core bounds on the
device (FrameworkBatch.with_forcefield with move_device and device_bounds), so geometry,
neighbour lists and structure factors are built once.
"""
import time
from dataclasses import dataclass, field

import numpy as np

from .adjoint import widom_grad
from .batch import FrameworkBatch
from .forcefield import ForceField, type_parameters
from .constants import KB
from .widom import _widom, lnkh_from_sums


def scaled_forcefield(ff, types, x):
    """ff with epsilon of `types` scaled by x[:k] and sigma by x[k:]."""
    sig, eps = type_parameters(ff)
    idx = np.array([ff.typeindex(t) - 1 for t in types])
    k = len(idx)
    eps[idx] *= np.asarray(x[:k], dtype=np.float64)
    sig[idx] *= np.asarray(x[k:], dtype=np.float64)
    return ForceField(ff.names, sig, eps, cutoff=ff.cutoff, tail=ff.tail)


def target_lnkh(fws, ff, guest, ewald, *, T, ninsert, seed, nblocks=10, backend=None, sk=None, self_term=None):
    """ln K_H of every framework from the plain FP64 path (the reference algorithm) at ff; -inf
    for a framework without accessible volume (every sampled weight zero)."""
    b64 = FrameworkBatch(fws, ff, guest, ewald, T=np.float64, sk=sk, self_term=self_term)
    lse, sw, suw, cnt = _widom(b64, guest, reject=True, T=T, ninsert=ninsert, seed=seed, nblocks=nblocks,
                               backend=backend, segment_range=(0, 0))
    kT = float(b64.T(KB * float(T)))
    out = lnkh_from_sums(b64, kT, nblocks, lse, sw, suw, cnt)
    b64.drop_device()
    return out


@dataclass
class FitResult:
    x: np.ndarray                                 # final scale factors (epsilon of types, then sigma)
    loss: list = field(default_factory=list)      # loss before each step's update
    ms: list = field(default_factory=list)        # wall milliseconds of each step
    xs: list = field(default_factory=list)        # x after each step


def fit_lj_scales(batch, guest, ff, types, targets, *, T, ninsert, steps=200, lr=1e-2, seed=0, nblocks=10,
                  backend=None, betas=(0.9, 0.999), adam_eps=1e-8, x0=None):
    """Adam (Kingma and Ba, 2015) on the 2 len(types) scale factors, one widom_grad call per step.
    `batch` must be an FP32 FrameworkBatch built with `ff`; `targets` holds one ln K_H per system.
    Systems whose target or current ln K_H is not finite (no accessible volume) are left out of
    the loss of that step."""
    k = len(types)
    idx = np.array([ff.typeindex(t) - 1 for t in types])
    sig0, eps0 = type_parameters(ff)
    x = np.ones(2 * k) if x0 is None else np.array(x0, dtype=np.float64)
    m = np.zeros(2 * k)
    v = np.zeros(2 * k)
    targets = np.asarray(targets, dtype=np.float64)
    out = FitResult(x.copy())
    b = batch
    for it in range(1, steps + 1):
        t0 = time.perf_counter()
        ffx = scaled_forcefield(ff, types, x)
        b = b.with_forcefield(ffx, move_device=True, device_bounds=True)
        lnk, grads = widom_grad(b, guest, ffx, T=T, ninsert=ninsert, backend=backend, seed=seed, nblocks=nblocks,
                                reduce=False, charges=False)
        use = np.isfinite(lnk) & np.isfinite(targets)
        r = lnk[use] - targets[use]
        g_eps = np.array([g.epsilon[idx] for g, u in zip(grads, use) if u]) * eps0[idx]
        g_sig = np.array([g.sigma[idx] for g, u in zip(grads, use) if u]) * sig0[idx]
        grad = np.concatenate([2 * (r[:, None] * g_eps).mean(axis=0), 2 * (r[:, None] * g_sig).mean(axis=0)])
        m = betas[0] * m + (1 - betas[0]) * grad
        v = betas[1] * v + (1 - betas[1]) * grad**2
        mhat = m / (1 - betas[0] ** it)
        vhat = v / (1 - betas[1] ** it)
        x = x - lr * mhat / (np.sqrt(vhat) + adam_eps)
        out.loss.append(float(np.mean(r**2)))
        out.ms.append((time.perf_counter() - t0) * 1e3)
        out.xs.append(x.copy())
    out.x = x
    return out


@dataclass
class Identifiability:
    """The loss's curvature at a point of the fit, from the adjoint Jacobian J (systems x scale
    factors) of ln K_H: the Gauss-Newton Hessian H = (2/n) J^T J, its eigenvalues (descending) and
    eigenvectors (columns), and, given reference scale factors, the parameter error split along
    those eigenvectors and the relative error of each type's eps sigma^6 (the dispersion
    coefficient, the combination ln K_H depends on most directly)."""
    eigenvalues: np.ndarray
    eigenvectors: np.ndarray
    error_along: np.ndarray = None       # |v_i . (x - x_ref)| per eigenvector
    loss_along: np.ndarray = None        # lambda_i (v_i . (x - x_ref))^2: its share of the loss
    eps_sigma6_rel_error: np.ndarray = None


def identifiability(batch, guest, ff, types, x, targets, *, T, ninsert, seed=0, nblocks=10, backend=None,
                    x_ref=None):
    """Identifiability at scale factors x (one widom_grad call): see Identifiability."""
    k = len(types)
    idx = np.array([ff.typeindex(t) - 1 for t in types])
    sig0, eps0 = type_parameters(ff)
    ffx = scaled_forcefield(ff, types, x)
    b = batch.with_forcefield(ffx, move_device=True, device_bounds=True)
    lnk, grads = widom_grad(b, guest, ffx, T=T, ninsert=ninsert, backend=backend, seed=seed, nblocks=nblocks,
                            reduce=False, charges=False)
    use = np.isfinite(lnk) & np.isfinite(np.asarray(targets, dtype=np.float64))
    J = np.array([np.concatenate([g.epsilon[idx] * eps0[idx], g.sigma[idx] * sig0[idx]])
                  for g, u in zip(grads, use) if u])
    H = 2.0 * J.T @ J / len(J)
    lam, V = np.linalg.eigh(H)
    order = np.argsort(-lam)
    out = Identifiability(lam[order], V[:, order])
    if x_ref is not None:
        d = np.asarray(x, dtype=np.float64) - np.asarray(x_ref, dtype=np.float64)
        proj = out.eigenvectors.T @ d
        out.error_along = np.abs(proj)
        out.loss_along = out.eigenvalues * proj**2
        xr = np.asarray(x_ref, dtype=np.float64)
        xx = np.asarray(x, dtype=np.float64)
        out.eps_sigma6_rel_error = np.abs(xx[:k] * xx[k:] ** 6 / (xr[:k] * xr[k:] ** 6) - 1.0)
    return out
