"""Host side of the fitting path: a batch re-derived for another force field equals a fresh build,
the hard-core bound's grouped bisections equal one bisection per atom, and the scaled force field
scales what it says."""
import math

import numpy as np
import pytest
from scipy.special import erfc


@pytest.fixture(scope="module")
def small(pa):
    return pa.synthetic.fitting(nfw=3, max_unit_atoms=150)


def test_with_forcefield_equals_fresh_build(pa, small):
    fws, ff, guest, ewald, prm = small
    b = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    ffx = pa.fit.scaled_forcefield(ff, prm["fitted_types"], prm["hidden"])
    new = b.with_forcefield(ffx)
    ref = pa.FrameworkBatch(fws, ffx, guest, ewald, T=np.float32)
    for k in ("sigma", "epsilon", "constant_offset", "bs", "kmin", "positions", "charges", "types", "Shost",
              "kprefactor", "cells", "atom_offsets", "k_offsets", "perm"):
        assert np.array_equal(getattr(new, k), getattr(ref, k)), k
    assert not np.array_equal(new.bs, b.bs)


def test_with_forcefield_rejects_other_types(pa, small):
    fws, ff, guest, ewald, prm = small
    b = pa.FrameworkBatch(fws, ff, guest, ewald)
    other = pa.ForceField(ff.names[:-1] + ["X"], np.diag(ff.sigma), np.diag(ff.epsilon), cutoff=ff.cutoff)
    with pytest.raises(pa.ArgumentError, match="same type names"):
        b.with_forcefield(other)


def test_scaled_forcefield(pa, small):
    fws, ff, guest, ewald, prm = small
    x = np.arange(1, 9) / 8.0 + 0.5
    ffx = pa.fit.scaled_forcefield(ff, prm["fitted_types"], x)
    sig0, eps0 = pa.forcefield.type_parameters(ff)
    sig, eps = pa.forcefield.type_parameters(ffx)
    for i, t in enumerate(prm["fitted_types"]):
        j = ff.typeindex(t) - 1
        assert eps[j] == pytest.approx(eps0[j] * x[i], rel=1e-15)
        assert sig[j] == pytest.approx(sig0[j] * x[4 + i], rel=1e-15)
    j = ff.typeindex("O_co2") - 1
    assert sig[j] == sig0[j] and eps[j] == eps0[j]


def test_hardcore_bound_matches_per_atom_bisection(pa, small):
    """The grouped, memoised bisections give exactly the per-atom loop of src/reject.jl:95-124."""
    fws, ff, guest, ewald, prm = small
    b = pa.FrameworkBatch(fws[:1], ff, guest, ewald)
    a0, a1 = b.atom_offsets[0], b.atom_offsets[1]
    k0, k1 = b.k_offsets[0], b.k_offsets[1]
    alpha = float(b.alphas[0])
    acc = 0.0
    for a in range(len(b.guest_types)):
        gt = int(b.guest_types[a]) - 1
        for j in range(a0, a1):
            ht = int(b.types[j]) - 1
            s, e = float(b.sigma[gt, ht]), float(b.epsilon[gt, ht])
            K = pa.KE * float(guest.charges[a]) * float(b.charges[j])
            if K < 0:
                r0 = float(pa.reject.find_r0(np.array([s]), np.array([e]), np.array([K]), alpha, b.cutoff)[0])
                acc += e + abs(K) * float(erfc(alpha * r0)) / r0
            else:
                acc += e
    Rs = 0.0
    for i in range(k0, k1):
        Rs += float(b.kprefactor[i]) * abs(complex(b.Shost[i]))
    ref = acc + 2 * pa.KE * float(np.sum(np.abs(guest.charges))) * Rs
    assert b.bs[0] == ref
    assert math.isfinite(ref)
