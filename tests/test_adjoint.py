"""Adjoint of ln K_H on the CPU: the host chain rule (tail correction, Lorentz-Berthelot mixing,
net-charge term, replica folding) and the oracle's adjoint sums against central finite
differences of the oracle's own ln K_H with common random numbers (the same counter-based poses
at every parameter value). PureAdsorb.jl has no gradients to pin against; the finite-difference
check on the FP64 oracle is the pin."""
import math

import numpy as np
import pytest

from conftest import kT_of, oracle_view

NINS = 20_000
SEED = 42
NBLOCKS = 10
RUN = 2000
H = 1.0e-4  # relative step


class CO2Case:
    """The charged CO2 workload (5,832 atoms) with cached structure factors, so a perturbed force
    field rebuilds its batch without recomputing S(k)."""

    def __init__(self, pa, orc):
        self.pa, self.orc = pa, orc
        self.fws, self.ff, self.guest, self.ewald, _ = pa.synthetic.co2(T=np.float64)
        self.cache = {}

    def sk(self, ks, pos, q):
        key = (ks.tobytes(), pos.tobytes(), np.asarray(q).tobytes())
        if key not in self.cache:
            self.cache[key] = self.pa.structure_factor(ks, pos, q)
        return self.cache[key]

    def batch(self, ff=None, fws=None, T=np.float64):
        return self.pa.FrameworkBatch(fws or self.fws, ff or self.ff, self.guest, self.ewald, T=T, sk=self.sk)

    def run(self, b):
        kT = kT_of(self.pa, b)
        v, keep = oracle_view(self.orc, b)
        rho2, reach0 = self.pa.build_rejection_tables(b, kT)
        out = self.orc.widom(v, 32, kT, NINS, SEED, NBLOCKS, RUN, True, rho2, reach0)
        return b, kT, v, keep, out

    def lnW(self, b):
        _, _, _, _, out = self.run(b)
        return math.log(float(np.sum(out["sW"])))

    def ff_scaled(self, t, which, f):
        sig, eps = self.pa.forcefield.type_parameters(self.ff)
        (sig if which == "sigma" else eps)[t] *= f
        return self.pa.ForceField(self.ff.names, sig, eps, cutoff=self.ff.cutoff, tail=self.ff.tail)

    def fws_charge(self, u, dq):
        fw = self.fws[0]
        nu = len(fw.charges) // int(np.prod(fw.replication))
        q = fw.charges.copy()
        q[u::nu] += dq
        return [self.pa.Framework(fw.cell, fw.frac, fw.labels, fw.symbols, q, fw.replication, fw.T)]


@pytest.fixture(scope="module")
def case(pa, orc):
    return CO2Case(pa, orc)


@pytest.fixture(scope="module")
def adjoint(pa, orc, case):
    b, kT, v, keep, out = case.run(case.batch())
    nat, nk = pa.adjoint.system_offsets(b)
    sums = orc.grad_sums(v, kT, NINS, RUN, out, nat, nk)
    return pa.adjoint.assemble(b, case.ff, 0, sums[0], kT), sums[0], b


def test_tail_pair_grad_matches_fd(pa):
    ff = pa.synthetic.co2()[1]
    n = len(ff.names)
    counts = np.array([216 * 27 // 5] * 5 + [0, 0])
    gc = np.array([0] * 5 + [1, 2])
    V = 74_000.0
    dS, dE = pa.forcefield.tail_delta_pair_grad(ff, counts, gc, V)
    g_sig, g_eps = pa.forcefield.pair_to_type_grad(ff, dS, dE)
    sig, eps = pa.forcefield.type_parameters(ff)
    for t in range(n):
        for which, g in (("sigma", g_sig), ("epsilon", g_eps)):
            vals = []
            for f in (1 + 1e-6, 1 - 1e-6):
                s2, e2 = sig.copy(), eps.copy()
                (s2 if which == "sigma" else e2)[t] *= f
                vals.append(pa.tail_delta(pa.ForceField(ff.names, s2, e2, cutoff=ff.cutoff), counts, gc, V))
            p = (sig if which == "sigma" else eps)[t]
            fd = (vals[0] - vals[1]) / (2e-6 * p)
            assert g[t] == pytest.approx(fd, rel=1e-6, abs=1e-12 * max(1.0, abs(fd))), (which, t)


def test_fold_replicas(pa):
    g = np.arange(12.0)
    assert np.array_equal(pa.adjoint.fold_replicas(g, 4), np.array([0 + 4 + 8, 1 + 5 + 9, 2 + 6 + 10, 3 + 7 + 11.0]))


@pytest.mark.parametrize("name,which", [("A_", "epsilon"), ("A_", "sigma"), ("C_", "epsilon"), ("C_", "sigma"),
                                        ("C_co2", "epsilon"), ("C_co2", "sigma"), ("O_co2", "epsilon"),
                                        ("O_co2", "sigma")])
def test_lj_gradient_matches_fd(case, adjoint, name, which):
    g, _, _ = adjoint
    t = case.ff.typeindex(name) - 1
    p = case.pa.forcefield.type_parameters(case.ff)[0 if which == "sigma" else 1][t]
    lp = case.lnW(case.batch(ff=case.ff_scaled(t, which, 1 + H)))
    lm = case.lnW(case.batch(ff=case.ff_scaled(t, which, 1 - H)))
    fd = (lp - lm) / (2 * H * p)
    ad = getattr(g, which)[t]
    assert ad == pytest.approx(fd, rel=1e-3), (name, which, ad, fd)


@pytest.mark.parametrize("u", [0, 7])
def test_charge_gradient_matches_fd(case, adjoint, u):
    g, _, b = adjoint
    nu = 216
    gu = case.pa.adjoint.fold_replicas(g.charges, nu)
    q = case.fws[0].charges[u]
    h = H * abs(q)
    lp = case.lnW(case.batch(fws=case.fws_charge(u, h)))
    lm = case.lnW(case.batch(fws=case.fws_charge(u, -h)))
    fd = (lp - lm) / (2 * h)
    scale = np.max(np.abs(gu))
    assert abs(gu[u] - fd) <= 1e-3 * max(abs(fd), 0.05 * scale), (u, gu[u], fd, scale)


def test_untouched_types_have_zero_gradient(case, adjoint):
    g, sums, _ = adjoint
    # every type of the force field appears in the batch, so all gradients are finite
    assert np.all(np.isfinite(g.epsilon)) and np.all(np.isfinite(g.sigma)) and np.all(np.isfinite(g.charges))
    assert g.sum_w > 0 and sums["sum_w"] == g.sum_w


def test_assemble_all_equals_per_system_chain_rule(pa):
    """The vectorised host assembly of the gradients (every system at once) against the per-system
    composition of the device-sum mapping, tail_delta_pair_grad and pair_to_type_grad, on a batch of
    several frameworks with synthetic adjoint sums."""
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=4, T=np.float64, max_unit_atoms=120)
    b = pa.FrameworkBatch(fws, ff, guest, ewald)
    rng = np.random.default_rng(3)
    N, nt = len(b.guest_types), len(b.sigma)
    nat, _ = pa.adjoint.system_offsets(b)
    sums = [dict(xmax=rng.normal(), sum_w=rng.uniform(1, 2), d_epsilon=rng.normal(size=N * nt),
                 d_sigma=rng.normal(size=N * nt), d_charge=rng.normal(size=int(nat[s])), recomputed=s)
            for s in range(b.nsys)]
    kT = 0.0257
    got = pa.adjoint.assemble_all(b, ff, sums, kT)
    nff = len(ff.names)
    c2o = np.asarray(b.compact_to_orig) - 1
    gt = np.asarray(b.guest_types) - 1
    for s in range(b.nsys):
        p = sums[s]
        dS, dE = np.zeros((nff, nff)), np.zeros((nff, nff))
        for a in range(N):
            dE[c2o[gt[a]], c2o] += p["d_epsilon"].reshape(N, nt)[a] / p["sum_w"]
            dS[c2o[gt[a]], c2o] += p["d_sigma"].reshape(N, nt)[a] / p["sum_w"]
        fw = b.framework_of[s] - 1
        a0, a1 = b.atom_offsets[fw], b.atom_offsets[fw + 1]
        counts = np.bincount(c2o[np.asarray(b.types[a0:a1]) - 1], minlength=nff)
        gc = np.bincount(np.asarray(b.guest_types_orig) - 1, minlength=nff)
        tS, tE = pa.forcefield.tail_delta_pair_grad(ff, counts, gc, b.volumes[fw])
        g_sig, g_eps = pa.forcefield.pair_to_type_grad(ff, dS + tS, dE + tE)
        ok = np.isfinite(g_eps)
        assert np.allclose(got[s].epsilon[ok], -g_eps[ok] / kT, rtol=1e-12, atol=0)
        assert np.array_equal(np.isfinite(got[s].epsilon), ok)
        assert np.allclose(got[s].sigma, -g_sig / kT, rtol=1e-12, atol=1e-300)
        assert got[s].charges.shape == (a1 - a0,) and got[s].recomputed == s
