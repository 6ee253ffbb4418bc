"""Insertion into a loaded configuration (Widom along an NVT chain, src/nvt.jl:85-124) on the host:
SystemState's running structure factor, insertion_constant_term, the per-system batch expansion,
argument checks, and the oracle's chain energy pinned against an independent total-energy
difference, as test/nvt_tests.jl:1-200 does: a literal Ewald sum over the host and every guest
(with and without the test molecule), direct-pair Lennard-Jones over every host-guest and
guest-guest pair, and the N-guest tail correction. The batch folds an orientation-averaged
reciprocal self term into the constant, so single poses differ by up to the self-term
half-range; the Boltzmann-weight averages over many poses agree within a few standard errors."""
import math

import numpy as np
import pytest


def _lj_ff(pa, extra):
    names = [n for n, _, _ in extra] + ["C_co2", "O_co2"]
    sig = [s for _, s, _ in extra] + [2.80, 3.05]
    eps = [e for _, _, e in extra] + [27.0 * pa.KB, 79.0 * pa.KB]
    return pa.ForceField(names, sig, eps, cutoff=12.0, tail=True)


def empty_box(pa):
    """A 30 Å cubic P1 cell with one non-interacting dummy site (sigma 1, epsilon 0, charge 0):
    CO2 guests with periodic images and nothing else (the reference's empty-box set-up)."""
    ff = _lj_ff(pa, [("X1_", 1.0, 0.0)])
    A = pa.cell_matrix(30.0, 30.0, 30.0, 90.0, 90.0, 90.0)
    fw = pa.Framework(A, np.zeros((1, 3)), ["X1"], ["X1"], np.zeros(1))
    return ff, pa.synthetic.co2_guest(ff), fw


def small_charged(pa, seed=4, T=np.float64):
    """A 28-30 Å triclinic cell with 60 charged atoms of two LJ types (net charge zero)."""
    rng = np.random.default_rng(seed)
    ff = _lj_ff(pa, [("Zn_", 2.46, 62.4 * pa.KB), ("Ow_", 3.12, 48.2 * pa.KB)])
    A = pa.cell_matrix(28.0, 29.0, 30.0, 88.0, 93.0, 91.0)
    frac = pa.synthetic._uniform_min_dist(rng, A, 60, 2.0)
    q = rng.normal(0.0, 0.5, 60)
    q -= q.mean()
    sym = ["Zn" if i % 2 else "Ow" for i in range(60)]
    return ff, pa.synthetic.co2_guest(ff), pa.Framework(A, frac, sym, sym, q, (1, 1, 1), T)


def random_poses(rng, A, n):
    pos = (A @ rng.uniform(0, 1, (n, 3)).T).T
    q = rng.normal(size=(n, 4))
    return pos, q / np.linalg.norm(q, axis=1)[:, None]


def explicit_state(pa, b, guest, rng, counts):
    """A configuration with counts[s] guests per system at uniform poses."""
    go = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    rp, qt = [], []
    for s, c in enumerate(counts):
        A = b.cells[b.framework_of[s] - 1]
        p, q = random_poses(rng, A, c)
        rp.append(p)
        qt.append(q)
    return pa.SystemState(b, guest, np.concatenate(rp), np.concatenate(qt), go, counts)


def total_energy(pa, orc, b, ff, guest, s, sites, precision):
    """Host + guests configuration energy minus the host-only energy: literal Ewald sums, direct
    LJ over every host-guest and guest-guest pair (minimum image), and the tail correction."""
    fw = b.framework_of[s] - 1
    A, iA = b.cells[fw], b.invcells[fw]
    a0, a1 = b.atom_offsets[fw], b.atom_offsets[fw + 1]
    hpos, hq = b.positions[a0:a1], b.charges[a0:a1]
    c2o = np.asarray(b.compact_to_orig) - 1
    htype = c2o[np.asarray(b.types[a0:a1]) - 1]
    ng, N = sites.shape[0], len(guest.sites)
    alpha = float(b.alphas[fw])
    ks, w, _ = orc.kvectors(A, pa.ewald_kmax(alpha, precision))
    gpos = sites.reshape(-1, 3)
    gq = np.tile(guest.charges, ng)
    gt = np.tile(np.asarray(guest.types) - 1, ng)
    mol = np.concatenate([np.arange(len(hpos)), len(hpos) + np.repeat(np.arange(ng), N)])
    Ec = (orc.ewald_energy(A, np.concatenate([hpos, gpos]), np.concatenate([hq, gq]), mol, alpha, b.ewald_cutoff, ks, w)
          - orc.ewald_energy(A, hpos, hq, np.arange(len(hpos)), alpha, b.ewald_cutoff, ks, w))
    rc2 = ff.cutoff**2

    def lj(d, ti, tj):
        d = d - (np.rint(d @ iA.T) @ A.T)
        r2 = np.einsum("ij,ij->i", d, d)
        m = r2 < rc2
        x = (ff.sigma[ti, tj][m] ** 2 / r2[m]) ** 3
        return float(np.sum(4 * ff.epsilon[ti, tj][m] * (x * x - x)))

    Elj = 0.0
    for i in range(len(gpos)):
        Elj += lj(gpos[i] - hpos, np.full(len(hpos), gt[i]), htype)
        later = np.arange(i + 1, len(gpos))
        later = later[later // N != i // N]
        if len(later):
            Elj += lj(gpos[i] - gpos[later], np.full(len(later), gt[i]), gt[later])
    nff = len(ff.names)
    gcounts = np.bincount(np.asarray(guest.types) - 1, minlength=nff)
    hcounts = np.bincount(htype, minlength=nff)
    return Elj + Ec + pa.tail_delta(ff, hcounts, ng * gcounts, float(b.volumes[fw]))


def chain_view(pa, orc, b, st, s):
    """The oracle's view of system s of the system-expanded batch with the running S(k)."""
    sb = pa.chain.system_batch(b)
    vb = type("View", (), {})()
    for k in ("positions", "types", "charges", "atom_offsets", "cells", "invcells", "volumes", "alphas", "ks",
              "kprefactor", "k_offsets", "constant_offset", "ncells", "cell_offsets", "cellgrid_offsets", "sigma",
              "epsilon", "guest_types", "framework_of"):
        setattr(vb, k, getattr(sb, k))
    vb.Shost = st.Sk
    return orc.view(vb, b.guest_sites_orig, b.guest_charges_orig, b.cutoff, b.ewald_cutoff)


@pytest.mark.parametrize("setup,ng,nposes", [("empty", 10, 1500), ("charged", 6, 400)])
def test_oracle_chain_energy_matches_total_energy_difference(pa, orc, setup, ng, nposes):
    ff, guest, fw = empty_box(pa) if setup == "empty" else small_charged(pa)
    precision = 1e-6
    b = pa.FrameworkBatch([fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=precision), fullk=True)
    rng = np.random.default_rng(41)
    st = explicit_state(pa, b, guest, rng, [ng])
    kT = pa.KB * 298.15
    sites = st.live_sites(guest, 0)
    (v, keep) = chain_view(pa, orc, b, st, 0)
    const = pa.insertion_constant_term(ff, b, guest, 0, ng)
    pos, quat = random_poses(rng, b.cells[0], nposes)
    dU = orc.chain_energy(v, 0, pos, quat, sites) + const
    E0 = total_energy(pa, orc, b, ff, guest, 0, sites, precision)
    dU_ref = np.empty(nposes)
    for m in range(nposes):
        test = np.array([pos[m] + pa.batch._rotate(quat[m], x) for x in guest.sites])[None]
        dU_ref[m] = total_energy(pa, orc, b, ff, guest, 0, np.concatenate([sites, test]), precision) - E0
    # single poses: within the self-term spread (plus FP64 rounding of overlapping poses' large ΔU)
    fin = np.isfinite(dU_ref)
    assert np.all(np.abs(dU - dU_ref)[fin] <= 2.6 * b.self_term_halfrange[0] + 1e-9 + 1e-12 * np.abs(dU_ref[fin]))
    w, wr = np.exp(-dU / kT), np.exp(-dU_ref / kT)
    se = math.sqrt(np.var(w, ddof=1) / nposes + np.var(wr, ddof=1) / nposes)
    assert abs(w.mean() - wr.mean()) <= 5 * se


def test_constant_term_at_zero_guests_is_the_constant_offset(pa):
    ff, guest, fw = small_charged(pa)
    b = pa.FrameworkBatch([fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    for s in range(2):
        assert pa.insertion_constant_term(ff, b, guest, s, 0) == b.constant_offset[0]
    # one more guest changes only the tail and net-charge terms (the charged guest is neutral
    # overall, so only the tail moves)
    nff = len(ff.names)
    gc = np.bincount(np.asarray(guest.types) - 1, minlength=nff)
    c2o = np.asarray(b.compact_to_orig) - 1
    hc = np.bincount(c2o[np.asarray(b.types) - 1], minlength=nff)
    V = float(b.volumes[0])
    for n in (1, 4):
        d = pa.insertion_constant_term(ff, b, guest, 0, n) - pa.insertion_constant_term(ff, b, guest, 0, n - 1)
        t = lambda m: pa.tail_delta(ff, hc, m * gc, V)
        d_ref = (t(n + 1) - t(n)) - (t(n) - t(n - 1)) if n > 1 else t(2) - 2 * t(1)
        assert d == pytest.approx(d_ref, rel=1e-9, abs=1e-15)


def test_system_state_structure_factor(pa, orc):
    ff, guest, fw = small_charged(pa)
    b = pa.FrameworkBatch([fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    st = explicit_state(pa, b, guest, np.random.default_rng(2), [0, 7])
    assert np.array_equal(st.k_offsets, [0, len(b.ks), 2 * len(b.ks)])
    assert np.array_equal(st.Sk[:len(b.ks)], b.Shost)
    sites = st.live_sites(guest, 1).reshape(-1, 3)
    S = orc.structure_factor(b.ks, np.concatenate([b.positions, sites]),
                             np.concatenate([b.charges, np.tile(guest.charges, 7)]))
    assert np.max(np.abs(st.Sk[len(b.ks):] - S)) <= 1e-9 * np.max(np.abs(S))


def test_system_batch_expands_shared_frameworks(pa):
    ff, guest, fw = small_charged(pa)
    b = pa.FrameworkBatch([fw, fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    assert b.nframeworks() == 1 and b.nsys == 3
    sb = pa.chain.system_batch(b)
    assert sb is pa.chain.system_batch(b)
    assert sb.nframeworks() == 3 and list(sb.framework_of) == [1, 2, 3]
    sb.check_axes()
    n = len(b.positions)
    for s in range(3):
        assert np.array_equal(sb.positions[s * n:(s + 1) * n], b.positions)
        assert np.array_equal(sb.ks[s * len(b.ks):(s + 1) * len(b.ks)], b.ks)
    assert np.array_equal(sb.constant_offset, np.repeat(b.constant_offset, 3))
    single = pa.FrameworkBatch([fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    assert pa.chain.system_batch(single) is single


def test_argument_checks(pa):
    ff, guest, fw = small_charged(pa)
    sparse = pa.FrameworkBatch([fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6))
    with pytest.raises(pa.ArgumentError, match="fullk=true"):
        pa.SystemState(sparse, guest, np.zeros((0, 3)), np.zeros((0, 4)), [0, 0], [0])
    b = pa.FrameworkBatch([fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    other = pa.Guest(guest.sites, guest.types, -guest.charges)
    with pytest.raises(pa.ArgumentError, match="does not match the guest"):
        pa.SystemState(b, other, np.zeros((0, 3)), np.zeros((0, 4)), [0, 0], [0])
    with pytest.raises(pa.ArgumentError, match="capacity"):
        pa.SystemState(b, guest, np.zeros((1, 3)), np.tile([0, 0, 0, 1.0], (1, 1)), [0, 1], [2])
    with pytest.raises(pa.DimensionMismatch, match="ncounts"):
        pa.SystemState.placed(b, guest, [1, 2], T=298.15)
    st = pa.SystemState(b, guest, np.zeros((0, 3)), np.zeros((0, 4)), [0, 0], [0])
    with pytest.raises(pa.ArgumentError, match="n_widom_per_cycle"):
        pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=0)
    with pytest.raises(pa.ArgumentError, match="Float32"):
        pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=8)
    with pytest.raises(pa.ArgumentError, match="two"):
        pa.widom_along_chain(b, [st], guest, ff, T=298.15, n_widom_per_cycle=8)


def test_placed_guests_clear_the_hard_core(pa):
    ff, guest, fw = small_charged(pa)
    b = pa.FrameworkBatch([fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    st = pa.SystemState.placed(b, guest, [3, 5], T=298.15, seed=9, capacities=[4, 5])
    assert list(st.guest_offsets) == [0, 4, 9] and list(st.occupancy) == [3, 5]
    assert np.array_equal(st.orientations[3], [0, 0, 0, 1]) and np.array_equal(st.refpoints[3], [0, 0, 0])
    kT = float(b.T(pa.KB * 298.15))
    rho2, _ = pa.build_rejection_tables(b, kT)
    N, nt = len(b.guest_types), len(b.sigma)
    for s in range(2):
        sites = st.live_sites(guest, s)
        for j in range(sites.shape[0]):
            for a in range(N):
                d = sites[j, a] - b.positions
                d = d - (np.rint(d @ b.invcells[0].T) @ b.cells[0].T)
                r2 = np.einsum("ij,ij->i", d, d)
                assert np.all(r2 >= rho2.reshape(2, N, nt)[s, a, np.asarray(b.types) - 1])
