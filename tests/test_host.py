"""Host-side logic of the product (CPU only): the FrameworkBatch builder against the oracle's
independent builder, the rejection tables, dedup, cell lists, and the reference's validation
messages of widom (raised before any device work)."""
import math

import numpy as np
import pytest

from conftest import kT_of, oracle_view

INT_FIELDS = ["types", "atom_offsets", "kcoeffs", "k_offsets", "ncells", "cell_offsets", "cellgrid_offsets",
              "compact_to_orig", "guest_types", "framework_of", "perm"]
FLOAT_FIELDS = ["positions", "charges", "cells", "invcells", "volumes", "alphas", "ks", "kprefactor", "Shost",
                "constant_offset", "self_term_halfrange", "sigma", "epsilon", "bs", "kmin"]


def oracle_batch(pa, orc, fws, ff, guest, ewald, cellwidth=2.0, fullk=False):
    frames = [(fw.cell, fw.frac, [ff.typeindex(s + "_") for s in fw.symbols], fw.charges, fw.replication) for fw in fws]
    qs = pa.batch.self_term_quaternions() if np.any(guest.charges != 0) else None
    return orc.OracleBatch(frames, (np.sqrt(np.diag(ff.sigma) ** 2), np.diag(ff.epsilon), ff.cutoff, ff.tail),
                           (guest.sites, guest.types, guest.charges), ewald.cutoff, ewald.precision, cellwidth, fullk, qs)


def compare(b, o):
    for f in INT_FIELDS:
        assert np.array_equal(np.asarray(getattr(b, f)).reshape(-1), np.asarray(getattr(o, f)).reshape(-1)), f
    for f in FLOAT_FIELDS:
        a, c = np.asarray(getattr(b, f)).reshape(-1), np.asarray(getattr(o, f)).reshape(-1)
        assert a.shape == c.shape, f
        if a.size:
            np.testing.assert_allclose(a, c, rtol=1e-11, atol=1e-11, err_msg=f)


def test_builder_matches_oracle_co2(pa, orc):
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    compare(pa.FrameworkBatch(fws, ff, guest, ewald), oracle_batch(pa, orc, fws, ff, guest, ewald))


def test_builder_matches_oracle_batched_and_fullk(pa, orc):
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=3, max_unit_atoms=150)
    fws = [fws[0], fws[1], fws[0], fws[2]]  # a repeated framework is stored once
    b = pa.FrameworkBatch(fws, ff, guest, ewald, cellwidth=3.0)
    assert b.nsys == 4 and b.nframeworks() == 3 and list(b.framework_of) == [1, 2, 1, 3]
    compare(b, oracle_batch(pa, orc, fws, ff, guest, ewald, 3.0))
    bf = pa.FrameworkBatch(fws[:1], ff, guest, ewald, fullk=True)
    compare(bf, oracle_batch(pa, orc, fws[:1], ff, guest, ewald, 2.0, True))


def test_builder_matches_oracle_neutral_guest(pa, orc):
    fws, ff, guest, ewald, _ = pa.synthetic.lj_ch4()
    b = pa.FrameworkBatch(fws, ff, guest, ewald)
    assert len(b.ks) == 0 and list(b.k_offsets) == [0, 0] and np.all(b.self_term_halfrange == 0)
    compare(b, oracle_batch(pa, orc, fws, ff, guest, ewald))


def test_cell_sort_is_a_permutation_and_cells_are_right(pa):
    # test/batch_tests.jl:187-224
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    b = pa.FrameworkBatch(fws, ff, guest, ewald, cellwidth=3.0)
    fw = fws[0]
    key = lambda p, t, q: tuple(np.round(p, 10)) + (int(t), q)
    orig = sorted(key(p, ff.typeindex(s + "_"), q) for p, s, q in zip(pa.cartesian(fw), fw.symbols, fw.charges))
    got = sorted(key(p, b.compact_to_orig[t - 1], q) for p, t, q in zip(b.positions, b.types, b.charges))
    assert orig == got
    n = b.ncells[0]
    inv = b.invcells[0]
    for c in range(int(np.prod(n))):
        for j in range(b.cell_offsets[c], b.cell_offsets[c + 1]):
            f = inv @ b.positions[j]
            assert pa.cell.cell_linear(pa.cell.cell_coord(f, n), n) == c


def test_rejection_tables_match_oracle(pa, orc):
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    for T in (np.float64, np.float32):
        b = pa.FrameworkBatch(fws * 3, ff, guest, ewald, T=T)
        v, keep = oracle_view(orc, b)
        kT = kT_of(pa, b)
        rho2, reach0 = pa.build_rejection_tables(b, kT)
        orho2, oreach0 = orc.rejection_tables(v, b.bs, b.kmin, kT, float(np.finfo(T).eps))
        np.testing.assert_allclose(rho2, orho2, rtol=1e-13)
        assert np.array_equal(reach0, oreach0)
    # a non-positive margin names the system (test/reject_tests.jl:179-190)
    with pytest.raises(pa.ArgumentError, match="system 1"):
        pa.build_rejection_tables(b, -1.0e30)


def test_lj_cutoff_clamps_rejection_radius(pa):
    # test/reject_tests.jl:219-245
    A = pa.cell_matrix(30.0, 30.0, 30.0, 90, 90, 90)
    fw = pa.Framework(A, [[0.5, 0.5, 0.5]], ["B"], ["B"], [1.0])
    g = pa.Guest(np.zeros((1, 3)), [1], [-1.0])
    ff = pa.ForceField(["G_", "B_"], [3.0, 3.0], [0.01, 0.01], cutoff=1.0, tail=False)
    b = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=12.0))
    rho2, _ = pa.build_rejection_tables(b, pa.KB * 298.15)
    assert np.all(rho2 <= ff.cutoff**2)


def test_widom_validation_messages(pa):
    # test/widom_tests.jl:168-207, 471-478 (raised on the host before any device work)
    A = pa.cell_matrix(30.0, 30.0, 30.0, 90, 90, 90)
    fw = pa.Framework(A, np.zeros((0, 3)), [], [], np.zeros(0))
    ff = pa.ForceField(["X_"], [3.0], [0.001], cutoff=12.0)
    g = pa.Guest(np.zeros((1, 3)), [1], np.zeros(1))
    b = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=12.0))
    with pytest.raises(pa.ArgumentError, match="ninsert"):
        pa.widom(b, g, T=300.0, ninsert=5, nblocks=10)
    with pytest.raises(pa.ArgumentError, match="nblocks"):
        pa.widom(b, g, T=300.0, ninsert=100, nblocks=1)
    with pytest.raises(pa.ArgumentError, match="chunk"):
        pa.widom(b, g, T=300.0, ninsert=100, chunk=0)
    with pytest.raises(pa.ArgumentError, match="run=0 must be ≥ 1"):
        pa.widom(b, g, T=300.0, ninsert=100, run=0)
    with pytest.raises(pa.ArgumentError, match="run=1000 must be ≤ per=100"):
        pa.widom(b, g, T=300.0, ninsert=100, run=1000)
    other = pa.Guest(g.sites, g.types, g.charges * 2 + 1)
    with pytest.raises(pa.ArgumentError, match="does not match the guest"):
        pa.widom(b, other, T=300.0, ninsert=100)
    bad = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=12.0))
    bad.types = np.concatenate([bad.types, [1]]).astype(np.int32)
    with pytest.raises(pa.DimensionMismatch):
        pa.widom(bad, g, T=300.0, ninsert=100)


def test_batch_guards(pa):
    # test/batch_tests.jl:149-185: a replication lie, and a strongly polar guest in a small cell
    A = pa.cell_matrix(30.0, 30.0, 30.0, 90, 90, 90)
    ff = pa.ForceField(["X_"], [3.0], [0.001], cutoff=12.0, tail=False)
    gq = pa.Guest(np.zeros((1, 3)), [1], [1.0])
    fw = pa.Framework(A, [[0.1, 0.1, 0.1], [0.6, 0.35, 0.7]], ["X", "X"], ["X", "X"], [1.0, -1.0], (2, 1, 1))
    with pytest.raises(pa.ArgumentError, match="replication"):
        pa.FrameworkBatch([fw], ff, gq, pa.EwaldParams(cutoff=12.0))
    cutoff, rg = 3.0, 0.3
    L = 2 * (cutoff + rg)
    fw2 = pa.Framework(pa.cell_matrix(L, L, L, 90, 90, 90), [[0.5, 0.5, 0.5]], ["Zr"], ["Zr"], [1.0])
    ff2 = pa.ForceField(["Zr_"], [2.78], [0.003], cutoff=cutoff, tail=False)
    g2 = pa.Guest([[0.0, 0, 0], [rg, 0, 0]], [1, 1], [20.0, -20.0])
    with pytest.raises(pa.ArgumentError, match="self-term half-range"):
        pa.FrameworkBatch([fw2], ff2, g2, pa.EwaldParams(cutoff=cutoff))


def test_default_run_and_counts(pa):
    assert pa.default_run(1_000_000, 1) == 256
    assert pa.default_run(100, 7) == 3
    assert pa.default_run(3, 7) == 1


def test_bounds_hook_sets_the_batch_bounds(pa):
    # the `bounds` hook receives the finished batch and its result becomes B_s
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    host = pa.FrameworkBatch(fws, ff, guest, ewald)
    seen = []

    def hook(b):
        seen.append(b)
        return np.full(b.nframeworks(), 1.25)

    b = pa.FrameworkBatch(fws, ff, guest, ewald, bounds=hook)
    assert len(seen) == 1 and seen[0] is b
    assert np.array_equal(b.bs, [1.25]) and np.array_equal(b.positions, host.positions)
