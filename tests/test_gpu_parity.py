"""Parity of the CUDA path (through the C ABI) with the oracle, on a B200.

Tolerances (stated here, used below):
- poses and phase-0 flags: bit-exact (both follow the same strict operation sequence);
- FP64 plain path: per-insertion dU rtol 1e-12 (the reference's insertion_energy vs brute-force
  bound, test/energy_tests.jl:115) plus 1e-12 eV absolute for energies near zero; mu_ex, K_H and
  q_st rtol 1e-10 (test/gpu_tests.jl:20-22);
- FP32 path (default split: pairs within 6 Å and at the cutoffs' rounding bands in FP64, the
  reciprocal term in FP64, every other pair FP32): per-insertion
  |dU32 - dU64| <= max(1e-5 |dU64|, 8.62e-8 eV), i.e. 1e-5 relative or 1e-3 K absolute, for every
  survivor; aggregate |Δ ln K_H| <= 1e-3 and |Δ q_st| <= 5.18e-4 eV (0.05 kJ/mol) against the
  all-FP64 oracle on the same stream;
- FP32 path with every pair and the reciprocal term in FP32 (near radius 0): per insertion
  |dU32 - dU64| <= 1e-5 |dU64| + 2e-6 eV (FP32 rounding of pair terms of up to ~1 eV), same
  aggregate bounds.
"""
import math

import numpy as np
import pytest

from conftest import kT_of, oracle_view

pytestmark = pytest.mark.gpu

F32_REL, F32_ABS = 1e-5, 8.62e-8    # max(rel |dU|, abs): the per-insertion criterion (1e-3 K = 8.62e-8 eV)
FAST_REL, FAST_ABS = 1e-5, 2e-6     # rel |dU| + abs: every pair and the reciprocal term in FP32


def within_f32(a, b):
    """Per-insertion FP32 criterion: |a - b| <= max(1e-5 |b|, 8.62e-8 eV)."""
    return np.abs(a - b) <= np.maximum(F32_REL * np.abs(b), F32_ABS)


F64_REL, F64_ABS = 1e-12, 1e-12  # the absolute floor covers energies that cross zero


def run_both(pa, orc, batch, guest, ninsert, seed, nblocks, reject=True, backend=None, T=298.15):
    ins = {}
    res = pa._widom(batch, guest, reject=reject, T=T, ninsert=ninsert, seed=seed, nblocks=nblocks,
                    insertions=ins, backend=backend)
    v, keep = oracle_view(orc, batch)
    kT = kT_of(pa, batch, T)
    rho2, reach0 = pa.build_rejection_tables(batch, kT) if reject else (None, None)
    prec = 32 if batch.T == np.float32 else 64
    run = pa.default_run(ninsert, batch.nsys)
    ref = orc.widom(v, prec, kT, ninsert, seed, nblocks, run, reject, rho2, reach0)
    return res, ins, ref, kT


def ref_results(pa, batch, ref, kT, nblocks):
    Vf = batch.volumes.astype(batch.T).astype(np.float64)
    return [pa._reduce(ref["sW"][s], ref["sUW"][s], ref["n"][s], kT, Vf[batch.framework_of[s] - 1], s + 1)
            for s in range(batch.nsys)]


@pytest.fixture(scope="module")
def co2_small(pa):
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    return fws, ff, guest, ewald


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_poses_flags_energies_co2(pa, orc, backend, co2_small, T):
    fws, ff, guest, ewald = co2_small
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=T)
    res, ins, ref, kT = run_both(pa, orc, batch, guest, 20_000, 5, 4, backend=backend)
    assert np.array_equal(ins["poses"], ref["poses"])
    assert np.array_equal(ins["flags"], ref["flags"])
    surv = ref["flags"] == 0
    assert np.all(np.isinf(ins["dU"][~surv]))
    a, b = ins["dU"][surv], ref["dU"][surv]
    if T == np.float64:
        np.testing.assert_allclose(a, b, rtol=F64_REL, atol=F64_ABS)
        for r, q in zip(res, ref_results(pa, batch, ref, kT, 4)):
            # test/gpu_tests.jl:20-22 compares mu_ex, K_H, q_st at rtol 1e-10. The delta-method
            # q_st_err cancels catastrophically when one insertion dominates the weight (here one
            # insertion carries 99.97 % of it), so it is compared on the scale of q_st itself.
            for f in ("mu_ex", "K_H", "q_st"):
                assert getattr(r, f) == pytest.approx(getattr(q, f), rel=1e-10)
            assert r.mu_ex_err == pytest.approx(q.mu_ex_err, rel=1e-8)
            assert r.K_H_err == pytest.approx(q.K_H_err, rel=1e-8)
            assert abs(r.q_st_err - q.q_st_err) <= 1e-10 * (abs(q.q_st) + q.q_st_err)
    else:
        # the default split on this workload evaluates its FP32 Coulomb pairs in the exp-free form
        exp_free, fit_err = backend.ctx.fp32_form()
        assert exp_free and 0 < fit_err <= 1.5e-7
        err = np.abs(a - b)
        assert np.all(within_f32(a, b)), f"{int(np.sum(~within_f32(a, b)))} outside, max err {err.max()}"
        for r, q in zip(res, ref_results(pa, batch, ref, kT, 4)):
            assert abs(math.log(r.K_H) - math.log(q.K_H)) <= 1e-3
            assert abs(r.q_st - q.q_st) <= 5.18e-4


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_two_phase_equals_single_phase(pa, backend, co2_small, T):
    fws, ff, guest, ewald = co2_small
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=T)
    r2 = pa.widom(batch, guest, T=298.15, ninsert=6000, seed=17, nblocks=4, chunk=4, backend=backend)
    r1 = pa.widom_singlephase(batch, guest, T=298.15, ninsert=6000, seed=17, nblocks=4, chunk=4, backend=backend)
    assert r1 == r2


def test_lj_ch4_parity(pa, orc, backend):
    fws, ff, guest, ewald, prm = pa.synthetic.lj_ch4()
    for T in (np.float64, np.float32):
        batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=T)
        res, ins, ref, kT = run_both(pa, orc, batch, guest, 30_000, 42, 10, backend=backend)
        assert np.array_equal(ins["flags"], ref["flags"])
        surv = ref["flags"] == 0
        a, b = ins["dU"][surv], ref["dU"][surv]
        if T == np.float64:
            np.testing.assert_allclose(a, b, rtol=F64_REL, atol=F64_ABS)
        else:
            assert np.all(within_f32(a, b))


def test_batched_frameworks_parity(pa, orc, backend):
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=4, max_unit_atoms=300)
    for T in (np.float64, np.float32):
        batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=T)
        res, ins, ref, kT = run_both(pa, orc, batch, guest, 16_000, 7, 4, backend=backend)
        assert np.array_equal(ins["poses"], ref["poses"])
        assert np.array_equal(ins["flags"], ref["flags"])
        surv = ref["flags"] == 0
        a, b = ins["dU"][surv], ref["dU"][surv]
        if T == np.float64:
            np.testing.assert_allclose(a, b, rtol=F64_REL, atol=F64_ABS)
        else:
            assert np.all(within_f32(a, b))


@pytest.mark.parametrize("case", ["co2", "lj_ch4"])
def test_fp32_all_pairs_mode(pa, orc, backend, case):
    # every pair and the reciprocal term in FP32 (near radius 0): the looser per-insertion bound,
    # the same aggregate bounds
    fws, ff, guest, ewald = getattr(pa.synthetic, case)(T=np.float32)[:4]
    batch = pa.FrameworkBatch(fws, ff, guest, ewald)
    ctx = backend.ctx
    old = ctx.fp32_split()
    ctx.set_fp32_split(near_radius=0.0, fp64_reciprocal=False)
    try:
        res, ins, ref, kT = run_both(pa, orc, batch, guest, 20_000, 11, 4, backend=backend)
        assert ctx.fp32_form() == (False, 0.0)  # no near radius: the rational form
    finally:
        ctx.set_fp32_split(near_radius=old.near_radius, fp64_reciprocal=old.fp64_reciprocal)
    assert np.array_equal(ins["flags"], ref["flags"])
    surv = ref["flags"] == 0
    a, b = ins["dU"][surv], ref["dU"][surv]
    assert np.all(np.abs(a - b) <= FAST_REL * np.abs(b) + FAST_ABS)
    for r, q in zip(res, ref_results(pa, batch, ref, kT, 4)):
        assert abs(math.log(r.K_H) - math.log(q.K_H)) <= 1e-3
        assert abs(r.q_st - q.q_st) <= 5.18e-4


@pytest.mark.parametrize("cutoff,precision", [(10.0, 1e-5), (14.0, 1e-7)])
def test_exp_free_form_other_ewald_settings(pa, orc, backend, co2_small, cutoff, precision):
    # an Ewald cutoff below and above the LJ one (the unequal-cutoff kernels) and other alphas: the
    # exp-free fit is accepted and every survivor meets the per-insertion criterion
    fws, ff, guest, _ = co2_small
    batch = pa.FrameworkBatch(fws, ff, guest, pa.EwaldParams(cutoff, precision), T=np.float32)
    res, ins, ref, kT = run_both(pa, orc, batch, guest, 20_000, 9, 4, backend=backend)
    exp_free, fit_err = backend.ctx.fp32_form()
    assert exp_free and 0 < fit_err <= 1.5e-7
    assert np.array_equal(ins["flags"], ref["flags"])
    surv = ref["flags"] == 0
    a, b = ins["dU"][surv], ref["dU"][surv]
    assert np.all(within_f32(a, b)), f"{int(np.sum(~within_f32(a, b)))} outside"


def test_rational_form_when_the_fit_is_refused(pa, orc, backend, co2_small):
    # a 4 Å near radius widens the exp-free fit's range until it misses 1.5e-7 at this alpha: the
    # FP32 Coulomb pairs take the rational form, within the all-FP32 bound (pairs at 4-6 Å in FP32)
    fws, ff, guest, ewald = co2_small
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    ctx = backend.ctx
    old = ctx.fp32_split()
    ctx.set_fp32_split(near_radius=4.0)
    try:
        res, ins, ref, kT = run_both(pa, orc, batch, guest, 20_000, 13, 4, backend=backend)
        assert ctx.fp32_form() == (False, 0.0)
    finally:
        ctx.set_fp32_split(near_radius=old.near_radius, fp64_reciprocal=old.fp64_reciprocal)
    surv = ref["flags"] == 0
    a, b = ins["dU"][surv], ref["dU"][surv]
    assert np.all(np.abs(a - b) <= FAST_REL * np.abs(b) + FAST_ABS)


def test_every_pair_in_fp64_when_the_near_radius_exceeds_the_cutoff(pa, orc, backend, co2_small):
    # a 13 Å near radius (cutoffs 12 Å) sends every in-cutoff pair through the FP64 pass: no FP32
    # Coulomb pairs are left (the form query reports the rational form, unused), and every survivor
    # lies far inside the per-insertion criterion (the FP32 rows of the reciprocal term remain)
    fws, ff, guest, ewald = co2_small
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    ctx = backend.ctx
    old = ctx.fp32_split()
    ctx.set_fp32_split(near_radius=13.0)
    try:
        res, ins, ref, kT = run_both(pa, orc, batch, guest, 20_000, 17, 4, backend=backend)
        assert ctx.fp32_form() == (False, 0.0)
    finally:
        ctx.set_fp32_split(near_radius=old.near_radius, fp64_reciprocal=old.fp64_reciprocal)
    assert np.array_equal(ins["flags"], ref["flags"])
    surv = ref["flags"] == 0
    a, b = ins["dU"][surv], ref["dU"][surv]
    ratio = np.abs(a - b) / np.maximum(F32_REL * np.abs(b), F32_ABS)
    assert ratio.max() <= 0.25, ratio.max()


def test_empty_box_ideal_gas(pa, backend):
    A = pa.cell_matrix(30.0, 30.0, 30.0, 90, 90, 90)
    fw = pa.Framework(A, np.zeros((0, 3)), [], [], np.zeros(0))
    ff = pa.ForceField(["X_"], [3.0], [0.001], cutoff=12.0, tail=False)
    g = pa.Guest(np.zeros((1, 3)), [1], np.zeros(1))
    for T in (np.float64, np.float32):
        b = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=12.0), T=T)
        r = pa.widom(b, g, T=300.0, ninsert=10_000, seed=1, backend=backend)[0]
        kT = float(T(pa.KB * 300.0))
        assert abs(r.mu_ex) < 1e-12
        assert r.K_H == pytest.approx(float(T(30.0**3)) / kT, rel=1e-6)
        assert r.q_st == pytest.approx(kT)
        assert r.nsamples == 10_000


def test_sharded_segments_combine_exactly(pa, backend, co2_small):
    fws, ff, guest, ewald = co2_small
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    ninsert, nblocks = 40_000, 4
    run = pa.default_run(ninsert, 1)
    full = pa.widom(batch, guest, T=298.15, ninsert=ninsert, seed=9, nblocks=nblocks, backend=backend)
    nseg = pa._lib.ctypes.c_int64()
    pa._lib.lib().pa_segment_count(ninsert, 1, run, nblocks, pa._lib.ctypes.byref(nseg))
    segs = np.zeros(3 * nseg.value)
    cut = nseg.value // 3
    for rng in ((0, cut), (cut, nseg.value)):
        pa._widom(batch, guest, reject=True, T=298.15, ninsert=ninsert, seed=9, nblocks=nblocks, backend=backend,
                  segment_range=rng, segments_out=segs)
    lse, sw, suw = np.zeros(nblocks), np.zeros(nblocks), np.zeros(nblocks)
    cnt = np.zeros(nblocks, dtype=np.int64)
    sums = pa._lib.BlockSums(*(pa._lib.ptr(a) for a in (lse, sw, suw, cnt)), None)
    assert pa._lib.lib().pa_combine_segments(ninsert, 1, run, nblocks, pa._lib.ptr(segs), sums) == 0
    kT = kT_of(pa, batch)
    sW, sUW = pa.block_sums(lse, sw, suw)
    combined = pa._reduce(sW, sUW, cnt, kT, float(np.float32(batch.volumes[0])), 1)
    assert combined == full[0]


def test_device_structure_factor(pa, backend, co2_small):
    fws, ff, guest, ewald = co2_small
    fw = fws[0]
    ks, w, c = pa.kvectors(fw.cell, 1.0)
    pos = pa.cartesian(fw)
    S_host = pa.structure_factor(ks, pos, fw.charges)
    S_dev = backend.ctx.structure_factor(ks, pos, fw.charges)
    np.testing.assert_allclose(S_dev, S_host, rtol=1e-10, atol=1e-10)
