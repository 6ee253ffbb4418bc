"""The oracle pinned against the reference's own known-answer tests (CPU only).

Each test names the reference test it restates (paths inside PureAdsorb.jl). Tests that need the
reference's data files (RUBTAK.cif, trappe.yaml, co2.yaml) read them from the reference checkout
when it is present and are skipped otherwise.
"""
import json
import math
import os

import numpy as np
import pytest
from scipy.special import erfc

from conftest import kT_of, oracle_view, reference_data, rubtak_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# --------------------------------------------------------------------------- RNG (test/rng_tests.jl)
def test_rng_golden_vectors(orc):
    kat = json.load(open(os.path.join(GOLDEN, "rng_kat.json")))
    L = orc.lib()
    for c in kat["pose_stream"]:
        seed, s, k = int(c["seed"]), c["s"], c["k"]
        for d in range(6):
            raw = L.or_chain_bits(L.or_splitmix64(seed, s), k, 0, d)
            assert raw == int(c["raw"][d])
            assert L.or_unit_f64(raw) == float.fromhex(c["u64"][d])
            bits = np.array([L.or_unit_f32(raw)], dtype=np.float32).view(np.uint32)[0]
            assert int(bits) == c["u32_bits"][d]
        # the FP32 quaternion, bit for bit (correctly rounded sinpi/cospi)
        _, q = orc.poses(32, seed, s, k, 1)
        assert q[0].astype(np.float32).view(np.uint32).tolist() == c["quat_f32_bits"]
    for m in kat["mulhi64"]:
        assert L.or_mulhi64(int(m["a"]), int(m["b"])) == int(m["hi"])


def test_mulhi64_matches_128_bit(orc):
    # test/rng_tests.jl:1-14
    rng = np.random.default_rng(1)
    L = orc.lib()
    for _ in range(20000):
        a, b = (int(x) for x in rng.integers(0, 2**64, size=2, dtype=np.uint64))
        assert L.or_mulhi64(a, b) == (a * b) >> 64


def test_chain_rng_key_sensitivity(orc):
    # test/rng_tests.jl:16-31
    L = orc.lib()
    b0 = L.or_chain_bits(7, 3, 2, 0)
    assert L.or_chain_bits(7, 3, 2, 0) == b0
    assert L.or_chain_bits(8, 3, 2, 0) != b0
    assert L.or_chain_bits(7, 4, 2, 0) != b0
    assert L.or_chain_bits(7, 3, 5, 0) != b0
    assert len({b0, L.or_chain_bits(7, 3, 2, 1), L.or_chain_bits(7, 3, 2, 2)}) == 3


@pytest.mark.parametrize("prec", [64, 32])
def test_uniform_moments(orc, prec):
    # test/rng_tests.jl:33-56 (5-sigma CLT band on mean and variance)
    n = 400_000
    r, q = orc.poses(prec, 123, 1, 1, n // 3 + 1)
    u = r.reshape(-1)[:n]
    m, v = u.mean(), u.var()
    assert abs(m - 0.5) < 5 * math.sqrt((1 / 12) / n)
    assert abs(v - 1 / 12) < 5 * math.sqrt((1 / 80 - (1 / 12) ** 2) / n)
    assert np.all((u >= 0) & (u < 1))


@pytest.mark.parametrize("prec", [64, 32])
def test_quaternions_uniform_on_so3(orc, prec):
    # test/rng_tests.jl quaternion CLT moments: unit norm, E[q_i^2] = 1/4, E[q_i] = 0
    n = 200_000
    _, q = orc.poses(prec, 5, 3, 1, n)
    tol = 1e-12 if prec == 64 else 1e-6
    assert np.all(np.abs(np.linalg.norm(q, axis=1) - 1) < tol)
    sd2 = math.sqrt((1 / 8 - 1 / 16) / n)  # Var(q_i^2) = E q^4 - 1/16 = 1/8 - 1/16
    assert np.all(np.abs((q**2).mean(axis=0) - 0.25) < 5 * sd2)
    assert np.all(np.abs(q.mean(axis=0)) < 5 * math.sqrt(0.25 / n))


def test_sincos2pi_accuracy_f64(orc):
    n = 100_001
    u = np.linspace(0, 1, n, endpoint=False)
    s, c = np.zeros(n), np.zeros(n)
    orc.lib().or_sincos2pi_f64(orc.P(u), n, orc.P(s), orc.P(c))
    tol = 1.2e-15  # the numpy reference itself rounds 2*pi*u (up to ~6e-16 near u = 1)
    assert np.max(np.abs(s - np.sin(2 * np.pi * u))) < tol
    assert np.max(np.abs(c - np.cos(2 * np.pi * u))) < tol


def test_sincos2pi_f32_correctly_rounded_exhaustive(orc):
    # Float32 sinpi(2u) / cospi(2u) of every FP32 uniform u = k 2^-24 (src/rng.jl:126-129): the
    # oracle's (and the library's) FP32 values must be the correctly rounded ones, +0 for zeros.
    # Reference: sin/cos((pi/2) r) in x87 extended precision (64-bit significand) after the exact
    # quadrant reduction 4u = q + r, rounded to FP32; any input whose extended value lies within
    # 1e-17 (relative) of an FP32 rounding midpoint is settled with mpmath at 50 digits.
    import mpmath as mp

    k = np.arange(2**24, dtype=np.int64)
    u = (k.astype(np.float64) * 2.0**-24).astype(np.float32)
    s, c = np.zeros(2**24, np.float32), np.zeros(2**24, np.float32)
    orc.lib().or_sincos2pi_f32(orc.P(u), 2**24, orc.P(s), orc.P(c))
    L = np.longdouble
    y = 4 * k  # 4u in units of 2^-24
    q = (y + 2**23) >> 24  # rint(4u), ties (r = 1/2) to even below
    q = np.where(((y & (2**24 - 1)) == 2**23) & ((q & 1) == 1), q - 1, q)
    r = (y - (q << 24)).astype(L) * L(2.0**-24)
    hp = L("1.570796326794896619231321691639751442")
    sr, cr = np.sin(hp * r), np.cos(hp * r)
    qi = q & 3
    ref = {"sin": np.select([qi == 0, qi == 1, qi == 2], [sr, cr, -sr], -cr),
           "cos": np.select([qi == 0, qi == 1, qi == 2], [cr, -sr, -cr], sr)}
    mp.mp.dps = 50
    for name, got in (("sin", s), ("cos", c)):
        e = ref[name]
        r32 = e.astype(np.float32) + np.float32(0)
        lo = np.nextafter(r32, np.float32(-np.inf)).astype(L)
        hi = np.nextafter(r32, np.float32(np.inf)).astype(L)
        m = r32.astype(L)
        dist = np.minimum(np.abs(e - (m + lo) / 2), np.abs(e - (m + hi) / 2)) / np.maximum(np.abs(e), L(1e-30))
        near = np.nonzero(dist < 1e-17)[0]
        for i in near:
            f = mp.sinpi if name == "sin" else mp.cospi
            r32[i] = round_f32(f(2 * mp.mpf(float(u[i]))))
        assert np.array_equal(got.view(np.uint32), r32.view(np.uint32)), name
    # spot checks of the extended-precision reference itself against mpmath
    for i in np.random.default_rng(3).integers(0, 2**24, 64):
        assert s[i].view(np.uint32) == round_f32(mp.sinpi(2 * mp.mpf(float(u[i])))).view(np.uint32)
        assert c[i].view(np.uint32) == round_f32(mp.cospi(2 * mp.mpf(float(u[i])))).view(np.uint32)


def round_f32(v):
    """The FP32 value nearest to the mpmath number v (ties to even), zero as +0."""
    f = np.float32(float(v))
    cands = [np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))]
    d = [abs(v - mp_of(x)) for x in cands]
    best = min(range(3), key=lambda i: (d[i], int(cands[i].view(np.uint32)) & 1))
    return cands[best] + np.float32(0)


def mp_of(x):
    import mpmath as mp

    return mp.mpf(float(x))


# ---------------------------------------------------------- Ewald (test/ewald_tests.jl)
def test_ewald_alpha_and_kmax(orc):
    # test/ewald_tests.jl:1-6
    a = orc.lib().or_ewald_alpha(12.0, 1e-6)
    assert erfc(a * 12.0) == pytest.approx(12.0 * 5e-7, rel=1e-9)
    assert orc.lib().or_ewald_kmax(a, 1e-6) == pytest.approx(2 * a * math.sqrt(-math.log(5e-7)))


def test_erfc_matches_scipy(orc):
    # test/ewald_tests.jl:8-29: the oracle evaluates erfc itself (glibc), which the reference's
    # erfc_dev / pair_erfc_dev series approximate at rtol 1e-11 / 1e-12
    for x in np.arange(0, 6.0001, 0.01):
        assert orc.lib().or_erfc(x) == pytest.approx(erfc(x), rel=1e-13)


def _nacl(a, rc):
    base = [((0, 0, 0), 1.0), ((0.5, 0.5, 0), 1.0), ((0.5, 0, 0.5), 1.0), ((0, 0.5, 0.5), 1.0),
            ((0.5, 0, 0), -1.0), ((0, 0.5, 0), -1.0), ((0, 0, 0.5), -1.0), ((0.5, 0.5, 0.5), -1.0)]
    A = np.diag([a, a, a])
    L = np.array([a, a, a])
    m = [int(math.ceil(2 * rc / L[i])) for i in range(3)]
    pos, q = [], []
    for k in range(m[2]):
        for j in range(m[1]):
            for i in range(m[0]):
                for f, c in base:
                    pos.append(A @ (np.array(f) + np.array([i, j, k])))
                    q.append(c)
    return A @ np.diag(m), np.array(pos), np.array(q), m


@pytest.mark.parametrize("rcf", [0.49, 2.0])
def test_madelung_nacl(orc, rcf):
    # test/ewald_tests.jl:31-53: -1.747565 per ion pair, rtol 1e-5
    a = 5.64
    rc, prec = a * rcf, 1e-8
    Asc, pos, q, m = _nacl(a, rc)
    alpha = orc.lib().or_ewald_alpha(rc, prec)
    ks, w, _ = orc.kvectors(Asc, orc.lib().or_ewald_kmax(alpha, prec))
    E = orc.ewald_energy(Asc, pos, q, np.arange(len(q)), alpha, rc, ks, w)
    KE = 14.399645351950548
    assert E / (4 * np.prod(m)) == pytest.approx(-1.747565 * KE / (a / 2), rel=1e-5)


def test_energy_independent_of_alpha(orc):
    # test/ewald_tests.jl:55-68
    rng = np.random.default_rng(3)
    A = np.diag([20.0, 20.0, 20.0])
    pos = rng.random((40, 3)) @ A.T
    q = np.array([0.5 if i % 2 == 0 else -0.5 for i in range(40)])
    Es = []
    for rc in (6.0, 8.0, 9.5):
        alpha = orc.lib().or_ewald_alpha(rc, 1e-8)
        ks, w, _ = orc.kvectors(A, orc.lib().or_ewald_kmax(alpha, 1e-8))
        Es.append(orc.ewald_energy(A, pos, q, np.arange(40), alpha, rc, ks, w))
    assert all(e == pytest.approx(Es[0], rel=1e-6) for e in Es)


def test_kvectors_brute_force_triclinic(orc, pa):
    # test/ewald_tests.jl:70-98 on the RUBTAK cell parameters
    A = pa.cell_matrix(14.7619, 14.80147, 14.76539, 59.84578, 60.04729, 59.8131)
    alpha = orc.lib().or_ewald_alpha(12.0, 1e-6)
    kmax = orc.lib().or_ewald_kmax(alpha, 1e-6)
    B = 2 * math.pi * np.linalg.inv(A).T
    lat = [np.linalg.norm(A[:, i]) for i in range(3)]
    N = max(int(math.ceil(kmax * l / (2 * math.pi))) for l in lat)
    cnt, wsum = 0, 0.0
    for n1 in range(0, 2 * N + 1):
        for n2 in range(-2 * N, 2 * N + 1):
            for n3 in range(-2 * N, 2 * N + 1):
                if n1 == n2 == n3 == 0:
                    continue
                k = B @ np.array([n1, n2, n3])
                if np.linalg.norm(k) <= kmax:
                    cnt += 1
                    wsum += 1.0 if n1 == 0 else 2.0
    ks, w, co = orc.kvectors(A, kmax)
    assert len(ks) == cnt and w.sum() == wsum
    # test/ewald_tests.jl:100-110: integer coefficients reproduce the vectors
    np.testing.assert_allclose(co @ B.T, ks, atol=1e-12)
    # the product's enumeration is the same list in the same order
    pks, pw, pco = pa.kvectors(A, kmax)
    assert np.array_equal(pco, co) and np.array_equal(pw, w)


def test_intramolecular_exclusion(orc):
    # test/ewald_tests.jl:112-122
    A = np.diag([30.0, 30.0, 30.0])
    pos = np.array([[15.0, 15.0, 15.0], [16.16, 15.0, 15.0]])
    q = np.array([0.7, -0.35])
    alpha = orc.lib().or_ewald_alpha(12.0, 1e-8)
    ks, w, _ = orc.kvectors(A, orc.lib().or_ewald_kmax(alpha, 1e-8))
    Esame = orc.ewald_energy(A, pos, q, [1, 1], alpha, 12.0, ks, w)
    Ediff = orc.ewald_energy(A, pos, q, [1, 2], alpha, 12.0, ks, w)
    assert Ediff - Esame == pytest.approx(14.399645351950548 * 0.7 * -0.35 / 1.16, rel=1e-3)


# ---------------------------------------------------------- rejection (test/reject_tests.jl)
def test_theta_F(orc, pa):
    # test/reject_tests.jl:1-11
    t64 = orc.lib().or_theta_f64()
    assert math.exp(-t64) == 0.0 and math.exp(-np.nextafter(t64, 0)) != 0.0
    assert 745 < t64 < 746
    t32 = np.float32(orc.lib().or_theta_f32())
    with np.errstate(under="ignore"):
        assert np.exp(-t32) == 0 and np.exp(-np.nextafter(t32, np.float32(0))) != 0
    assert 103 < t32 < 105
    assert float(pa.reject.theta_F(np.float64)) == t64
    assert np.float32(pa.reject.theta_F(np.float32)) == t32


def test_find_r0_sign_change(orc, pa):
    # test/reject_tests.jl:13-27
    rng = np.random.default_rng(1)
    for _ in range(200):
        s, e, K, a = 2 + 3 * rng.random(), 0.0005 + 0.02 * rng.random(), -20 * rng.random(), 0.2 + 0.3 * rng.random()
        r0 = orc.find_r0(s, e, K, a, math.inf)
        assert abs(orc.lib().or_pair_energy(r0, s, e, K, a)) < 1e-9 * e
        assert orc.lib().or_pair_energy(r0 * (1 - 1e-8), s, e, K, a) > 0
        assert orc.lib().or_pair_energy(r0 * 1.001, s, e, K, a) < 0
        assert float(pa.reject.find_r0(s, e, K, a, math.inf)) == pytest.approx(r0, rel=1e-13)


def test_find_r0_rho2_guards_and_clamps(orc, pa):
    # test/reject_tests.jl:29-32, 165-177, 192-205
    with pytest.raises(pa.ArgumentError, match="must be positive"):
        pa.reject.find_r0(3.0, 0.0, -1.0, 0.2, math.inf)
    with pytest.raises(pa.ArgumentError, match="must be negative"):
        pa.reject.find_r0(3.0, 0.01, 1.0, 0.2, math.inf)
    with pytest.raises(pa.ArgumentError, match="margin=0.0 must be positive"):
        pa.reject.find_rho2(3.0, 0.01, -14.0, 0.0, math.inf)
    assert pa.reject.find_rho2(3.0, 0.0, 0.0, 25.0, math.inf)[0] == 0
    assert pa.reject.find_rho2(3.0, 0.0, -14.0, 25.0, math.inf)[0] == 0
    s, e = 3.0, 0.01
    alpha = orc.lib().or_ewald_alpha(12.0, 1e-6)
    K = -14.399645351950548
    r0u = orc.find_r0(s, e, K, alpha, math.inf)
    assert orc.find_r0(s, e, K, alpha, 1.9) == 1.9
    assert orc.find_r0(s, e, K, alpha, 3.0) == r0u
    rho = math.sqrt(orc.find_rho2(s, e, K, 25.0, math.inf))
    assert math.sqrt(orc.find_rho2(s, e, K, 25.0, 1.0)) == 1.0
    assert math.sqrt(orc.find_rho2(s, e, K, 25.0, 3.0)) == rho
    assert float(pa.reject.find_rho2(s, e, K, 25.0, math.inf)[0]) == pytest.approx(rho * rho, rel=1e-14)


# ------------------------------------------------------- widom bookkeeping (test/widom_tests.jl)
def test_sys_of_index_and_counts(orc, pa):
    # test/widom_tests.jl:209-219
    for ninsert, nsys, run in ((37, 4, 3), (100, 7, 5), (11, 3, 2), (1, 1, 1), (500, 13, 1), (45, 2, 5)):
        counts = np.zeros(nsys, int)
        for g in range(1, ninsert + 1):
            s = orc.lib().or_sys_of_index(g, run, nsys)
            assert s == pa.sys_of_index(g, run, nsys)
            counts[s - 1] += 1
        out = np.zeros(nsys, np.int64)
        orc.lib().or_system_counts(ninsert, nsys, run, orc.P(out))
        assert list(counts) == list(out) == pa.system_counts(ninsert, nsys, run)


def test_reduce_overflow_names_system(pa):
    # test/widom_tests.jl:148-156
    with pytest.raises(pa.ArgumentError, match="system 4"):
        pa._reduce([math.inf, math.inf], [-math.inf, -math.inf], [50, 50], 1.0, 1.0, 4)


def test_boltzmann_weight(pa):
    # test/widom_tests.jl:1-41
    w, uw = pa.boltzmann_weight(1000.0, 0.0257)
    assert w == 0 and uw == 0
    w, uw = pa.boltzmann_weight(math.inf, 0.0257)
    assert w == 0 and uw == 0 and not math.isnan(uw)
    w, uw = pa.boltzmann_weight(np.float32(-100.0), np.float32(1.0))
    assert w == math.exp(100.0) and uw == -100.0 * math.exp(100.0)


# ------------------------------------------------ phase 0 and energies on synthetic systems
def small_charged_batch(pa, T=np.float64, cellwidth=2):
    fws, ff, guest, ewald, _ = pa.synthetic.co2(T=T, replication=(3, 3, 3))
    return pa.FrameworkBatch(fws, ff, guest, ewald, cellwidth=cellwidth), guest


@pytest.mark.parametrize("prec", [64, 32])
def test_phase0_stencil_equals_brute_force(pa, orc, prec):
    # test/widom_tests.jl:393-469: the per-site stencil flags exactly what a brute-force scan does
    batch, guest = small_charged_batch(pa)
    v, keep = oracle_view(orc, batch)
    kT = kT_of(pa, batch)
    rho2, reach0 = pa.build_rejection_tables(batch, kT)
    r, q = orc.poses(prec, 101, 1, 1, 4000)
    st = orc.hardcore_flags(v, prec, 0, r, q, rho2, reach0, brute=False)
    br = orc.hardcore_flags(v, prec, 0, r, q, rho2, reach0, brute=True)
    assert np.array_equal(st, br)
    # a small cubic cell whose cell width is below the guest reach (test/widom_tests.jl:451-468)
    A2 = pa.cell_matrix(20.0, 20.0, 20.0, 90, 90, 90)
    fw2 = pa.Framework(A2, [[0.5, 0.5, 0.5], [0.2, 0.7, 0.3]], ["H", "H"], ["H", "H"], [1.0, -1.0])
    ff2 = pa.ForceField(["H_", "G_"], [3.0, 3.0], [0.01, 0.01], cutoff=6.0, tail=False)
    g2 = pa.Guest([[0.0, 0, 0], [3.0, 0, 0]], [2, 2], [0.05, -0.05])
    b2 = pa.FrameworkBatch([fw2], ff2, g2, pa.EwaldParams(cutoff=6.0))
    v2, keep2 = oracle_view(orc, b2)
    rho2b, reach0b = pa.build_rejection_tables(b2, kT)
    r, q = orc.poses(prec, 202, 1, 1, 20000)
    st = orc.hardcore_flags(v2, prec, 0, r, q, rho2b, reach0b, brute=False)
    br = orc.hardcore_flags(v2, prec, 0, r, q, rho2b, reach0b, brute=True)
    assert np.array_equal(st, br) and st.sum() > 0


@pytest.mark.parametrize("prec", [64, 32])
def test_rejection_only_zero_weights_two_phase_equals_single(pa, orc, prec):
    # test/reject_tests.jl:129-163 and test/widom_tests.jl:300-338 on the oracle: every flagged
    # insertion has an exactly-zero FP64 weight, so two-phase and single-phase sums are equal
    fws, ff, guest, ewald, _ = pa.synthetic.co2(replication=(3, 3, 3))
    batch = pa.FrameworkBatch(fws, ff, guest, ewald)
    v, keep = oracle_view(orc, batch)
    kT = kT_of(pa, batch)
    rho2, reach0 = pa.build_rejection_tables(batch, kT)
    n = 3000
    two = orc.widom(v, prec, kT, n, 17, 4, pa.default_run(n, 1), True, rho2, reach0)
    one = orc.widom(v, prec, kT, n, 17, 4, pa.default_run(n, 1), False)
    flagged = two["flags"] == 1
    assert np.all(np.exp(-one["dU"][flagged] / kT) == 0)
    assert np.array_equal(two["sW"], one["sW"]) and np.array_equal(two["sUW"], one["sUW"])


def test_insertion_energy_vs_full_reference(pa, orc):
    # test/reference_tests.jl:1-60: production energy (coupled k, self term averaged into the
    # constant offset) vs the full-k oracle within 2 x self_term_halfrange
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    batch = pa.FrameworkBatch(fws, ff, guest, ewald)
    v, keep = oracle_view(orc, batch)
    fw = fws[0]
    A = fw.cell
    alpha = batch.alphas[0]
    kmax = pa.ewald_kmax(alpha, ewald.precision)
    ks, kp, S, _ = pa.full_ktables(A, pa.cartesian(fw), fw.charges, alpha, kmax)
    hpos = pa.cartesian(fw)
    htype = np.array([ff.typeindex(s + "_") for s in fw.symbols], dtype=np.int32)
    N = 3
    self_e = -pa.KE * alpha / math.sqrt(math.pi) * float(np.sum(guest.charges**2))
    excl = 0.0
    for a in range(N):
        for c in range(a + 1, N):
            r = float(np.linalg.norm(guest.sites[a] - guest.sites[c]))
            excl -= pa.KE * guest.charges[a] * guest.charges[c] * (1 - erfc(alpha * r)) / r
    counts = np.bincount(htype - 1, minlength=len(ff.names))
    gcounts = np.bincount(guest.types - 1, minlength=len(ff.names))
    old_offset = self_e + excl + pa.tail_delta(ff, counts, gcounts, pa.volume(A))
    rng = np.random.default_rng(21)
    L = orc.lib()
    nt = len(ff.names)
    a = [orc.c64(x) for x in (guest.sites.reshape(-1), guest.charges, ff.sigma.T.reshape(-1), ff.epsilon.T.reshape(-1),
                              hpos.reshape(-1), fw.charges, A.T.reshape(-1), ks.reshape(-1), kp,
                              np.stack([S.real, S.imag], 1).reshape(-1))]
    gti, hti = orc.c32i(guest.types), orc.c32i(htype)
    for _ in range(20):
        pos = orc.c64(A @ rng.random(3))
        q = rng.random(4) - 0.5
        q = orc.c64(q / np.linalg.norm(q))
        prod = orc.insertion_energy(v, 0, pos, q)[0] + batch.constant_offset[0]
        ref = L.or_insertion_energy_reference(orc.P(pos), orc.P(q), N, orc.P(a[0]), orc.P(gti), orc.P(a[1]), nt,
                                              orc.P(a[2]), orc.P(a[3]), ff.cutoff, ewald.cutoff, len(htype),
                                              orc.P(a[4]), orc.P(hti), orc.P(a[5]), orc.P(a[6]), alpha, len(ks),
                                              orc.P(a[7]), orc.P(a[8]), orc.P(a[9])) + old_offset
        assert abs(prod - ref) <= 2 * batch.self_term_halfrange[0] + 1e-12 * abs(ref)


def test_oracle_energy_equals_full_ewald_difference(pa, orc):
    # test/energy_tests.jl:164-206: the full-k oracle energy equals a from-scratch Ewald
    # difference (system with guest minus system without), rtol 1e-8
    rng = np.random.default_rng(7)
    A = pa.cell_matrix(21.0, 22.0, 23.0, 90, 95, 90)
    na = 40
    hf = rng.random((na, 3))
    hpos = hf @ A.T
    hq = rng.normal(0, 0.4, na)
    hq -= hq.mean()
    htype = np.ones(na, np.int32)
    gs = np.array([[0.0, 0, 0], [-1.16, 0, 0], [1.16, 0, 0]])
    gq = np.array([0.7, -0.35, -0.35])
    gt = np.array([2, 3, 3], np.int32)
    sig = np.array([3.0, 2.8, 3.05])
    eps = np.array([0.003, 0.0023, 0.0068])
    S2 = (sig[:, None] + sig[None, :]) / 2
    E2 = np.sqrt(eps[:, None] * eps[None, :])
    rc, prec = 10.0, 1e-7
    alpha = orc.lib().or_ewald_alpha(rc, prec)
    ks, w, _ = orc.kvectors(A, orc.lib().or_ewald_kmax(alpha, prec))
    V = abs(np.linalg.det(A))
    kp = w * np.array([orc.lib().or_pk(float(k @ k), alpha, V) for k in ks])
    Sh = orc.structure_factor(ks, hpos, hq)
    pos = A @ rng.random(3)
    q = rng.random(4) - 0.5
    q /= np.linalg.norm(q)
    L = orc.lib()
    a = [orc.c64(x) for x in (pos, q, gs.reshape(-1), gq, S2.T.reshape(-1), E2.T.reshape(-1), hpos.reshape(-1), hq,
                              A.T.reshape(-1), ks.reshape(-1), kp, np.stack([Sh.real, Sh.imag], 1).reshape(-1))]
    gti, hti = orc.c32i(gt), orc.c32i(htype)
    dU = L.or_insertion_energy_reference(orc.P(a[0]), orc.P(a[1]), 3, orc.P(a[2]), orc.P(gti), orc.P(a[3]), 3,
                                         orc.P(a[4]), orc.P(a[5]), rc, rc, na, orc.P(a[6]), orc.P(hti), orc.P(a[7]),
                                         orc.P(a[8]), alpha, len(ks), orc.P(a[9]), orc.P(a[10]), orc.P(a[11]))
    gpos = np.array([pos + pa.batch._rotate(q, s) for s in gs])
    allpos = np.vstack([hpos, gpos])
    allq = np.concatenate([hq, gq])
    mol = np.concatenate([np.arange(1, na + 1), np.zeros(3, int)])
    Ecoul = orc.ewald_energy(A, allpos, allq, mol, alpha, rc, ks, w) - \
        orc.ewald_energy(A, hpos, hq, np.arange(1, na + 1), alpha, rc, ks, w)
    invA = np.linalg.inv(A)
    Elj = 0.0
    for s in range(3):
        d = pa.minimum_image(A, invA, gpos[s] - hpos)
        r = np.linalg.norm(d, axis=1)
        x = (S2[gt[s] - 1, 0] / r[r < rc]) ** 6
        Elj += float(np.sum(4 * E2[gt[s] - 1, 0] * (x * x - x)))
    KE = pa.KE
    Eself = -KE * alpha / math.sqrt(math.pi) * float(np.sum(gq**2))
    Eexcl = 0.0
    for i in range(3):
        for j in range(i + 1, 3):
            r = float(np.linalg.norm(gpos[i] - gpos[j]))
            Eexcl -= KE * gq[i] * gq[j] * (1 - erfc(alpha * r)) / r
    Enet = 0.0  # neutral guest
    assert dU == pytest.approx(Elj + Ecoul - Eself - Eexcl - Enet, rel=1e-8)


def test_hardcore_bound_holds(pa, orc):
    # test/reject_tests.jl:103-127: dU - u_trigger >= -B_s + c_s - 1e-6 B_s on random poses
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    batch = pa.FrameworkBatch(fws, ff, guest, ewald)
    v, keep = oracle_view(orc, batch)
    Bs, cs = batch.bs[0], batch.constant_offset[0]
    assert math.isfinite(Bs) and Bs > 0
    A = batch.cells[0]
    invA = np.linalg.inv(A)
    rng = np.random.default_rng(3)
    gt = batch.guest_types - 1
    for _ in range(60):
        pos = A @ rng.random(3)
        q = rng.random(4) - 0.5
        q /= np.linalg.norm(q)
        dU = orc.insertion_energy(v, 0, pos, q)[0] + cs
        gs = np.array([pa.batch._rotate(q, s) for s in guest.sites])
        d0 = pa.minimum_image(A, invA, pos - batch.positions)
        u_trig = math.inf
        for a in range(3):
            r = np.linalg.norm(d0 + gs[a], axis=1)
            m = r < ff.cutoff
            ht = batch.types[m] - 1
            K = pa.KE * guest.charges[a] * batch.charges[m]
            u = pa.reject.pair_energy(r[m], batch.sigma[gt[a], ht], batch.epsilon[gt[a], ht], K, batch.alphas[0])
            if len(u):
                u_trig = min(u_trig, float(np.min(u)))
        if math.isfinite(u_trig):
            assert dU - u_trig >= -Bs + cs - 1e-6 * Bs


def test_ideal_gas_empty_box_oracle(pa, orc):
    # test/widom_tests.jl:43-56
    A = pa.cell_matrix(30.0, 30.0, 30.0, 90, 90, 90)
    fw = pa.Framework(A, np.zeros((0, 3)), [], [], np.zeros(0))
    ff = pa.ForceField(["X_"], [3.0], [0.001], cutoff=12.0, tail=False)
    g = pa.Guest(np.zeros((1, 3)), [1], np.zeros(1))
    b = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=12.0))
    v, keep = oracle_view(orc, b)
    kT = pa.KB * 300.0
    rho2, reach0 = pa.build_rejection_tables(b, kT)
    o = orc.widom(v, 64, kT, 10_000, 1, 10, pa.default_run(10_000, 1), True, rho2, reach0)
    r = pa._reduce(o["sW"][0], o["sUW"][0], o["n"][0], kT, b.volumes[0], 1)
    assert abs(r.mu_ex) < 1e-12
    assert r.K_H == pytest.approx(30.0**3 / kT)
    assert r.q_st == pytest.approx(kT)
    assert r.nsamples == 10_000


def test_single_lj_atom_radial_integral(pa, orc):
    # test/widom_tests.jl:97-114 (400k insertions here; within 4 standard errors)
    from scipy.integrate import quad
    Lb = 40.0
    A = pa.cell_matrix(Lb, Lb, Lb, 90, 90, 90)
    fw = pa.Framework(A, [[0.5, 0.5, 0.5]], ["X"], ["X"], [0.0])
    s, e, rc = 3.4, 0.0103, 12.0
    ff = pa.ForceField(["X_"], [s], [e], cutoff=rc, tail=False)
    g = pa.Guest(np.zeros((1, 3)), [1], np.zeros(1))
    b = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=rc))
    v, keep = oracle_view(orc, b)
    Tk = 300.0
    kT = pa.KB * Tk
    rho2, reach0 = pa.build_rejection_tables(b, kT)
    n = 400_000
    o = orc.widom(v, 64, kT, n, 2, 20, pa.default_run(n, 1), True, rho2, reach0, want_insertions=False)
    r = pa._reduce(o["sW"][0], o["sUW"][0], o["n"][0], kT, b.volumes[0], 1)
    u = lambda x: 4 * e * ((s / x) ** 12 - (s / x) ** 6)
    integral, _ = quad(lambda x: (1 - math.exp(-u(x) / kT)) * x * x, 1e-3, rc, epsabs=0, epsrel=1e-10, limit=200)
    expected = 1 - 4 * math.pi * integral / Lb**3
    meanW = r.K_H * kT / Lb**3
    errW = r.K_H_err * kT / Lb**3
    assert abs(meanW - expected) < 4 * errW


# ---------------------------------------------------------- RUBTAK (reference data files)
def test_rubtak_readers_reproduce_fixture(pa):
    # the readers on the reference's own files give the committed fixture's values exactly
    fw = pa.read_cif(reference_data("RUBTAK.cif"))
    ff = pa.read_forcefield(reference_data("trappe.yaml"))
    g = pa.read_guest(reference_data("co2.yaml"), ff)
    (sc,), ffx, gx, _, d = rubtak_case(pa)
    assert np.array_equal(fw.frac, np.array(d["framework"]["frac"])) and fw.symbols == d["framework"]["symbols"]
    assert np.array_equal(fw.charges, np.array(d["framework"]["charges"]))
    for n in ffx.names:
        i, j = ff.typeindex(n) - 1, ffx.typeindex(n) - 1
        assert ff.sigma[i, i] == ffx.sigma[j, j] and ff.epsilon[i, i] == ffx.epsilon[j, j]
    assert np.array_equal(g.sites, gx.sites) and np.array_equal(g.charges, gx.charges)


def test_rubtak_batch_known_answers(pa, orc):
    # test/structure_tests.jl:1-11, test/batch_tests.jl:1-30, 71-88:
    # 114 atoms, q1 = 2.38565, 3,078 atoms after 3x3x3, 190 coupled k-vectors, dropped |S| < 1e-9
    (sc,), ff, g, _, d = rubtak_case(pa)
    f = d["framework"]
    fw = pa.Framework(np.array(f["cell"]), np.array(f["frac"]), f["labels"], f["symbols"], np.array(f["charges"]))
    assert pa.natoms(fw) == 114 and fw.symbols[0] == "Zr" and fw.charges[0] == pytest.approx(2.38565)
    assert abs(pa.total_charge(fw)) < 1e-3
    sc = pa.replicate(fw, (3, 3, 3))
    assert pa.natoms(sc) == 3078 and sc.replication == (3, 3, 3)
    b = pa.FrameworkBatch([sc, sc], ff, g, pa.EwaldParams(cutoff=12.0, precision=1e-6))
    assert b.nsys == 2 and b.nframeworks() == 1 and list(b.framework_of) == [1, 1]
    assert list(b.atom_offsets) == [0, 3078]
    assert len(b.ks) == 190
    alpha = pa.ewald_alpha(12.0, 1e-6)
    ks, kp, S, co = pa.full_ktables(sc.cell, pa.cartesian(sc), sc.charges, alpha, pa.ewald_kmax(alpha, 1e-6))
    dropped = np.any(np.mod(co, 3) != 0, axis=1)
    assert int(np.sum(~dropped)) == 190
    assert np.all(np.abs(S[dropped]) < 1e-9)
    # the oracle's own k enumeration and structure factor agree
    oks, ow, oco = orc.kvectors(sc.cell, pa.ewald_kmax(alpha, 1e-6))
    assert np.array_equal(oco, co)
    np.testing.assert_allclose(orc.structure_factor(ks, pa.cartesian(sc), sc.charges), S, atol=1e-10)
    with pytest.raises(pa.ArgumentError, match="replicate"):
        pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=12.0))
    with pytest.raises(pa.ArgumentError, match="exceeds PAIR_ERFC_XMAX"):
        pa.FrameworkBatch([sc], ff, g, pa.EwaldParams(cutoff=12.0, precision=1e-12))
