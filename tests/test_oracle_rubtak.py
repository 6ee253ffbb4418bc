"""The oracle's Widom output against the results the reference records for RUBTAK 3x3x3 + CO2
(298.15 K, 12 A cutoffs, Ewald precision 1e-6, 10^6 insertions, seed 42, 20 blocks):

- kUPS's numbers, test/reference/rubtak_co2_kups.json, compared as test/reference_tests.jl:62-74
  does: |ours - theirs| < 3 hypot(SE_ours, SE_theirs) for mu_ex, K_H and q_st;
- PureAdsorb.jl's own FP64 numbers for the same case, docs/src/validation.md:50-52, the same way.

The pose stream here is the counter-based one (the reference draws from Julia's Xoshiro), so the
agreement is statistical. The oracle runs with its own batch builder and rejection tables; the
inputs come from tests/golden/rubtak_co2.json (made by make_rubtak_fixture.py from the reference's
data files)."""
import numpy as np

from conftest import rubtak_case


def oracle_rubtak(pa, orc):
    fws, ff, g, ew, d = rubtak_case(pa)
    frames = [(fw.cell, fw.frac, [ff.typeindex(s + "_") for s in fw.symbols], fw.charges, fw.replication)
              for fw in fws]
    quats = orc.poses(64, pa.batch.SELF_TERM_SEED, 0, 1, pa.batch.SELF_TERM_NORIENT)[1]
    ob = orc.OracleBatch(frames, (np.diag(ff.sigma), np.diag(ff.epsilon), ff.cutoff, ff.tail),
                         (g.sites, g.types, g.charges), ew.cutoff, ew.precision, 2.0, False, quats)
    v, keep = orc.view(ob, g.sites, g.charges, ff.cutoff, ew.cutoff)
    return ob, v, keep, d


def test_rubtak_co2_matches_recorded_results(pa, orc):
    ob, v, keep, d = oracle_rubtak(pa, orc)
    c = d["case"]
    # the reference batch tables: 3,078 atoms, 190 coupled k-vectors (test/batch_tests.jl:14,79)
    assert len(ob.positions) == 3078 and len(ob.ks) == 190
    kT = pa.KB * c["T"]
    rho2, reach0 = orc.rejection_tables(v, ob.bs, ob.kmin, kT, float(np.finfo(np.float64).eps))
    n, nb = c["ninsert"], c["nblocks"]
    out = orc.widom(v, 64, kT, n, c["seed"], nb, pa.default_run(n, 1), True, rho2, reach0, want_insertions=False)
    r = pa._reduce(out["sW"][0], out["sUW"][0], out["n"][0], kT, ob.volumes[0], 1)
    assert r.nsamples == n and r.nblocks == nb
    for src in ("kups", "pureadsorb_fp64"):
        for key in ("mu_ex", "K_H", "q_st"):
            m, s = d[src][key]["mean"], d[src][key]["sem"]
            ours, err = getattr(r, key), getattr(r, key + "_err")
            assert abs(ours - m) < 3 * np.hypot(err, s), (src, key, ours, err, m, s)
