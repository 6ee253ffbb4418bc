"""Writes tests/golden/rubtak_co2.json: the RUBTAK + CO2 case of PureAdsorb.jl's own validation,
parsed from the reference checkout's data files with this package's readers, together with the
results the reference records for it.

    python tests/golden/make_rubtak_fixture.py <reference checkout>

Inputs read from the checkout (the data files are kUPS's examples, copied unchanged into the
reference, data/NOTICE):
- data/RUBTAK.cif (114-atom P1 cell with partial charges), data/trappe.yaml, data/co2.yaml;
- test/reference/rubtak_co2_kups.json: kUPS's mu_ex, K_H, q_st and their standard errors for
  RUBTAK 3x3x3 + CO2, 298.15 K, 12 A cutoffs, Ewald precision 1e-6, 10^6 insertions, seed 42;
- docs/src/validation.md:50-52: PureAdsorb.jl's own FP64 numbers for the same case (20 blocks),
  copied below as numbers because the document is prose.

Only the force-field types the case uses are kept. The fixture lets the tests run this case where
the reference checkout is absent.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

# docs/src/validation.md:50-52 (PureAdsorb column): mu_ex (eV), K_H (A^3/eV), q_st (eV), each +- SE
PUREADSORB_FP64 = {"mu_ex": {"mean": -0.1436470, "sem": 0.0002190},
                   "K_H": {"mean": 6.410616e8, "sem": 5.4634e6},
                   "q_st": {"mean": 0.2629071, "sem": 0.0002836}}


def main(ref):
    import __graft_entry__ as ge

    pa = ge.load_package()
    data = lambda *p: os.path.join(ref, *p)
    fw = pa.read_cif(data("data", "RUBTAK.cif"))
    ff = pa.read_forcefield(data("data", "trappe.yaml"))
    g = pa.read_guest(data("data", "co2.yaml"), ff)
    with open(data("test", "reference", "rubtak_co2_kups.json")) as fh:
        kups = json.load(fh)
    used = sorted({s + "_" for s in fw.symbols} | {ff.names[t - 1] for t in g.types}, key=ff.typeindex)
    sig = {n: float(ff.sigma[ff.typeindex(n) - 1, ff.typeindex(n) - 1]) for n in used}
    eps = {n: float(ff.epsilon[ff.typeindex(n) - 1, ff.typeindex(n) - 1]) for n in used}
    out = {
        "source": "reference data/RUBTAK.cif, data/trappe.yaml, data/co2.yaml (kUPS examples, Apache-2.0)",
        "framework": {"cell": fw.cell.tolist(), "frac": fw.frac.tolist(), "labels": fw.labels, "symbols": fw.symbols,
                      "charges": fw.charges.tolist()},
        "forcefield": {"names": used, "sigma": [sig[n] for n in used], "epsilon": [eps[n] for n in used],
                       "cutoff": ff.cutoff, "tail": ff.tail},
        "guest": {"sites": g.sites.tolist(), "type_names": [ff.names[t - 1] for t in g.types],
                  "charges": g.charges.tolist(), "tc": g.tc, "pc": g.pc, "omega": g.omega},
        "case": {"replication": [3, 3, 3], "T": 298.15, "ninsert": 1_000_000, "seed": 42, "nblocks": 20,
                 "ewald_cutoff": 12.0, "ewald_precision": 1.0e-6},
        "kups": {k: {"mean": kups[k]["mean"], "sem": kups[k]["sem"]} for k in ("mu_ex", "K_H", "q_st")},
        "pureadsorb_fp64": PUREADSORB_FP64,
    }
    with open(os.path.join(HERE, "rubtak_co2.json"), "w") as fh:
        json.dump(out, fh, indent=1)
        fh.write("\n")


if __name__ == "__main__":
    main(sys.argv[1])
