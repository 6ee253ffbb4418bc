import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

# a checkout of the reference project (its data files), for the few tests that read them
# directly; those tests skip when PUREADSORB_REFERENCE is unset or does not exist
REFERENCE = os.environ.get("PUREADSORB_REFERENCE", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pa():
    return ge.load_package()


@pytest.fixture(scope="session")
def orc():
    return ge.load_oracle()


@pytest.fixture(scope="session")
def backend(pa):
    return pa.B200Backend(0)


def reference_data(name):
    """Path of a data file of the reference checkout, or skip (it is absent on GPU machines)."""
    p = os.path.join(REFERENCE, "data", name)
    if not REFERENCE or not os.path.exists(p):
        pytest.skip("reference data not available")
    return p


def oracle_view(orc, batch):
    return orc.view(batch, batch.guest_sites_orig, batch.guest_charges_orig, batch.cutoff, batch.ewald_cutoff)


def kT_of(pa, batch, T=298.15):
    return float(batch.T(pa.KB * T))


def rubtak_case(pa, T=np.float64):
    """RUBTAK 3x3x3 + CO2 from the committed fixture (tests/golden/rubtak_co2.json): frameworks,
    force field, guest, Ewald parameters and the fixture dict (case settings, recorded results)."""
    import json

    with open(os.path.join(ROOT, "tests", "golden", "rubtak_co2.json")) as fh:
        d = json.load(fh)
    f, c = d["framework"], d["case"]
    fw = pa.Framework(np.array(f["cell"]), np.array(f["frac"]), f["labels"], f["symbols"], np.array(f["charges"]),
                      (1, 1, 1), T)
    ffd = d["forcefield"]
    ff = pa.ForceField(ffd["names"], ffd["sigma"], ffd["epsilon"], cutoff=ffd["cutoff"], tail=ffd["tail"])
    gd = d["guest"]
    g = pa.Guest(np.array(gd["sites"]), [ff.typeindex(n) for n in gd["type_names"]], np.array(gd["charges"]),
                 gd["tc"], gd["pc"], gd["omega"])
    sc = pa.replicate(fw, tuple(c["replication"]))
    return [sc], ff, g, pa.EwaldParams(cutoff=c["ewald_cutoff"], precision=c["ewald_precision"]), d
