import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

REFERENCE = "/root/reference"


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
    if not os.path.exists(p):
        pytest.skip("reference data not available")
    return p


def oracle_view(orc, batch):
    return orc.view(batch, batch.guest_sites_orig, batch.guest_charges_orig, batch.cutoff, batch.ewald_cutoff)


def kT_of(pa, batch, T=298.15):
    return float(batch.T(pa.KB * T))
