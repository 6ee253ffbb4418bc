"""The adjoint workload at full size: the charged CO2 framework (5,832 atoms), 4,000,000 insertions,
seed 42, T = 298.15 K. d ln K_H / dθ from the device for the 14 per-type LJ parameters (ε and σ of
the 5 host and 2 guest types) and all 216 unit-cell charges, against central finite differences
(relative step 1e-4) of the FP64 oracle's ln K_H with common random numbers.

The finite differences evaluate the oracle's FP64 insertion energies at the base run's poses.
Insertions whose weight at the base parameters is below exp(-50) times the largest are left out of
every evaluation: a relative change of 1e-4 in one parameter moves no weight by more than a
factor e^{0.1} or so, so they stay below 1e-20 of the sum, far under the 1e-3 being checked."""
import math

import numpy as np
import pytest

from conftest import kT_of, oracle_view
from test_adjoint import CO2Case

pytestmark = pytest.mark.gpu

NINS = 4_000_000
SEED = 42
NBLOCKS = 10
H = 1.0e-4
WINDOW = 50.0


class HeavyFD:
    """ln <W> of a perturbed batch from the FP64 oracle energies of the base run's heavy poses."""

    def __init__(self, pa, orc, case, b):
        self.pa, self.orc, self.case = pa, orc, case
        self.kT = kT_of(pa, b)
        v, keep = oracle_view(orc, b)
        rho2, reach0 = pa.build_rejection_tables(b, self.kT)
        run = pa.default_run(NINS, 1)
        out = orc.widom(v, 32, self.kT, NINS, SEED, NBLOCKS, run, True, rho2, reach0)
        x = np.where(out["flags"] == 0, -out["dU"] / self.kT, -np.inf)
        keep_i = np.nonzero(x >= np.max(x) - WINDOW)[0]
        self.rpos = out["poses"][keep_i, :3]
        self.quat = np.ascontiguousarray(out["poses"][keep_i, 3:])
        self.nheavy = len(keep_i)
        self.base = self.lnW(b)
        self.lnW_full = math.log(float(np.sum(out["sW"])))

    def lnW(self, b):
        v, keep = oracle_view(self.orc, b)
        A = np.asarray(b.cells[0])
        pos = np.ascontiguousarray(self.rpos @ A.T)
        e = self.orc.insertion_energy(v, 0, pos, self.quat) + float(b.constant_offset[0])
        x = -e / self.kT
        m = np.max(x)
        return m + math.log(float(np.sum(np.exp(x - m))))


@pytest.fixture(scope="module")
def c3(pa, orc, backend):
    case = CO2Case(pa, orc)
    ctx = backend.ctx
    case.sk = lambda ks, pos, q: ctx.structure_factor(ks, pos, q)  # FP64 S(k) on the device
    b64 = case.batch()
    fd = HeavyFD(pa, orc, case, b64)
    res, grads = pa.widom_grad(case.batch(T=np.float32), case.guest, case.ff, T=298.15, ninsert=NINS,
                               backend=backend, seed=SEED, nblocks=NBLOCKS)
    return case, fd, res[0], grads[0]


def test_heavy_subset_reproduces_full_sum(c3):
    case, fd, res, g = c3
    assert fd.base == pytest.approx(fd.lnW_full, abs=1e-10)


def test_lj_gradients_match_fd(pa, c3):
    case, fd, res, g = c3
    errs = []
    for name in case.ff.names:
        t = case.ff.typeindex(name) - 1
        for which in ("epsilon", "sigma"):
            p = pa.forcefield.type_parameters(case.ff)[0 if which == "sigma" else 1][t]
            d = (fd.lnW(case.batch(ff=case.ff_scaled(t, which, 1 + H)))
                 - fd.lnW(case.batch(ff=case.ff_scaled(t, which, 1 - H)))) / (2 * H * p)
            ad = getattr(g, which)[t]
            errs.append((abs(ad - d) / abs(d), name, which, ad, d))
    worst = max(errs)
    print(f"\nC3 LJ: 14 parameters, worst relative error {worst[0]:.2e} ({worst[1]} {worst[2]}: "
          f"adjoint {worst[3]:.6g}, fd {worst[4]:.6g}); recomputed {g.recomputed}, heavy {fd.nheavy}")
    assert worst[0] <= 1e-3, worst


def test_unit_cell_charge_gradients_match_fd(pa, c3):
    case, fd, res, g = c3
    gu = pa.fold_replicas(g.charges, 216)
    fdv = np.zeros(216)
    for u in range(216):
        h = H * abs(case.fws[0].charges[u])
        fdv[u] = (fd.lnW(case.batch(fws=case.fws_charge(u, h))) - fd.lnW(case.batch(fws=case.fws_charge(u, -h)))) / (2 * h)
    scale = np.max(np.abs(fdv))
    rel = np.abs(gu - fdv) / np.abs(fdv)
    big = np.abs(fdv) >= 0.05 * scale
    print(f"\nC3 charges: 216 parameters, max |adjoint - fd| / max|fd| = {np.max(np.abs(gu - fdv)) / scale:.2e}, "
          f"worst relative error over the {int(big.sum())} with |fd| >= 5% of the largest = {np.max(rel[big]):.2e}")
    assert np.max(np.abs(gu - fdv)) <= 1e-3 * scale
    assert np.max(rel[big]) <= 1e-3
