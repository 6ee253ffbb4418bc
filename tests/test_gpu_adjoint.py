"""Adjoint on the B200 (pa_widom_grad through pureadsorb_b200.widom_grad) against the oracle:
the device's weighted sums against the oracle's adjoint sums at the same poses and on the same
FP32 batch, and the assembled d ln K_H / dθ against central finite differences of the FP64
oracle's ln K_H with common random numbers."""
import numpy as np
import pytest

from conftest import kT_of, oracle_view
from test_adjoint import CO2Case, H, NBLOCKS, NINS, RUN, SEED

pytestmark = pytest.mark.gpu

# The device computes pair terms in FP32 and weights from FP32-path energies; the oracle is FP64
# throughout. Sums agree to about 1e-5 of their largest element; the stated bound is 1e-3.
SUM_REL = 1e-3


def _device(pa, backend, case, b32, fws=None):
    return pa.widom_grad(b32, case.guest, case.ff, T=298.15, ninsert=NINS, backend=backend, seed=SEED,
                         nblocks=NBLOCKS, run=RUN)


def _oracle_sums(pa, orc, b):
    kT = kT_of(pa, b)
    v, keep = oracle_view(orc, b)
    rho2, reach0 = pa.build_rejection_tables(b, kT)
    out = orc.widom(v, 32, kT, NINS, SEED, NBLOCKS, RUN, True, rho2, reach0)
    nat, nk = pa.adjoint.system_offsets(b)
    return orc.grad_sums(v, kT, NINS, RUN, out, nat, nk), kT


@pytest.fixture(scope="module")
def case(pa, orc):
    return CO2Case(pa, orc)


def test_device_sums_match_oracle(pa, orc, backend, case):
    b32 = case.batch(T=np.float32)
    res, grads = _device(pa, backend, case, b32)
    sums, kT = _oracle_sums(pa, orc, b32)
    g_or = pa.adjoint.assemble(b32, case.ff, 0, sums[0], kT)
    g = grads[0]
    assert g.xmax == pytest.approx(sums[0]["xmax"], abs=1e-3)
    assert g.sum_w == pytest.approx(g_or.sum_w, rel=1e-3)
    assert g.recomputed > 0
    for name in ("epsilon", "sigma", "charges"):
        a, o = getattr(g, name), getattr(g_or, name)
        scale = np.max(np.abs(o))
        assert np.max(np.abs(a - o)) <= SUM_REL * scale, (name, np.max(np.abs(a - o)) / scale)


@pytest.mark.parametrize("name,which", [("A_", "epsilon"), ("B_", "sigma"), ("O_co2", "epsilon"), ("C_co2", "sigma")])
def test_device_gradient_matches_fd(pa, backend, case, name, which):
    """d ln K_H / dθ from the device against central differences on the FP64 oracle (relative step
    1e-4, the same counter-based poses at θ ± h): agreement within 1e-3 relative."""
    res, grads = _device(pa, backend, case, case.batch(T=np.float32))
    t = case.ff.typeindex(name) - 1
    p = pa.forcefield.type_parameters(case.ff)[0 if which == "sigma" else 1][t]
    lp = case.lnW(case.batch(ff=case.ff_scaled(t, which, 1 + H)))
    lm = case.lnW(case.batch(ff=case.ff_scaled(t, which, 1 - H)))
    fd = (lp - lm) / (2 * H * p)
    assert getattr(grads[0], which)[t] == pytest.approx(fd, rel=1e-3)


def test_device_charge_gradient_matches_fd(pa, backend, case):
    res, grads = _device(pa, backend, case, case.batch(T=np.float32))
    gu = pa.fold_replicas(grads[0].charges, 216)
    scale = np.max(np.abs(gu))
    for u in (0, 7, 100):
        q = case.fws[0].charges[u]
        h = H * abs(q)
        fd = (case.lnW(case.batch(fws=case.fws_charge(u, h))) - case.lnW(case.batch(fws=case.fws_charge(u, -h)))) / (2 * h)
        assert abs(gu[u] - fd) <= 1e-3 * max(abs(fd), 0.05 * scale), (u, gu[u], fd)


def test_two_systems_share_a_framework(pa, orc, backend, case):
    """Two systems on one framework: every per-system sum stays with its own system."""
    b32 = pa.FrameworkBatch(case.fws * 2, case.ff, case.guest, case.ewald, T=np.float32, sk=case.sk)
    assert b32.nsys == 2 and len(b32.volumes) == 1
    res, grads = _device(pa, backend, case, b32)
    sums, kT = _oracle_sums(pa, orc, b32)
    for s in range(2):
        g_or = pa.adjoint.assemble(b32, case.ff, s, sums[s], kT)
        for name in ("epsilon", "sigma", "charges"):
            a, o = getattr(grads[s], name), getattr(g_or, name)
            assert np.max(np.abs(a - o)) <= SUM_REL * np.max(np.abs(o)), (s, name)


def test_lj_only_guest(pa, orc, backend):
    """Neutral single-site guest (no Ewald terms): LJ gradients only, zero charge gradients."""
    fws, ff, guest, ewald, prm = pa.synthetic.lj_ch4(T=np.float32)
    b32 = pa.FrameworkBatch(fws, ff, guest, ewald)
    res, grads = pa.widom_grad(b32, guest, ff, T=298.15, ninsert=NINS, backend=backend, seed=SEED, nblocks=NBLOCKS,
                               run=RUN)
    sums, kT = _oracle_sums(pa, orc, b32)
    g_or = pa.adjoint.assemble(b32, ff, 0, sums[0], kT)
    assert np.all(grads[0].charges == 0)
    for name in ("epsilon", "sigma"):
        a, o = getattr(grads[0], name), getattr(g_or, name)
        assert np.max(np.abs(a - o)) <= SUM_REL * np.max(np.abs(o)), name


def test_fp64_batch_is_refused(pa, backend, case):
    b64 = case.batch(T=np.float64)
    with pytest.raises(Exception, match="PA_PRECISION_F32"):
        _device(pa, backend, case, b64)


def test_lj_only_mode_keeps_lj_gradients(pa, backend, case):
    """charges=False skips the device's charge terms: the ε and σ derivatives are those of the full
    adjoint (to the rounding of their atomic accumulation order), and no charge gradient is made."""
    b32 = case.batch(T=np.float32)
    full, gf = _device(pa, backend, case, b32)
    lj, gl = pa.widom_grad(b32, case.guest, case.ff, T=298.15, ninsert=NINS, backend=backend, seed=SEED,
                           nblocks=NBLOCKS, run=RUN, charges=False)
    assert gl[0].charges is None
    assert gl[0].recomputed == 0 and gf[0].recomputed > 0
    assert lj[0].K_H == full[0].K_H
    for name in ("epsilon", "sigma"):
        a, f = getattr(gl[0], name), getattr(gf[0], name)
        assert np.max(np.abs(a - f)) <= 1e-9 * np.max(np.abs(f)), name
