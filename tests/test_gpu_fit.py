"""Fitting path on the B200: hard-core bounds on the device against the host's, pair tables
replaced in place against a fresh upload, and an Adam fit of the palette's LJ scale factors that
recovers hidden parameters from FP64 targets."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T_K = 298.15


@pytest.fixture(scope="module")
def palette(pa):
    return pa.synthetic.fitting(nfw=16, max_unit_atoms=200, T=np.float32)


def test_device_bounds_match_host(pa, backend, palette):
    fws, ff, guest, ewald, prm = palette
    b = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    bs = b.device(backend.ctx).hardcore_bounds(b.nframeworks())
    assert np.allclose(bs, b.bs, rtol=1e-12, atol=0)
    co2 = pa.FrameworkBatch(*pa.synthetic.co2()[:4], T=np.float32)
    bs2 = co2.device(backend.ctx).hardcore_bounds(1)
    assert bs2[0] == pytest.approx(co2.bs[0], rel=1e-12)
    b.drop_device()
    co2.drop_device()


def test_pair_tables_in_place_equal_fresh_upload(pa, palette):
    fws, ff, guest, ewald, prm = palette
    be = pa.B200Backend(0)
    b = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    b.device(be.ctx)
    ffx = pa.fit.scaled_forcefield(ff, prm["fitted_types"], prm["hidden"])
    moved = b.with_forcefield(ffx, move_device=True)       # tables replaced in place
    fresh = pa.FrameworkBatch(fws, ffx, guest, ewald, T=np.float32)
    n = 16 * 4096
    ra = pa._widom(moved, guest, reject=True, T=T_K, ninsert=n, seed=4, nblocks=4, backend=be, segment_range=(0, 0))
    rb = pa._widom(fresh, guest, reject=True, T=T_K, ninsert=n, seed=4, nblocks=4, backend=be, segment_range=(0, 0))
    for x, y in zip(ra, rb):
        assert np.array_equal(x, y)
    moved.drop_device()
    fresh.drop_device()


def test_adam_recovers_hidden_scales(pa, palette):
    """16 frameworks, 2^13 insertions each, targets from the plain FP64 path at the hidden
    parameters; 120 Adam steps from the unscaled force field cut the loss by 1000x and move every
    scale factor towards its hidden value on the whole. (With 16 frameworks the 8 factors are
    weakly identifiable: epsilon and sigma of one type trade off, so the loss falls much further
    than the parameter error.)"""
    fws, ff, guest, ewald, prm = palette
    be = pa.B200Backend(0)
    per = 2**13
    n = len(fws) * per
    ffh = pa.fit.scaled_forcefield(ff, prm["fitted_types"], prm["hidden"])
    targets = pa.fit.target_lnkh(fws, ffh, guest, ewald, T=T_K, ninsert=n, seed=prm["seed"], backend=be)
    b = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    res = pa.fit.fit_lj_scales(b, guest, ff, prm["fitted_types"], targets, T=T_K, ninsert=n, steps=120, lr=2e-2,
                               seed=prm["seed"], backend=be)
    err0 = np.max(np.abs(1.0 - prm["hidden"]))
    err = np.max(np.abs(res.x - prm["hidden"]))
    print(f"\nfit: loss {res.loss[0]:.3e} -> {res.loss[-1]:.3e}, max scale error {err0:.3e} -> {err:.3e}, "
          f"{np.median(res.ms):.1f} ms per step")
    assert res.loss[-1] < 1e-3 * res.loss[0]
    assert err < err0
    assert np.linalg.norm(res.x - prm["hidden"]) < np.linalg.norm(1.0 - prm["hidden"])
    # what the data determine: along the loss's stiffest curvature directions (Gauss-Newton
    # eigenvectors at the fitted point) the error falls far more than the raw parameter error
    kw = dict(T=T_K, ninsert=n, seed=prm["seed"], backend=be, x_ref=prm["hidden"])
    fin = pa.fit.identifiability(b, guest, ff, prm["fitted_types"], res.x, targets, **kw)
    ini = pa.fit.identifiability(b, guest, ff, prm["fitted_types"], np.ones(8), targets, **kw)
    V = fin.eigenvectors
    stiff = fin.eigenvalues >= 1e-2 * fin.eigenvalues[0]
    e0 = np.abs(V.T @ (1.0 - prm["hidden"]))
    e1 = fin.error_along
    print(f"curvature eigenvalues {np.array2string(fin.eigenvalues, precision=2)}; error along them "
          f"{np.array2string(e0, precision=3)} -> {np.array2string(e1, precision=3)}; eps sigma^6 rel error "
          f"{np.array2string(ini.eps_sigma6_rel_error, precision=3)} -> "
          f"{np.array2string(fin.eps_sigma6_rel_error, precision=3)}")
    assert stiff.sum() >= 1
    assert np.linalg.norm(e1[stiff]) < 0.2 * np.linalg.norm(e0[stiff])
