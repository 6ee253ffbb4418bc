"""Batch construction on the B200: the FP64 device structure factor and guest self term
(FrameworkBatch(sk=Context.structure_factor, self_term=Context.self_term)) against the host's
FP64 evaluation of the same sums: S(k), the constant offset (which folds the self term's mean)
and the self term's half-range, to the rounding of the summation order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fullk", [False, True])
def test_device_structure_factor_and_self_term(pa, backend, fullk):
    fws, ff, guest, ewald, _ = pa.synthetic.co2(T=np.float32)
    host = pa.FrameworkBatch(fws, ff, guest, ewald, fullk=fullk)
    dev = pa.FrameworkBatch(fws, ff, guest, ewald, fullk=fullk, sk=backend.ctx.structure_factor,
                            self_term=backend.ctx.self_term)
    assert np.max(np.abs(dev.Shost - host.Shost)) <= 1e-9 * np.max(np.abs(host.Shost))
    assert np.allclose(dev.constant_offset, host.constant_offset, rtol=0, atol=1e-12)
    assert np.allclose(dev.self_term_halfrange, host.self_term_halfrange, rtol=1e-9, atol=1e-15)


def test_device_self_term_on_the_batched_frameworks(pa, backend):
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=6, T=np.float32, max_unit_atoms=300)
    host = pa.FrameworkBatch(fws, ff, guest, ewald)
    dev = pa.FrameworkBatch(fws, ff, guest, ewald, sk=backend.ctx.structure_factor, self_term=backend.ctx.self_term)
    assert np.allclose(dev.constant_offset, host.constant_offset, rtol=0, atol=1e-11)
    assert np.allclose(dev.self_term_halfrange, host.self_term_halfrange, rtol=1e-9, atol=1e-15)


def test_device_hardcore_bounds_hook(pa, backend):
    # FrameworkBatch(..., bounds=ctx.batch_bounds): B_s from the device through the batch's upload,
    # equal to the host loop's to rounding; the upload is kept, and the rejection tables and a
    # widom call on it work as with host bounds
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=5, max_unit_atoms=300)
    ctx = backend.ctx
    host = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    dev = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32, bounds=ctx.batch_bounds)
    assert len(dev._device) == 1
    fin = np.isfinite(host.bs)
    assert np.array_equal(fin, np.isfinite(dev.bs))
    np.testing.assert_allclose(dev.bs[fin], host.bs[fin], rtol=1e-10, atol=1e-12)
    raw = pa._widom(dev, guest, reject=True, T=298.15, ninsert=20_000, seed=3, nblocks=4, backend=backend,
                    segment_range=(0, 0))
    assert np.all(np.asarray(raw[3]) > 0)
    dev.drop_device()


# ------------------------------------------------- the rest of construction on the device
# pa_kvectors, pa_kmin_table and pa_cell_sort against the host builders on the CO2, RUBTAK and
# batched cells: enumeration, coefficients, weights, k-vectors, kmin and the cell sort bit for bit,
# the prefactors to the last bits of exp (2 ulp); pa_batch_rejection_tables against pa_rejection_tables bit
# for bit, on FP32 and FP64 uploads and after an in-place force-field change.

def _cells(pa):
    from conftest import rubtak_case

    out = [pa.synthetic.co2()[0][0], rubtak_case(pa)[0][0]]
    out += pa.synthetic.batched(nfw=6, max_unit_atoms=800)[0]
    return out


def test_device_kvectors(pa, backend):
    alpha = pa.ewald_alpha(12.0, 1e-6)
    kmax = pa.ewald_kmax(alpha, 1e-6)
    for fw in _cells(pa):
        A = fw.cell
        ks, w, coeffs = pa.ewald.kvectors(A, kmax)
        V = pa.volume(A)
        kpref = w * pa.pk(pa.ewald.k2_of(ks), alpha, V)
        dks, dw, dkp, dco = backend.ctx.kvectors(pa.cell.reciprocal_basis(A), pa.ewald.kvector_bounds(A, kmax), kmax,
                                                 alpha, V)
        assert np.array_equal(dco, coeffs) and np.array_equal(dw, w)
        assert np.array_equal(dks, ks)
        np.testing.assert_allclose(dkp, kpref, rtol=1e-15, atol=0)  # exp: host vs CUDA, last bits


def test_device_kmin_and_cell_sort(pa, backend):
    rng = np.random.default_rng(5)
    fws = _cells(pa)
    for fw in fws:
        n = len(fw.frac)
        types = rng.integers(1, 7, n).astype(np.int32)
        gq = np.array([0.7, -0.35, -0.35])
        assert np.array_equal(backend.ctx.kmin_table(gq, types, fw.charges, 6),
                              pa.reject.kmin_table(gq, types, fw.charges, 6))
        grid = pa.cell.grid_dims(pa.perpendicular_lengths(fw.cell), 2.0)
        perm, off = pa.cell.cell_sort(fw.frac, grid)
        dperm, doff = backend.ctx.cell_sort(fw.frac, grid)
        assert np.array_equal(dperm, perm) and np.array_equal(doff, off)
    # many atoms per cell, coordinates outside [0, 1) and on cell faces
    frac = np.concatenate([rng.random((40_000, 3)) * 3 - 1, np.repeat([[0.25, 0.5, 0.75]], 97, axis=0),
                           np.array([[0.0, 1.0, -1e-17]])])
    perm, off = pa.cell.cell_sort(frac, np.array([7, 5, 3]))
    dperm, doff = backend.ctx.cell_sort(frac, np.array([7, 5, 3]))
    assert np.array_equal(dperm, perm) and np.array_equal(doff, off)


def test_device_rejection_tables(pa):
    for T, case in ((np.float32, "co2"), (np.float64, "co2"), (np.float32, "batched")):
        be = pa.B200Backend(0)
        if case == "co2":
            fws, ff, guest, ewald, _ = pa.synthetic.co2()
        else:
            fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=8, max_unit_atoms=600)
        b = pa.FrameworkBatch(fws, ff, guest, ewald, T=T)
        for kT in (float(T(pa.KB * 298.15)), float(T(pa.KB * 77.0))):
            b.drop_host_caches()
            host = pa.build_rejection_tables(b, kT)
            b.drop_host_caches()
            dev = pa.build_rejection_tables(b, kT, be.ctx)
            assert np.array_equal(host[0], dev[0]) and np.array_equal(host[1], dev[1])
        b.drop_device()
    # after an in-place force-field change of the upload (the fitting step)
    fws, ff, guest, ewald, prm = pa.synthetic.fitting(nfw=12, max_unit_atoms=300, T=np.float32)
    be = pa.B200Backend(0)
    b = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    b.device(be.ctx)
    b2 = b.with_forcefield(pa.fit.scaled_forcefield(ff, prm["fitted_types"], prm["hidden"]), move_device=True,
                           device_bounds=True)
    kT = float(np.float32(pa.KB * 298.15))
    host = pa.build_rejection_tables(b2, kT)
    b2.drop_host_caches()
    dev = pa.build_rejection_tables(b2, kT, be.ctx)
    assert np.array_equal(host[0], dev[0]) and np.array_equal(host[1], dev[1])
    b2.drop_device()


def test_device_built_batch_equals_host_built(pa, backend):
    # FrameworkBatch(device=ctx): every table built on the device where it can be
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=6, max_unit_atoms=500, T=np.float32)
    host = pa.FrameworkBatch(fws, ff, guest, ewald)
    dev = pa.FrameworkBatch(fws, ff, guest, ewald, device=backend.ctx)
    for f in ("types", "atom_offsets", "k_offsets", "kcoeffs", "ncells", "cell_offsets", "cellgrid_offsets", "perm",
              "framework_of"):
        assert np.array_equal(np.asarray(getattr(dev, f)), np.asarray(getattr(host, f))), f
    for f in ("positions", "charges", "ks", "kmin"):
        assert np.array_equal(np.asarray(getattr(dev, f)), np.asarray(getattr(host, f))), f
    np.testing.assert_allclose(dev.kprefactor, host.kprefactor, rtol=1e-15, atol=0)
    assert np.max(np.abs(dev.Shost - host.Shost)) <= 1e-9 * np.max(np.abs(host.Shost))
    np.testing.assert_allclose(dev.constant_offset, host.constant_offset, rtol=0, atol=1e-11)
    fin = np.isfinite(host.bs)
    np.testing.assert_allclose(dev.bs[fin], host.bs[fin], rtol=1e-10)
    # widom on it with the rejection radii from the device equals widom with the host's, bit for bit
    be = pa.B200Backend(0, device_tables=True)
    kw = dict(reject=True, T=298.15, ninsert=60_000, seed=5, nblocks=4, segment_range=(0, 0))
    r_dev = pa._widom(dev, guest, backend=be, **kw)
    dev.drop_device()
    dev.drop_host_caches()
    r_host = pa._widom(dev, guest, backend=backend, **kw)
    for x, y in zip(r_dev, r_host):
        assert np.array_equal(x, y)
    dev.drop_device()
    host.drop_device()
