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
