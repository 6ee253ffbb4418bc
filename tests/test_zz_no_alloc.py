"""The allocation-free widom entry point (pa_widom_static) against pa_widom, through the C ABI.

pa_widom_static serves callers that may not allocate device memory during a call: it computes
what pa_widom computes with all per-call scratch in one static device array. Its block sums and
per-insertion energies must equal pa_widom's on two calls in a row, which also shows that the
shared array is cleared between calls; after those warm-up calls, a call of a shape not seen
before leaves the device's free memory and its default memory pool unchanged; a call beyond the
array's size limit is refused with PA_ERR_ARG. Kept in a file of its own that pytest collects
last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NINSERT, NBLOCKS, SEED = 100_000, 10, 3


def device_memory(device):
    """(free bytes of the device, (used, reserved) bytes of its default memory pool)."""
    from cuda.bindings import runtime as rt

    (err,) = rt.cudaDeviceSynchronize()  # pending stream-ordered frees settle first
    assert err == rt.cudaError_t.cudaSuccess
    err, free, total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    assert err == rt.cudaError_t.cudaSuccess
    vals = []
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        vals.append(int(v))
    return int(free), tuple(vals)


def call(pa, fn, ctx, dev, args, nsys):
    n = nsys * NBLOCKS
    lse, sw, suw = np.zeros(n), np.zeros(n), np.zeros(n)
    cnt = np.zeros(n, dtype=np.int64)
    dU = np.full(NINSERT, np.nan)
    sums = pa._lib.BlockSums(*(pa._lib.ptr(a) for a in (lse, sw, suw, cnt)), None)
    out = pa._lib.InsertionOut(pa._lib.ptr(dU), None, None)
    st = fn(ctx.handle, dev.handle, args, sums, out)
    return st, (lse, sw, suw, cnt, dU)


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_static_scratch_matches_widom_on_two_calls(pa, T):
    fws, ff, guest, ewald, _ = pa.synthetic.co2(T=T)
    batch = pa.FrameworkBatch(fws, ff, guest, ewald)
    backend = pa.B200Backend(0)
    ctx = backend.ctx
    dev = batch.device(ctx)
    kT = float(T(pa.KB * 298.15))
    rho2, reach0 = pa.build_rejection_tables(batch, kT)
    reach0 = np.ascontiguousarray(reach0.reshape(-1))
    args = pa._lib.WidomArgs()
    args.kT, args.ninsert, args.seed, args.nblocks = kT, NINSERT, SEED, NBLOCKS
    args.run, args.reject = pa.default_run(NINSERT, batch.nsys), 1
    args.rho2, args.reach0 = pa._lib.ptr(rho2), pa._lib.ptr(reach0)
    L = pa._lib.lib()
    st, ref = call(pa, L.pa_widom, ctx, dev, args, batch.nsys)
    assert st == 0
    for _ in range(2):
        st, got = call(pa, L.pa_widom_static, ctx, dev, args, batch.nsys)
        assert st == 0, L.pa_last_error(ctx.handle)
        for a, b in zip(got[:3], ref[:3]):
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)
        assert np.array_equal(got[3], ref[3])
        fin = np.isfinite(ref[4])
        assert np.array_equal(np.isfinite(got[4]), fin)
        np.testing.assert_allclose(got[4][fin], ref[4][fin], rtol=1e-12, atol=1e-12)
    # a shape not seen before allocates nothing: device free memory and the default pool's
    # used and reserved bytes are unchanged across the call
    free0, pool0 = device_memory(ctx.device)
    args.ninsert = 50_000
    args.run = pa.default_run(50_000, batch.nsys)
    st, got = call(pa, L.pa_widom_static, ctx, dev, args, batch.nsys)
    assert st == 0, L.pa_last_error(ctx.handle)
    free1, pool1 = device_memory(ctx.device)
    assert free1 == free0 and pool1 == pool0
    assert np.all(np.isfinite(got[4][:50_000]) | np.isinf(got[4][:50_000]))
    # beyond the static array's limit: refused before any device work
    args.ninsert = 200_000
    st, _ = call(pa, L.pa_widom_static, ctx, dev, args, batch.nsys)
    assert st == pa._lib.PA_ERR_ARG
    assert b"exceeds its maximum" in L.pa_last_error(ctx.handle)
