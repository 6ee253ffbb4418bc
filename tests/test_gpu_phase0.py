"""Phase 0 of the FP32 path on a B200 against the oracle's per-site stencil scan: the warp kernel
(one region of cells per 32 insertions, strict tests queued and decided in parallel) must flag
exactly the insertions the stencil scan flags, including

- several systems of one framework in the same warps (one group per system);
- finer cell grids (a larger stencil reach) and coarser ones;
- a cell whose stencil is as wide as the grid (the per-site scan inside the kernel);
- a cell wide enough that most insertions survive.

Flags and poses are compared bit for bit (test/widom_tests.jl:393-469 asks the stencil scan to
equal a brute-force scan, which the oracle pins separately)."""
import numpy as np
import pytest

from conftest import kT_of, oracle_view

pytestmark = pytest.mark.gpu


def flags_both(pa, orc, batch, guest, ninsert, seed, backend, nblocks=4):
    ins = {}
    pa._widom(batch, guest, reject=True, T=298.15, ninsert=ninsert, seed=seed, nblocks=nblocks, insertions=ins,
              backend=backend, segment_range=(0, 0))
    v, keep = oracle_view(orc, batch)
    kT = kT_of(pa, batch)
    rho2, reach0 = pa.build_rejection_tables(batch, kT)
    run = pa.default_run(ninsert, batch.nsys)
    ref = orc.widom(v, 32, kT, ninsert, seed, nblocks, run, True, rho2, reach0)
    return ins, ref


def check(ins, ref):
    assert np.array_equal(ins["poses"], ref["poses"])
    assert np.array_equal(ins["flags"], ref["flags"])
    surv = ref["flags"] == 0
    assert np.all(np.isinf(ins["dU"][~surv]))
    assert np.all(np.isfinite(ins["dU"][surv]))


@pytest.mark.parametrize("cellwidth", [1.0, 2.0, 3.0])
def test_co2_cell_widths(pa, orc, backend, cellwidth):
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, cellwidth=cellwidth, T=np.float32)
    ins, ref = flags_both(pa, orc, batch, guest, 40_000, 11, backend)
    check(ins, ref)
    assert 0 < int(ref["flags"].sum()) < len(ref["flags"])


def test_two_systems_one_framework(pa, orc, backend):
    # the same framework twice: one deduplicated framework, two systems whose insertions share the
    # framework's sub-bins, so warps hold lanes of both systems
    fws, ff, guest, ewald, _ = pa.synthetic.co2()
    batch = pa.FrameworkBatch([fws[0], fws[0]], ff, guest, ewald, T=np.float32)
    assert batch.nsys == 2 and batch.nframeworks() == 1
    ins, ref = flags_both(pa, orc, batch, guest, 40_000, 23, backend)
    check(ins, ref)


@pytest.mark.parametrize("cellwidth", [2.0, 8.0])
def test_small_cell(pa, orc, backend, cellwidth):
    # a 20 A cubic cell with two atoms and a 3 A guest; with 8 A cells the stencil covers the whole
    # 2 x 2 x 2 grid on every axis (the per-site scan), with 2 A cells it does not (the region)
    A = pa.cell_matrix(20.0, 20.0, 20.0, 90, 90, 90)
    fw = pa.Framework(A, [[0.5, 0.5, 0.5], [0.2, 0.7, 0.3]], ["H", "H"], ["H", "H"], [1.0, -1.0])
    ff = pa.ForceField(["H_", "G_"], [3.0, 3.0], [0.01, 0.01], cutoff=6.0, tail=False)
    g = pa.Guest([[0.0, 0, 0], [3.0, 0, 0]], [2, 2], [0.05, -0.05])
    batch = pa.FrameworkBatch([fw], ff, g, pa.EwaldParams(cutoff=6.0), cellwidth=cellwidth, T=np.float32)
    ins, ref = flags_both(pa, orc, batch, g, 20_000, 202, backend)
    check(ins, ref)
    assert int(ref["flags"].sum()) > 0


def test_batched_frameworks(pa, orc, backend):
    fws, ff, guest, ewald, _ = pa.synthetic.batched(nfw=6, max_unit_atoms=400)
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    ins, ref = flags_both(pa, orc, batch, guest, 60_000, 31, backend)
    check(ins, ref)
