"""Insertion into a loaded configuration on the B200 (pa_widom with pa_chain_args; Widom along an
NVT chain, src/nvt.jl:85-124): with no guests the cycles are exactly single-phase widom over the
same stream (poses and ΔU bit for bit, test/nvt_tests.jl's "N=0 reproduces Milestone A's widom"),
and with guests every insertion's ΔU matches the oracle's chain energy (host-guest, reciprocal
against the running S(k), guest-guest, constant term) at the device's poses within the FP32
tolerance of the parity tests."""
import numpy as np
import pytest

from test_chain import chain_view, small_charged
from test_gpu_parity import FAST_ABS, FAST_REL

pytestmark = pytest.mark.gpu

NPER = 4096


def _empty(pa, b, guest):
    return pa.SystemState(b, guest, np.zeros((0, 3)), np.zeros((0, 4)), np.zeros(b.nsys + 1, np.int64),
                          np.zeros(b.nsys, np.int64))


def test_no_guests_equals_singlephase_widom(pa, backend):
    fws, ff, guest, ewald, _ = pa.synthetic.co2(T=np.float32)
    b = pa.FrameworkBatch(fws * 2, ff, guest, ewald, fullk=True)  # two systems sharing one framework
    st = _empty(pa, b, guest)
    ref = {}
    pa._widom(b, guest, reject=False, T=298.15, ninsert=2 * 2 * NPER, seed=7, nblocks=2, run=1, backend=backend,
              insertions=ref, segment_range=(0, 0))
    for c in range(2):
        ins = {}
        W, UW, cnt = pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=NPER, seed=7, cycle=c,
                                    backend=backend, insertions=ins)
        assert list(cnt) == [NPER, NPER]
        for s in range(2):
            r = slice(s * 2 * NPER + c * NPER, s * 2 * NPER + (c + 1) * NPER)
            a = slice(s * NPER, (s + 1) * NPER)
            assert np.array_equal(ins["poses"][a], ref["poses"][r])
            assert np.array_equal(ins["dU"][a], ref["dU"][r])
    b.drop_device()
    pa.chain.system_batch(b).drop_device()


def _device_vs_oracle(pa, orc, b, st, guest, ff, ins, kT):
    sb = pa.chain.system_batch(b)
    v, keep = chain_view(pa, orc, b, st, 0)
    bad, n = 0, 0
    for s in range(b.nsys):
        sl = slice(s * NPER, (s + 1) * NPER)
        A = sb.cells[s]
        pos = ins["poses"][sl, :3] @ A.T
        ref = orc.chain_energy(v, s, pos, ins["poses"][sl, 3:], st.live_sites(guest, s))
        ref += pa.insertion_constant_term(ff, b, guest, s, st.nguests(s))
        dev = ins["dU"][sl]
        fin = np.isfinite(ref) & (ref < 50.0)  # the weight of larger ΔU is exp(-1900) or less
        err = np.abs(dev[fin] - ref[fin])
        tol = FAST_ABS + FAST_REL * np.abs(ref[fin])  # the guest-guest term is FP32
        bad += int(np.sum(err > tol))
        n += int(fin.sum())
        assert np.all(err <= 2 * tol), (s, np.max(err / tol))
        w_dev = np.exp(-dev / kT)
        w_ref = np.exp(-ref / kT)
        assert abs(np.log(w_dev.sum()) - np.log(w_ref.sum())) <= 1e-3
    assert bad <= 1e-4 * n


def test_loaded_configuration_against_oracle(pa, orc, backend):
    ff, guest, fw = small_charged(pa, T=np.float32)
    b = pa.FrameworkBatch([fw, fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    st = pa.SystemState.placed(b, guest, [0, 6, 20], T=298.15, seed=3, capacities=[2, 6, 24])
    kT = float(b.T(pa.KB * 298.15))
    ins = {}
    pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=NPER, seed=11, cycle=1, backend=backend,
                   insertions=ins)
    _device_vs_oracle(pa, orc, b, st, guest, ff, ins, kT)
    pa.chain.system_batch(b).drop_device()


def test_graph_replay_across_cycles(pa, backend):
    ff, guest, fw = small_charged(pa, T=np.float32)
    b = pa.FrameworkBatch([fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    st = pa.SystemState.placed(b, guest, [3, 5], T=298.15, seed=3)
    direct = {}
    for c in (0, 1):
        direct[c] = {}
        pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=NPER, seed=5, cycle=c, backend=backend,
                       insertions=direct[c])
    be = pa.B200Backend(0)
    be.ctx.set_tuning(use_graphs=True)
    for c in (0, 0, 1, 0, 1):  # first run, capture, replays with another cycle offset
        ins = {}
        pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=NPER, seed=5, cycle=c, backend=be, insertions=ins)
        assert np.array_equal(ins["dU"], direct[c]["dU"])
        assert np.array_equal(ins["poses"], direct[c]["poses"])
    pa.chain.system_batch(b).drop_device()


def test_widom_along_chain_blocks_are_cycles(pa, backend):
    ff, guest, fw = small_charged(pa, T=np.float32)
    b = pa.FrameworkBatch([fw, fw], ff, guest, pa.EwaldParams(cutoff=12.0, precision=1e-6), fullk=True)
    states = [pa.SystemState.placed(b, guest, [2, 4], T=298.15, seed=s) for s in (21, 22, 23)]
    res = pa.widom_along_chain(b, states, guest, ff, T=298.15, n_widom_per_cycle=NPER, seed=9, backend=backend)
    kT = float(b.T(pa.KB * 298.15))
    sW = np.zeros((2, 3))
    sUW = np.zeros((2, 3))
    for c, st in enumerate(states):
        W, UW, cnt = pa.widom_chain(b, st, guest, ff, T=298.15, n_widom_per_cycle=NPER, seed=9, cycle=c,
                                    backend=backend)
        sW[:, c], sUW[:, c] = W, UW
    for s in range(2):
        assert res[s].nblocks == 3 and res[s].nsamples == 3 * NPER
        V = float(np.float32(b.volumes[0]))
        assert res[s].K_H == pytest.approx(V * sW[s].sum() / (3 * NPER) / kT, rel=1e-12)
    pa.chain.system_batch(b).drop_device()
