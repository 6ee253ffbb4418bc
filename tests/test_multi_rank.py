"""Multi-GPU sharding logic on CPU ranks (gloo, world size 2).

A job's PA_SEGMENT-insertion segments are split into contiguous ranges, one per rank; every rank
writes the (max, Σ w, Σ ΔU w) triplets of its own segments into a job-sized array, the arrays
are summed across ranks (the ranges are disjoint) and the library combines them into block sums.
Here the per-segment triplets come from the oracle's per-insertion energies (a CPU stand-in for
the device's segment reduction); the test checks that the sharded result equals the unsharded
one bit for bit and matches the oracle's own block sums.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

NINSERT, NBLOCKS, SEED = 24_000, 4, 11


def segment_table(pa, ninsert, nsys, run, nblocks):
    ns = pa.system_counts(ninsert, nsys, run)
    off = np.concatenate([[0], np.cumsum(ns)])
    segs = []
    for s in range(nsys):
        blen = ns[s] // nblocks
        for b in range(nblocks):
            k0, k1 = b * blen, (ns[s] if b == nblocks - 1 else (b + 1) * blen)
            for k in range(k0, k1, 2048):
                segs.append((s, b, off[s] + k, off[s] + min(k + 2048, k1)))
    return segs


def triplets(dU, kT, segs, lo, hi):
    out = np.zeros(3 * len(segs))
    for q in range(lo, hi):
        _, _, i0, i1 = segs[q]
        x = -dU[i0:i1] / kT
        m = np.max(x)
        if np.isneginf(m):
            out[3 * q:3 * q + 3] = (m, 0.0, 0.0)
            continue
        e = np.exp(x - m)
        nz = e != 0
        out[3 * q:3 * q + 3] = (m, float(np.sum(e[nz])), float(np.sum(dU[i0:i1][nz] * e[nz])))
    return out


def job():
    import sys
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    pa, orc = ge.load_package(), ge.load_oracle()
    fws, ff, guest, ewald, _ = pa.synthetic.co2(replication=(3, 3, 3))
    batch = pa.FrameworkBatch(fws + fws[:1], ff, guest, ewald)  # two systems, one framework
    v, keep = orc.view(batch, batch.guest_sites_orig, batch.guest_charges_orig, batch.cutoff, batch.ewald_cutoff)
    kT = float(pa.KB * 298.15)
    rho2, reach0 = pa.build_rejection_tables(batch, kT)
    run = pa.default_run(NINSERT, batch.nsys)
    ref = orc.widom(v, 64, kT, NINSERT, SEED, NBLOCKS, run, True, rho2, reach0)
    return pa, batch, kT, run, ref


def combine(pa, segs_arr, nsys, run):
    lse, sw, suw = (np.zeros(nsys * NBLOCKS) for _ in range(3))
    cnt = np.zeros(nsys * NBLOCKS, np.int64)
    sums = pa._lib.BlockSums(*(pa._lib.ptr(a) for a in (lse, sw, suw, cnt)), None)
    assert pa._lib.lib().pa_combine_segments(NINSERT, nsys, run, NBLOCKS, pa._lib.ptr(segs_arr), sums) == 0
    return lse, sw, suw, cnt


def worker(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pa, batch, kT, run, ref = job()
        segs = segment_table(pa, NINSERT, batch.nsys, run, NBLOCKS)
        lo, hi = len(segs) * rank // world, len(segs) * (rank + 1) // world
        mine = torch.from_numpy(triplets(ref["dU"], kT, segs, lo, hi))
        dist.all_reduce(mine)
        if rank == 0:
            np.save(os.path.join(outdir, "sharded.npy"), mine.numpy())
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_shards_combine_exactly(tmp_path):
    world = 2
    mp.spawn(worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    sharded = np.load(tmp_path / "sharded.npy")
    pa, batch, kT, run, ref = job()
    segs = segment_table(pa, NINSERT, batch.nsys, run, NBLOCKS)
    full = triplets(ref["dU"], kT, segs, 0, len(segs))
    assert np.array_equal(sharded, full)
    a = combine(pa, sharded, batch.nsys, run)
    b = combine(pa, full, batch.nsys, run)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    sW, sUW = pa.block_sums(a[0], a[1], a[2])
    np.testing.assert_allclose(sW, ref["sW"].reshape(-1), rtol=1e-12)
    np.testing.assert_allclose(sUW, ref["sUW"].reshape(-1), rtol=1e-10, atol=1e-300)
    assert np.array_equal(a[3], ref["n"].reshape(-1))


def grad_worker(rank, world, port, outdir):
    """Each rank takes the adjoint sums of its own half of the job's insertions (the rest masked
    as rejected, which carries zero weight), with its own shift; rank 0 combines the gathered
    shards."""
    import pickle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pa, batch, kT, run, ref = job()
        v, keep = pa_oracle_view(batch)
        flags = ref["flags"].copy()
        lo, hi = NINSERT * rank // world, NINSERT * (rank + 1) // world
        flags[:lo] = 1
        flags[hi:] = 1
        mine = grad_sums_oracle(pa, batch, kT, run, dict(ref, flags=flags))
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        if rank == 0:
            combined = [pa.adjoint.combine_sums([shards[r][s] for r in range(world)]) for s in range(batch.nsys)]
            with open(os.path.join(outdir, "grad.pkl"), "wb") as fh:
                pickle.dump(combined, fh)
    finally:
        dist.destroy_process_group()


def pa_oracle_view(batch):
    import sys
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    orc = ge.load_oracle()
    return orc.view(batch, batch.guest_sites_orig, batch.guest_charges_orig, batch.cutoff, batch.ewald_cutoff)


def grad_sums_oracle(pa, batch, kT, run, out):
    import sys
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    orc = ge.load_oracle()
    v, keep = pa_oracle_view(batch)
    nat, nk = pa.adjoint.system_offsets(batch)
    return orc.grad_sums(v, kT, NINSERT, run, out, nat, nk)


def test_two_rank_adjoint_shards_combine(tmp_path):
    import pickle
    world = 2
    mp.spawn(grad_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    with open(tmp_path / "grad.pkl", "rb") as fh:
        combined = pickle.load(fh)
    pa, batch, kT, run, ref = job()
    full = grad_sums_oracle(pa, batch, kT, run, ref)
    for s in range(batch.nsys):
        assert combined[s]["xmax"] == full[s]["xmax"]
        for k in ("sum_w", "d_epsilon", "d_sigma", "d_charge"):
            np.testing.assert_allclose(combined[s][k], full[s][k], rtol=1e-12, atol=1e-14 * np.max(np.abs(full[s][k])))
