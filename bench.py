"""Widom insertion throughput on B200: the FP32 path on the charged rigid-CO2 workload.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--ninsert n]

One step = one widom call over the workload's 1,000,000 insertions (5,832-atom framework, 3-site
CO2, 227 coupled k-vectors). `value` times the device pipeline with the batch resident in HBM
(CUDA events on the context's stream, L2 flushed between steps by a 256 MB write); `e2e` times
the public API call widom(batch, guest; T, ninsert, seed, backend) from host arrays, re-uploading
the batch every step. Under torchrun each rank processes its own contiguous share of the
PA_SEGMENT-insertion segments of an N x 1e6 job (weak scaling); rank 0 gathers the segment
triplets and combines them exactly.
"""
import argparse
import json
import math
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FP32_PEAK_NOMINAL = 148 * 128 * 2 * 1.965e9 / 1e12  # TFLOP/s at the maximum SM clock
# DRAM bytes (read + write) of one k_energy32 launch on this workload, per bin width (the
# autotuner's choice), from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum); they
# cannot be measured inside the bench
# (with the default FP32/FP64 split)
ENERGY32_TRAFFIC_BYTES = {3.0: 130.300928e6 + 9.088256e6, 3.5: 105.949696e6 + 8.178432e6}
# Warp instructions of one k_energy32 launch on this workload (smsp__inst_executed.sum from the same
# captures): the issue-slot roofline divides them by the launch's CUDA-event time
ENERGY32_INSTRUCTIONS = {3.0: 1469443993, 3.5: 1513756043}
ISSUE_PER_CYCLE = 148 * 4  # one warp instruction per cycle per SM sub-partition
FP64_PEAK_NOMINAL = 148 * 64 * 2 * 1.965e9 / 1e12  # TFLOP/s: 64 FP64 FMA lanes per SM
# the metric and workload names of both arms (ours and the reference's CPU implementation)
METRIC = "Widom insertions/s (CO2, 5,832-atom framework)"
WORKLOAD = "co2_5832_atoms_3x3x3_monoclinic"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--ninsert", type=int, default=1_000_000)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-fit", action="store_true")
    p.add_argument("--no-chain", action="store_true")
    p.add_argument("--no-parity", action="store_true", help="skip the per-insertion parity fractions")
    p.add_argument("--no-ch4", action="store_true", help="skip the CH4 configuration")
    p.add_argument("--no-all-fp32", action="store_true", help="skip the all-FP32 comparison steps")
    p.add_argument("--no-tune", action="store_true", help="default bin width and grid (e.g. for profiling)")
    p.add_argument("--bin-width", type=float, default=0.0, help="with --no-tune: this bin width (Å) instead of 3.0")
    return p.parse_args()


class Clocks:
    """SM clock and throttle reasons sampled through NVML (read-only) every 5 ms during the timed
    region; the summary reports "unsampled" when NVML is unavailable. The NVML device is found by
    the CUDA device's PCI address, since NVML's indices ignore CUDA_VISIBLE_DEVICES."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, device):
        self.device = device
        self.samples = []  # (sm MHz, reason bits)
        self.max_mhz = None
        self.pci = None
        self.stop = threading.Event()

    def handle(self, pynvml):
        import torch
        p = torch.cuda.get_device_properties(self.device)
        self.pci = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        return pynvml.nvmlDeviceGetHandleByPciBusId(self.pci.encode())

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = self.handle(pynvml)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    try:
                        self.samples.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM),
                                             pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)))
                    except Exception:
                        pass
                    time.sleep(0.005)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = sorted({name for _, bits in self.samples for bit, name in self.REASONS.items() if bits & bit})
        return {"sm_mhz": float(np.median([m for m, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "pci_bus_id": self.pci}


def load_peaks():
    try:
        with open(PEAKS) as fh:
            return json.load(fh)
    except OSError:
        return {}


def fp32_peak(torch):
    """The FP32 FMA peak the energy kernel's roofline uses (TFLOP/s): the nominal figure at the
    maximum SM clock. The measured peaks file holds HBM copy bandwidth and bf16 GEMM throughput
    only, neither of which bounds this FP32 CUDA-core kernel."""
    return FP32_PEAK_NOMINAL


def workload(pa, T):
    fws, ff, guest, ewald, prm = pa.synthetic.co2(T=T)
    return pa.FrameworkBatch(fws, ff, guest, ewald), guest, prm


def count_pairs(batch, poses, near_radius=0.0):
    """Mean numbers of (site, atom) pairs inside the LJ and the Ewald cutoff per insertion, and
    of pairs inside either cutoff closer than near_radius, for survivors' poses (fractional
    position, quaternion) of a one-framework batch: one minimum image per atom, as the
    reference's insertion_energy visits them (numpy, FP64)."""
    A = np.asarray(batch.cells[0])
    iA = np.linalg.inv(A)
    atoms = np.asarray(batch.positions)
    sites = np.asarray(batch.guest_sites_orig)
    rl2, re2 = batch.cutoff ** 2, batch.ewald_cutoff ** 2
    nl = ne = nn = 0
    for p in poses:
        pos = A @ p[:3]
        u, w = p[3:6], p[6]
        for g in sites:
            t = 2 * np.cross(u, g)
            r = pos + g + w * t + np.cross(u, t)
            d = r - atoms
            d -= (A @ np.rint(iA @ d.T)).T
            r2 = np.einsum("ij,ij->i", d, d)
            nl += int(np.sum(r2 < rl2))
            ne += int(np.sum(r2 < re2))
            nn += int(np.sum((r2 < near_radius ** 2) & ((r2 < rl2) | (r2 < re2))))
    n = max(1, len(poses))
    return nl / n, ne / n, nn / n


class OracleWorkload:
    """The CO2 workload as the CPU implementation sees it: the oracle's own FrameworkBatch builder
    (dedup, compact types, cell sort, k tables, self term, constant offset, B_s and kmin) and its
    own rejection tables, from the same synthetic frameworks, force field and guest. Nothing of
    the product library is loaded on this path; `product_library_loaded` checks that."""

    def __init__(self, pa, orc, T_K=298.15):
        fws, ff, guest, ewald, prm = pa.synthetic.co2(T=np.float64)
        frames = [(fw.cell, fw.frac, [ff.typeindex(s + "_") for s in fw.symbols], fw.charges, fw.replication)
                  for fw in fws]
        # the self term's orientations: the pose stream's quaternions for its fixed seed
        quats = orc.poses(64, pa.batch.SELF_TERM_SEED, 0, 1, pa.batch.SELF_TERM_NORIENT)[1]
        self.orc, self.prm = orc, prm
        self.b = orc.OracleBatch(frames, (np.diag(ff.sigma), np.diag(ff.epsilon), ff.cutoff, ff.tail),
                                 (guest.sites, guest.types, guest.charges), ewald.cutoff, ewald.precision, 2.0,
                                 False, quats)
        self.v, self.keep = orc.view(self.b, guest.sites, guest.charges, ff.cutoff, ewald.cutoff)
        self.kT = float(np.float64(pa.KB * T_K))
        self.natoms = int(len(self.b.positions))
        self.coupled_k = int(self.b.k_offsets[-1])

    def rejection_tables(self):
        """The rejection radii of one call, recomputed like every reference widom call does."""
        return self.orc.rejection_tables(self.v, self.b.bs, self.b.kmin, self.kT, float(np.finfo(np.float64).eps))

    def widom(self, n, nthreads=0):
        rho2, reach0 = self.rejection_tables()
        run = max(1, min(256, n // 4))  # default_run for one system (src/widom.jl:39)
        return self.orc.widom(self.v, 64, self.kT, n, self.prm["seed"], self.prm["nblocks"], run, True, rho2, reach0,
                              nthreads=nthreads, want_insertions=False)


def product_library_loaded():
    """True when this process has mapped the product's CUDA library."""
    try:
        with open("/proc/self/maps") as fh:
            return "libpureadsorb_b200.so" in fh.read()
    except OSError:
        return False


def cpu_baseline_port(wl, ninsert_full, target_s=12.0, nthreads=0):
    """Times the oracle (FP64 C++ restatement of the reference CPU path, OpenMP over the host
    cores) on a bounded sample of the same workload, rejection tables included in every call;
    returns (insertions/s, sample size, cores)."""
    n = 4000
    while True:
        t0 = time.perf_counter()
        wl.widom(n, nthreads=nthreads)
        dt = time.perf_counter() - t0
        if dt > 0.25 * target_s or n >= ninsert_full:
            return n / dt, n, (nthreads or os.cpu_count())
        n = int(min(ninsert_full, n * max(2.0, 0.5 * target_s / max(dt, 1e-3))))


def bench_config(ninsert, world, natoms, coupled_k, prm):
    """The workload description both arms print (same keys and values for the same run)."""
    return {"workload": WORKLOAD, "ninsert_per_gpu": ninsert, "ninsert_total": ninsert * world, "natoms": natoms,
            "guest_sites": 3, "coupled_k": coupled_k, "nblocks": prm["nblocks"], "seed": prm["seed"],
            "T_K": prm["T"], "l2": "flushed between steps (256 MB write)", "parallelism": f"shard{world}"}


def chain_workload(pa, orc, backend, torch, stream, flush, no_cpu=False):
    """Widom along an NVT chain on the CO2 framework: its full k table (fullk, every k-vector of
    the supercell), two systems sharing the framework at 10 and 40 CO2 guests (placed clear of the
    host's hard core), 2^18 insertions per system per cycle, no rejection, as widom_chain_kernel!
    computes them; CUDA events around each cycle's call (graph-replayed, the cycle index moving the
    pose stream on), per-kernel times from one timed call, and the FP64 oracle's chain energy on the
    host cores over a sample of the same insertions."""
    ctx = backend.ctx
    fws, ff, guest, ewald, prm = pa.synthetic.co2(T=np.float32)
    t0 = time.perf_counter()
    b = pa.FrameworkBatch(fws * 2, ff, guest, ewald, fullk=True, sk=ctx.structure_factor, self_term=ctx.self_term)
    st = pa.SystemState.placed(b, guest, [10, 40], T=prm["T"], seed=1001)
    build_s = time.perf_counter() - t0
    nper, T, seed = 2**18, prm["T"], prm["seed"]
    ctx.set_tuning(bin_width=3.5, ctas_per_sm=8, use_graphs=True)

    def cycle(c, **kw):
        return pa.widom_chain(b, st, guest, ff, T=T, n_widom_per_cycle=nper, seed=seed, cycle=c, backend=backend, **kw)

    for c in range(2):
        cycle(c)
    ms = []
    for c in range(2, 7):
        flush.zero_()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cycle(c)
        e.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(e))
    ms_cycle = float(np.median(ms))
    ctx.set_timing(True)
    k0, _ = ctx.kernel_times()
    cycle(7)
    torch.cuda.synchronize()
    k1, _ = ctx.kernel_times()
    ctx.set_timing(False)
    kd = k1 - k0
    out = {"workload": "chain_co2_5832_atoms_fullk_2_systems", "systems": 2, "guests": [10, 40],
           "k_vectors_per_system": int(len(b.ks)), "ninsert_per_cycle": 2 * nper, "ms_per_cycle": ms_cycle,
           "value": 2 * nper / (ms_cycle / 1e3), "unit": "insertions/s",
           "kernel_ms": {"poses": float(kd[0]), "scan_scatter": float(kd[1]), "energy": float(kd[2]),
                         "guest_guest": float(kd[7]), "reciprocal_combine": float(kd[6]), "segment_reduce": float(kd[3])},
           "build_s": build_s}
    if not no_cpu:
        # the oracle's FP64 chain energy at the device's poses of a sample cycle, OpenMP on the host
        ns = 4096
        ins = {}
        pa.widom_chain(b, st, guest, ff, T=T, n_widom_per_cycle=ns, seed=seed, cycle=0, backend=backend,
                       insertions=ins)
        sb = pa.chain.system_batch(b)
        vb = type("View", (), {})()
        for k in ("positions", "types", "charges", "atom_offsets", "cells", "invcells", "volumes", "alphas", "ks",
                  "kprefactor", "k_offsets", "constant_offset", "ncells", "cell_offsets", "cellgrid_offsets", "sigma",
                  "epsilon", "guest_types", "framework_of"):
            setattr(vb, k, getattr(sb, k))
        vb.Shost = st.Sk
        v, keep = orc.view(vb, b.guest_sites_orig, b.guest_charges_orig, b.cutoff, b.ewald_cutoff)
        kT = float(b.T(pa.KB * T))
        t0 = time.perf_counter()
        dln = []
        for s in range(2):
            sl = slice(s * ns, (s + 1) * ns)
            ref = orc.chain_energy(v, s, ins["poses"][sl, :3] @ sb.cells[s].T, ins["poses"][sl, 3:],
                                   st.live_sites(guest, s))
            ref += pa.insertion_constant_term(ff, b, guest, s, st.nguests(s))
            with np.errstate(over="ignore"):
                dln.append(abs(math.log(np.sum(np.exp(-ins["dU"][sl] / kT))) - math.log(np.sum(np.exp(-ref / kT)))))
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 2 * ns / dt, "unit": "insertions/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"{2 * ns} insertions of the workload (FP64 oracle chain energy, OpenMP)"}
        out["sample_max_dlnW"] = float(max(dln))
    b.drop_device()
    pa.chain.system_batch(b).drop_device()
    return out


def batched_workload(pa, backend, torch, stream, flush):
    """64 uneven frameworks, 2^20 insertions each, in one call (one persistent energy launch over
    all frameworks' bins), batch tables built with device structure factors and self terms,
    autotuned, replayed
    from a CUDA graph; FP32 against the plain FP64 form on 2^14 insertions per framework."""
    ctx = backend.ctx
    fws, ff, guest, ewald, prm = pa.synthetic.batched(T=np.float32)
    t0 = time.perf_counter()
    b = pa.FrameworkBatch(fws, ff, guest, ewald, device=ctx)
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    pa.FrameworkBatch(fws, ff, guest, ewald, sk=ctx.structure_factor, self_term=ctx.self_term)
    build_host_tables_s = time.perf_counter() - t0
    n, T, seed, nb = prm["ninsert"], prm["T"], prm["seed"], prm["nblocks"]
    tune = pa.autotune(b, guest, T=T, ninsert=n, backend=backend, seed=seed, nblocks=nb, bin_widths=(3.0, 3.5, 4.0),
                       ctas_per_sm=(8,), repeats=1)
    ctx.set_tuning(use_graphs=True)
    pa._widom(b, guest, reject=True, T=T, ninsert=n, seed=seed, nblocks=nb, backend=backend, segment_range=(0, 0))
    ms = []
    for _ in range(3):
        flush.zero_()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pa._widom(b, guest, reject=True, T=T, ninsert=n, seed=seed, nblocks=nb, backend=backend, segment_range=(0, 0))
        e.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(e))
    ms_call = float(np.median(ms))
    # accuracy against the plain FP64 form, per framework, from the raw block sums (the generator
    # can draw frameworks so dense that every insertion overlaps: W = 0 there, which widom's
    # reduction reports as an error, so those are counted instead)
    n64 = len(fws) * 2**14

    def raw(batch):
        lse, sw, suw, cnt = pa._widom(batch, guest, reject=True, T=T, ninsert=n64, seed=seed, nblocks=nb,
                                      backend=backend, segment_range=(0, 0))
        sW, sUW = pa.block_sums(lse, sw, suw)
        W = sW.reshape(len(fws), nb).sum(axis=1)
        UW = sUW.reshape(len(fws), nb).sum(axis=1)
        return W, UW

    b64 = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float64, sk=ctx.structure_factor, self_term=ctx.self_term)
    raw(b64)
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    W64, UW64 = raw(b64)
    e.record(stream)
    torch.cuda.synchronize()
    rate64 = n64 / (a.elapsed_time(e) / 1e3)
    W32, UW32 = raw(b)
    ok = (W64 > 0) & (W32 > 0)
    dln = np.abs(np.log(W32[ok]) - np.log(W64[ok]))
    dq = np.abs(UW32[ok] / W32[ok] - UW64[ok] / W64[ok])
    b.drop_device()
    b64.drop_device()
    return {"workload": "batched_64_frameworks", "frameworks": len(fws), "natoms": int(len(b.positions)),
            "coupled_k": int(b.k_offsets[-1]), "ninsert": n, "ms_per_call": ms_call, "value": n / (ms_call / 1e3),
            "unit": "insertions/s", "batch_build_s": build_s,
            "batch_build_note": "every table the device can build built there (FrameworkBatch(device=ctx)); "
                                "batch_build_host_tables_s: k-vectors, kmin and cell sort on the host instead",
            "batch_build_host_tables_s": build_host_tables_s, "tuning": {"bin_width": tune.bin_width,
                                                                         "ctas_per_sm": tune.ctas_per_sm,
                                                                         "cuda_graphs": True},
            "fp64_plain": {"value": rate64, "ninsert": n64, "ratio_fp32_over_fp64": n / (ms_call / 1e3) / rate64,
                           "max_dlnKH": float(np.max(dln)), "max_dqst_eV": float(np.max(dq)),
                           "frameworks_compared": int(ok.sum()),
                           "frameworks_without_accessible_volume": int(np.sum((W64 == 0) & (W32 == 0))),
                           "note": "the two forms draw the same uniforms at 24 and 53 bits, so the difference "
                                   "includes the pose rounding; the same-pose comparison against the FP64 oracle "
                                   "is tests/test_gpu_batched.py"}}


def ch4_workload(pa, backend, torch, stream, flush):
    """The plain FP64 LJ-only CH4 configuration (cubic P1, a = 25.832 A, 424 atoms of 4 types,
    united-atom CH4, 12.8 A cutoff, 10^5 insertions, seed 42, T = 298.15 K, 10 blocks), in both
    forms: mu_ex, K_H, q_st with their block standard errors, and insertions/s from CUDA events
    around one widom call (median of 5, batch resident)."""
    fws, ff, guest, ewald, prm = pa.synthetic.lj_ch4()
    out = {"workload": "lj_ch4_424_atoms_cubic", "ninsert": prm["ninsert"], "seed": prm["seed"], "T_K": prm["T"],
           "nblocks": prm["nblocks"]}
    for name, T in (("fp64_plain", np.float64), ("fp32", np.float32)):
        b = pa.FrameworkBatch(fws, ff, guest, ewald, T=T)
        call = lambda: pa.widom(b, guest, T=prm["T"], ninsert=prm["ninsert"], seed=prm["seed"], nblocks=prm["nblocks"],
                                backend=backend)
        for _ in range(3):
            r = call()[0]
        ms = []
        for _ in range(5):
            flush.zero_()
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r = call()[0]
            e.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(e))
        out[name] = {"mu_ex_eV": r.mu_ex, "mu_ex_err": r.mu_ex_err, "K_H": r.K_H, "K_H_err": r.K_H_err,
                     "q_st_eV": r.q_st, "q_st_err": r.q_st_err, "nsamples": r.nsamples,
                     "ms_per_call": float(np.median(ms)), "value": prm["ninsert"] / (float(np.median(ms)) / 1e3),
                     "unit": "insertions/s"}
        b.drop_device()
    out["dlnKH_fp32_vs_fp64"] = abs(math.log(out["fp32"]["K_H"]) - math.log(out["fp64_plain"]["K_H"]))
    out["dqst_eV_fp32_vs_fp64"] = abs(out["fp32"]["q_st_eV"] - out["fp64_plain"]["q_st_eV"])
    return out


def parity_fractions(pa, orc, backend, n=20_000):
    """Per workload, the fraction of survivors whose FP32 dU lies within max(1e-5 |dU|, 8.62e-8 eV)
    of the FP64 oracle at the same poses, with the default split and with every pair and the
    reciprocal term in FP32; and the worst error in units of that tolerance."""
    ctx = backend.ctx
    default = ctx.fp32_split()
    out = {}
    for name, gen, seed in (("co2_5832_atoms", pa.synthetic.co2, 42), ("lj_ch4_424_atoms", pa.synthetic.lj_ch4, 42)):
        fws, ff, guest, ewald = gen(T=np.float32)[:4]
        b = pa.FrameworkBatch(fws, ff, guest, ewald)
        kT = float(np.float32(pa.KB * 298.15))
        v, keep = orc.view(b, b.guest_sites_orig, b.guest_charges_orig, b.cutoff, b.ewald_cutoff)
        rho2, reach0 = pa.build_rejection_tables(b, kT)
        ref = orc.widom(v, 32, kT, n, seed, 10, pa.default_run(n, 1), True, rho2, reach0)
        surv = ref["flags"] == 0
        res = {"insertions": n, "survivors": int(surv.sum())}
        for mode, rn, r64 in (("default", default.near_radius, default.fp64_reciprocal), ("all_fp32", 0.0, 0)):
            ctx.set_fp32_split(near_radius=rn, fp64_reciprocal=r64)
            ins = {}
            pa._widom(b, guest, reject=True, T=298.15, ninsert=n, seed=seed, nblocks=10, backend=backend,
                      insertions=ins)
            a, r = ins["dU"][surv], ref["dU"][surv]
            tol = np.maximum(1e-5 * np.abs(r), 8.62e-8)
            res[mode] = {"near_radius": rn, "fp64_reciprocal": bool(r64),
                         "fraction_within": float(np.mean(np.abs(a - r) <= tol)),
                         "worst_over_tolerance": float(np.max(np.abs(a - r) / tol))}
        ctx.set_fp32_split(near_radius=default.near_radius, fp64_reciprocal=default.fp64_reciprocal)
        b.drop_device()
        out[name] = res
    return out


def fitting_workload(pa, backend):
    """Adam on the 8 palette scale factors of 128 frameworks, 2^18 insertions per framework per
    step (batched FP32 widom + adjoint), targets from the plain FP64 form at the hidden factors."""
    ctx = backend.ctx
    fws, ff, guest, ewald, prm = pa.synthetic.fitting(T=np.float32)
    n, T, seed = len(fws) * prm["ninsert_per_framework"], prm["T"], prm["seed"]
    t0 = time.perf_counter()
    ffh = pa.fit.scaled_forcefield(ff, prm["fitted_types"], prm["hidden"])
    targets = pa.fit.target_lnkh(fws, ffh, guest, ewald, T=T, ninsert=n, seed=seed, backend=backend,
                                 sk=ctx.structure_factor, self_term=ctx.self_term)
    target_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32, device=ctx, bounds=ctx.batch_bounds)
    build_s = time.perf_counter() - t0
    # each step's rejection radii from the device as well
    tables = backend.device_tables
    backend.device_tables = True
    try:
        res = pa.fit.fit_lj_scales(b, guest, ff, prm["fitted_types"], targets, T=T, ninsert=n, steps=prm["steps"],
                                   lr=prm["lr"], seed=seed, backend=backend)
    finally:
        backend.device_tables = tables
    # what the data determine: the loss's Gauss-Newton curvature at the start and at the end, the
    # parameter error along its eigenvectors, and each type's eps sigma^6 against the hidden one
    ones = np.ones(len(prm["hidden"]))
    ident = {}
    for name, xv in (("initial", ones), ("final", res.x)):
        idf = pa.fit.identifiability(b, guest, ff, prm["fitted_types"], xv, targets, T=T, ninsert=n, seed=seed,
                                     backend=backend, x_ref=prm["hidden"])
        ident[name] = {"hessian_eigenvalues": idf.eigenvalues.tolist(), "error_along_eigenvectors":
                       idf.error_along.tolist(), "loss_along_eigenvectors": idf.loss_along.tolist(),
                       "eps_sigma6_rel_error": idf.eps_sigma6_rel_error.tolist()}
    lam = np.asarray(ident["final"]["hessian_eigenvalues"])
    stiff = lam >= 1e-2 * lam[0]
    err_f = np.asarray(ident["final"]["error_along_eigenvectors"])
    err_i = np.asarray(ident["initial"]["error_along_eigenvectors"])
    return {"workload": "fitting_128_frameworks_palette4", "frameworks": len(fws), "natoms": int(len(b.positions)),
            "ninsert_per_step": n, "steps": prm["steps"], "lr": prm["lr"],
            "frameworks_fitted": int(np.sum(np.isfinite(targets))),
            "ms_per_step_median": float(np.median(res.ms)), "wall_s": float(np.sum(res.ms) / 1e3),
            "loss_first": res.loss[0], "loss_last": res.loss[-1],
            "max_scale_error_initial": float(np.max(np.abs(1 - prm["hidden"]))),
            "max_scale_error_final": float(np.max(np.abs(res.x - prm["hidden"]))),
            "scales_final": res.x.tolist(), "scales_hidden": prm["hidden"].tolist(),
            "identifiability": ident,
            "stiff_directions": int(stiff.sum()),
            "error_in_stiff_directions_initial": float(np.linalg.norm(err_i[stiff])),
            "error_in_stiff_directions_final": float(np.linalg.norm(err_f[stiff])),
            "error_in_soft_directions_final": float(np.linalg.norm(err_f[~stiff])),
            "max_eps_sigma6_rel_error_initial": float(np.max(ident["initial"]["eps_sigma6_rel_error"])),
            "max_eps_sigma6_rel_error_final": float(np.max(ident["final"]["eps_sigma6_rel_error"])),
            "identifiability_note": "stiff directions: Gauss-Newton eigenvalues >= 1e-2 of the largest at the fitted "
                                    "point; the error norms are of (x - hidden) projected on the eigenvectors",
            "targets_s": target_s, "batch_build_s": build_s}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    pa = ge.load_package()
    orc = ge.load_oracle()

    if args.impl == "reference":
        if rank != 0:
            return 0
        # the reference is Julia (no toolchain here): its CPU path is the oracle, the C++ FP64
        # restatement, with the oracle's own batch builder and rejection tables
        wl = OracleWorkload(pa, orc)
        rates = []
        for i in range(args.warmup + args.steps):
            r, n, cores = cpu_baseline_port(wl, args.ninsert, target_s=8.0)
            if i >= args.warmup:
                rates.append(r)
        if product_library_loaded():
            raise RuntimeError("the reference arm loaded the product library")
        v = float(np.median(rates))
        line = {"metric": METRIC, "value": v, "unit": "insertions/s",
                "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "dtype": "f64", "data": "synthetic",
                "config": bench_config(args.ninsert, max(1, args.gpus), wl.natoms, wl.coupled_k, wl.prm),
                "cpu_baseline": {"value": v, "unit": "insertions/s", "cores": cores, "kind": "port",
                                 "sample": f"{n} insertions of the workload per step (two-phase, FP64, rejection "
                                           "tables rebuilt per call, oracle batch builder; OpenMP)"},
                "e2e": {"value": v, "unit": "insertions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "product_library_loaded": False,
                "vs_baseline": None}
        print(json.dumps(line))
        return 0

    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    backend = pa.B200Backend(local)
    ctx = backend.ctx
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)

    batch, guest, prm = workload(pa, np.float32)
    ninsert = args.ninsert * world
    nblocks = prm["nblocks"]
    run = pa.default_run(ninsert, batch.nsys)
    nseg = pa._lib.ctypes.c_int64()
    pa._lib.lib().pa_segment_count(ninsert, batch.nsys, run, nblocks, pa._lib.ctypes.byref(nseg))
    nseg = nseg.value
    s0, s1 = nseg * rank // world, nseg * (rank + 1) // world
    segs = np.zeros(3 * nseg)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        return pa._widom(batch, guest, reject=True, T=prm["T"], ninsert=ninsert, seed=prm["seed"], nblocks=nblocks,
                         backend=backend, segment_range=(s0, s1), segments_out=segs)

    # layout and launch shape chosen by the autotuner on this rank's own call, then every step
    # replayed from a CUDA graph
    if args.no_tune:
        bw = args.bin_width if args.bin_width > 0 else 3.0
        ctx.set_tuning(bin_width=bw, ctas_per_sm=8)
        batch.drop_device()
        tune = pa.TuneReport(bw, 8, float("nan"), [])
    else:
        tune = pa.autotune(batch, guest, T=prm["T"], ninsert=args.ninsert, backend=backend, seed=prm["seed"],
                           nblocks=nblocks)
    ctx.set_tuning(use_graphs=True)
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms_steps = [a.elapsed_time(b) for a, b in ev]
    ms_total = float(sum(ms_steps))
    # per-kernel device times from a second pass of the same steps with kernel timing on (direct
    # launches: graphs are not used while timing)
    ctx.set_timing(True)
    for i in range(args.steps):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    kms, kn = ctx.kernel_times()
    ctx.set_timing(False)
    if world > 1:
        t = torch.tensor([ms_total], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_total = float(t.item())
        g = torch.from_numpy(segs).cuda()
        torch.distributed.all_reduce(g)  # disjoint segment ranges: each entry comes from one rank
        segs[:] = g.cpu().numpy()
    ms_per_step = ms_total / args.steps
    value = ninsert / (ms_per_step / 1e3)

    line = None
    if rank == 0:
        # block sums of the whole job from the gathered segments, and the reduced result
        lse, sw, suw = np.zeros(nblocks), np.zeros(nblocks), np.zeros(nblocks)
        cnt = np.zeros(nblocks, dtype=np.int64)
        sums = pa._lib.BlockSums(*(pa._lib.ptr(a) for a in (lse, sw, suw, cnt)), None)
        pa._lib.lib().pa_combine_segments(ninsert, batch.nsys, run, nblocks, pa._lib.ptr(segs), sums)
        kT32 = float(np.float32(pa.KB * prm["T"]))
        sW, sUW = pa.block_sums(lse, sw, suw)
        res32 = pa._reduce(sW, sUW, cnt, kT32, float(np.float32(batch.volumes[0])), 1)

        # roofline of the energy kernel: executed FP32 work per launch (the model below)
        ins = {}
        sample_n = 20_000
        pa._widom(batch, guest, reject=True, T=prm["T"], ninsert=sample_n, seed=prm["seed"], nblocks=nblocks,
                  backend=backend, insertions=ins)
        surv_frac = float(np.mean(ins["flags"] == 0))
        rn = ctx.fp32_split().near_radius
        n_lj, n_ew, n_near = count_pairs(batch, ins["poses"][ins["flags"] == 0][:512], rn)
        dev = batch.device(ctx)
        list_entries, nbins = dev.info()
        L = list_entries / nbins
        N = len(batch.guest_types)
        nk = int(batch.k_offsets[1])
        kc = batch.kcoeffs
        rows = 1 + int(np.sum(~((kc[1:, 0] == kc[:-1, 0]) & (kc[1:, 1] == kc[:-1, 1])))) if nk else 0
        # executed work of k_energy32 per survivor (FMA = 2 flops): each of its N (insertion,
        # site) items walks its bin's list, 8 FP32 flops per entry for the distance; a pair in
        # the cutoff takes, in FP32, 29 flops in the exp-free form (reciprocal 1, LJ 5, screened
        # Coulomb 23) or 48 in the rational one (LJ 10, screened Coulomb 38), plus one FP64 add
        # into the item's sum, or, closer than the near radius, 55 FP64 flops (distance 8,
        # reciprocal square root 6, LJ 7, screened Coulomb 33, sum 1). The bound is the FP32
        # flops at the FP32 FMA peak plus the FP64 flops at the FP64 peak; `achieved` is the
        # FP32-equivalent rate (FP64 flops weighted by the peak ratio), so frac = that bound's
        # time / the measured time. The reciprocal term (10 per (k, site) + 7 per k, 25 per
        # (row start, site)) runs in its own kernel.
        exp_free, fit_err = ctx.fp32_form()
        flops32 = 8 * N * L + (29 if exp_free else 48) * (n_lj - n_near)
        flops64 = 55 * n_near + (n_lj - n_near)
        peak = fp32_peak(torch)
        flops_surv = flops32 + flops64 * (peak / FP64_PEAK_NOMINAL)
        flops_recip = (10 * N + 7) * nk + 25 * N * rows
        e_ms = kms[2] / max(1, kn[2])
        surv_per_launch = surv_frac * (s1 - s0) * (ninsert / nseg)
        achieved = flops_surv * surv_per_launch / (e_ms / 1e3) / 1e12
        ref_alg = (30 * 5832 + 8 * N * 5832 + 11 * n_lj + 36 * n_ew + 15 * N * nk + 4 * nk)
        # the issue-slot roofline: the kernel's warp instructions (ncu, this workload and bin width)
        # per second against one per cycle per SM sub-partition at the SM clock sampled while timing
        ncu_workload = args.ninsert == 1_000_000 and world == 1 and rn == 6.0
        n_inst = ENERGY32_INSTRUCTIONS.get(float(tune.bin_width)) if ncu_workload else None
        sm_mhz = clk.summary().get("sm_mhz") or 1965.0
        issue = None
        if n_inst is not None:
            ach = n_inst / (e_ms / 1e3) / 1e9
            pk = ISSUE_PER_CYCLE * sm_mhz * 1e6 / 1e9
            issue = {"instructions": n_inst, "achieved": ach, "peak": pk, "unit": "Ginst/s", "frac": ach / pk,
                     "note": "warp instructions per launch from ncu (smsp__inst_executed.sum) on this workload and "
                             "bin width; peak one warp instruction per cycle per SM sub-partition at the sampled "
                             "SM clock"}
        roof = {"bound": "fp32+fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": ENERGY32_TRAFFIC_BYTES.get(float(tune.bin_width)) if ncu_workload else None,
                "issue": issue,
                "kernel": "k_energy32", "kernel_ms_per_launch": e_ms,
                "peak_note": "nominal FP32 FMA peak at the maximum SM clock (148 SMs x 128 lanes x 2 x 1.965 GHz); "
                             "FP64 flops weighted by FP32/FP64 nominal peaks (74.4 / 37.2 TFLOP/s)",
                "fp32_flops_per_survivor": flops32, "fp64_flops_per_survivor": flops64,
                "flops_per_survivor_fp32_equivalent": flops_surv, "reciprocal_flops_per_survivor": flops_recip,
                "reciprocal_combine_ms_per_step": kms[6] / args.steps, "reference_algorithm_flops_per_survivor": ref_alg,
                "survivor_fraction": surv_frac, "list_entries_per_bin": L, "pairs_lj": n_lj, "pairs_ewald": n_ew,
                "pairs_fp64": n_near, "fp32_coulomb_form": "exp-free" if exp_free else "rational",
                "fp32_coulomb_fit_error": fit_err}

        # plain FP64 form on the same workload and stream (the >= 3x denominator)
        fp64 = None
        if not args.no_fp64:
            b64 = pa.FrameworkBatch(*pa.synthetic.co2(T=np.float64)[:4])
            n64 = args.ninsert
            for _ in range(2):
                pa.widom(b64, guest, T=prm["T"], ninsert=n64, seed=prm["seed"], nblocks=nblocks, backend=backend)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r64 = pa.widom(b64, guest, T=prm["T"], ninsert=n64, seed=prm["seed"], nblocks=nblocks, backend=backend)
            b.record(stream)
            torch.cuda.synchronize()
            rate64 = n64 / (a.elapsed_time(b) / 1e3)
            # accuracy of the FP32 form against the FP64 form on the same stream and count
            r32 = pa.widom(batch, guest, T=prm["T"], ninsert=n64, seed=prm["seed"], nblocks=nblocks, backend=backend)
            fp64 = {"value": rate64, "unit": "insertions/s", "ninsert": n64, "ratio_fp32_over_fp64": value / world / rate64,
                    "dlnKH": abs(math.log(r32[0].K_H) - math.log(r64[0].K_H)),
                    "dqst_eV": abs(r32[0].q_st - r64[0].q_st),
                    "note": "k_energy64 as it is: the plain FP64 reference algorithm, one thread per survivor over "
                            "every atom (min image per atom), with about 7 of 32 lanes active (divergent cutoff "
                            "branches); the ratio is against that kernel"}

        # end to end through the public API from host arrays (batch re-uploaded each step)
        e2e_ms = []
        h2d = sum(a.nbytes for a in batch.desc()[1].values()) + 8 * (len(batch.guest_types) * len(batch.sigma) + 3)
        d2h = 3 * 8 * nseg + 4 * 8 * nblocks
        for i in range(args.warmup + max(3, args.steps // 2)):
            # every step re-uploads the batch and rebuilds its descriptor and rejection tables
            batch.drop_device()
            batch.drop_host_caches()
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            pa.widom(batch, guest, T=prm["T"], ninsert=args.ninsert, seed=prm["seed"], nblocks=nblocks, backend=backend)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                e2e_ms.append(dt * 1e3)
        e2e_value = args.ninsert / (float(np.mean(e2e_ms)) / 1e3)

        # the adjoint workload: widom plus d ln K_H / dθ (14 LJ parameters, 5,832 charges) over
        # 4,000,000 insertions of the same framework
        adj = None
        if not args.no_adjoint and world == 1:
            nadj = 4_000_000
            ff = pa.synthetic.co2(T=np.float32)[1]
            for _ in range(2):
                pa.widom_grad(batch, guest, ff, T=prm["T"], ninsert=nadj, seed=prm["seed"], nblocks=nblocks,
                              backend=backend)
            torch.cuda.synchronize()
            ctx.set_timing(True)
            k0, n0 = ctx.kernel_times()
            ms_adj = []
            for _ in range(3):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                _, gr = pa.widom_grad(batch, guest, ff, T=prm["T"], ninsert=nadj, seed=prm["seed"], nblocks=nblocks,
                                      backend=backend)
                b.record(stream)
                torch.cuda.synchronize()
                ms_adj.append(a.elapsed_time(b))
            k1, n1 = ctx.kernel_times()
            ctx.set_timing(False)
            ms_call = float(np.median(ms_adj))
            adj = {"ninsert": nadj, "ms_per_call": ms_call, "value": nadj / (ms_call / 1e3), "unit": "insertions/s",
                   "adjoint_kernel_ms_per_call": float((k1[5] - k0[5]) / 3), "recomputed": int(gr[0].recomputed),
                   "parameters": int(2 * len(ff.names) + len(gr[0].charges)),
                   "note": "widom_grad: forward pass + adjoint pass + host chain rule, CUDA events around the call"}

        # the same steps with every pair and the reciprocal term in FP32 (the cost of the default
        # split's FP64 near pairs and reciprocal term)
        fast = None
        if world == 1 and not args.no_all_fp32:
            split = ctx.fp32_split()
            ctx.set_fp32_split(near_radius=0.0, fp64_reciprocal=False)
            step()
            step()
            torch.cuda.synchronize()
            fms = []
            for i in range(args.steps):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                step()
                b.record(stream)
                torch.cuda.synchronize()
                fms.append(a.elapsed_time(b))
            ctx.set_fp32_split(near_radius=split.near_radius, fp64_reciprocal=split.fp64_reciprocal)
            fast = {"near_radius": 0.0, "fp64_reciprocal": False, "ms_per_step": float(np.mean(fms)),
                    "value": ninsert / (float(np.mean(fms)) / 1e3), "unit": "insertions/s",
                    "note": "every pair and the reciprocal term in FP32: meets the aggregate bounds, not the "
                            "per-insertion one (see parity)"}
        parity = None if world > 1 or args.no_parity else parity_fractions(pa, orc, backend)
        ch4 = None if world > 1 or args.no_ch4 else ch4_workload(pa, backend, torch, stream, flush)
        batched = None if args.no_batched or world > 1 else batched_workload(pa, backend, torch, stream, flush)
        chain = None if args.no_chain or world > 1 else chain_workload(pa, orc, backend, torch, stream, flush,
                                                                       no_cpu=args.no_cpu)
        fitting = None if args.no_fit or world > 1 else fitting_workload(pa, backend)

        cpu = None
        if not args.no_cpu:
            r, n, cores = cpu_baseline_port(OracleWorkload(pa, orc), args.ninsert)
            cpu = {"value": r, "unit": "insertions/s", "cores": cores, "kind": "port",
                   "sample": f"{n} insertions of the workload (FP64 oracle, two-phase, rejection tables rebuilt "
                             "per call, OpenMP)"}

        line = {"metric": METRIC,
                "value": value, "unit": "insertions/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": bench_config(args.ninsert, world, int(len(batch.positions)), nk, prm),
                "result": {"mu_ex": res32.mu_ex, "mu_ex_err": res32.mu_ex_err, "K_H": res32.K_H,
                           "K_H_err": res32.K_H_err, "q_st": res32.q_st, "q_st_err": res32.q_st_err,
                           "note": "this synthetic framework is so dense that a handful of insertions carry "
                                   "nearly all the weight (K_H_err / K_H large); the batched and CH4 sections "
                                   "are the meaningful aggregate comparisons"},
                "fp32_split": {"near_radius": ctx.fp32_split().near_radius,
                               "fp64_reciprocal": bool(ctx.fp32_split().fp64_reciprocal)},
                "all_fp32": fast,
                "parity": parity,
                "ch4_config": ch4,
                "clocks": clk.summary(),
                "tuning": {"bin_width": tune.bin_width, "ctas_per_sm": tune.ctas_per_sm, "cuda_graphs": True,
                           "candidates": [list(r) for r in tune.table]},
                "gpu_launches": int(10 * args.steps),
                "kernel_ms": {"pose_phase0": kms[0] / args.steps, "scan_scatter": kms[1] / args.steps,
                              "energy": kms[2] / args.steps, "reciprocal_combine": kms[6] / args.steps,
                              "segment_reduce": kms[3] / args.steps},
                "roofline": roof,
                "fp64_plain": fp64,
                "adjoint": adj,
                "batched": batched,
                "chain": chain,
                "fitting": fitting,
                "e2e": {"value": e2e_value, "unit": "insertions/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h), "ms_per_step": float(np.mean(e2e_ms))},
                "cpu_baseline": cpu}
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
