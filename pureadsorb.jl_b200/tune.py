"""Autotuner of the FP32 path's layout and launch shape (no counterpart in the reference).

Two choices set the cost of a widom call on a given batch and insertion count:
- the spatial bin width: wider bins mean longer neighbour lists (each insertion of a bin walks
  the whole list) but fuller 32-insertion tiles; narrower bins the opposite;
- the persistent CTAs per SM of the energy kernel (occupancy against per-warp shared memory).
The optimum depends on the framework sizes, the insertion density and the survivor fraction, so
`autotune` times the candidates on the device with the call the user will make and leaves the
fastest set on the backend's context.
"""
from dataclasses import dataclass, field

import numpy as np

from .widom import _widom, default_backend

BIN_WIDTHS = (2.5, 3.0, 3.5, 4.0, 5.0)
CTAS_PER_SM = (4, 6, 8)


@dataclass
class TuneReport:
    bin_width: float
    ctas_per_sm: int
    ms: float                               # device milliseconds per call of the chosen shape
    table: list = field(default_factory=list)  # (bin_width, ctas_per_sm, ms) of every candidate


def _device_ms(ctx, call, repeats):
    times = []
    for _ in range(repeats):
        ctx.set_timing(True)
        call()
        ms, n = ctx.kernel_times()
        ctx.set_timing(False)
        times.append(float(np.sum(ms[:4]) + ms[6] + ms[7]))
    return float(np.median(times))


def autotune(batch, guest, *, T, ninsert, backend=None, seed=0, nblocks=10, run=None, bin_widths=BIN_WIDTHS,
             ctas_per_sm=CTAS_PER_SM, repeats=2):
    """Times widom(batch, guest; T, ninsert, seed, nblocks, run) on the device for every
    (bin width, CTAs per SM) candidate (device time of the pose, scan, energy, reciprocal and
    reduction kernels, median of `repeats` calls after one warm-up) and sets the fastest on the
    backend's context, preferring the widest bin among those within 2 % of the fastest (its
    neighbour lists are the shortest to build and hold); the batch is re-uploaded with the chosen
    bin width. Returns a TuneReport."""
    backend = backend or default_backend()
    ctx = backend.ctx
    old = ctx.tuning()
    table = []

    def call():
        # the raw block sums: a framework without accessible volume (every weight zero) does not
        # stop the timing the way widom's reduction would
        _widom(batch, guest, reject=True, T=T, ninsert=ninsert, backend=backend, seed=seed, nblocks=nblocks, run=run,
               segment_range=(0, 0))

    try:
        for w in bin_widths:
            ctx.set_tuning(bin_width=w)
            batch.drop_device()
            call()  # upload and warm-up
            for c in ctas_per_sm:
                ctx.set_tuning(ctas_per_sm=c)
                table.append((float(w), int(c), _device_ms(ctx, call, repeats)))
    except Exception:
        ctx.set_tuning(bin_width=old.bin_width, ctas_per_sm=old.ctas_per_sm)
        batch.drop_device()
        raise
    best = min(r[2] for r in table)
    w, c, ms = max((r for r in table if r[2] <= 1.02 * best), key=lambda r: (r[0], -r[2]))
    ctx.set_tuning(bin_width=w, ctas_per_sm=c)
    batch.drop_device()
    batch.device(ctx)
    return TuneReport(w, c, ms, table)
