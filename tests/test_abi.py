"""The C-ABI library loads and exports every entry point include/pureadsorb_b200.h declares; the
host-callable parts behave without a GPU (CPU only)."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pureadsorb_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:pa_status|const char\*)\s+(pa_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol(pa):
    names = declared()
    assert len(names) >= 15
    L = pa._lib.lib()
    for n in names:
        assert hasattr(L, n), n
    assert sorted(n for n, _, _ in pa._lib.SIGNATURES) == names
    assert L.pa_version().startswith(b"pureadsorb-b200")


def test_host_pose_stream_matches_oracle(pa, orc):
    for prec in (32, 64):
        r, q = orc.poses(prec, 0xDEADBEEF, 5, 1, 300)
        for k in (1, 7, 300):
            rr, qq = pa._lib.pose_host(prec, 0xDEADBEEF, 5, k)
            assert np.array_equal(rr, r[k - 1]) and np.array_equal(qq, q[k - 1])


def test_host_pose_stream_matches_golden_quaternions(pa):
    # the library's FP32 quaternions equal the independent Python/mpmath restatement bit for bit
    import json
    import os

    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rng_kat.json")) as fh:
        kat = json.load(fh)
    for c in kat["pose_stream"]:
        _, qq = pa._lib.pose_host(32, int(c["seed"]), c["s"], c["k"])
        assert qq.astype(np.float32).view(np.uint32).tolist() == c["quat_f32_bits"]


def test_segment_count_and_combine_host(pa):
    L = pa._lib.lib()
    n = pa._lib.ctypes.c_int64()
    assert L.pa_segment_count(1_000_000, 1, 256, 10, pa._lib.ctypes.byref(n)) == 0
    assert n.value == 10 * 49  # 100,000-insertion blocks in 2,048-insertion segments
    assert L.pa_segment_count(5, 1, 1, 10, pa._lib.ctypes.byref(n)) == pa._lib.PA_ERR_ARG
    # combining triplets: 40,960 insertions in 10 blocks is two segments per block; the first
    # block gets two segments with different maxima, every other segment has zero weight
    lse, sw, suw = np.zeros(10), np.zeros(10), np.zeros(10)
    cnt = np.zeros(10, np.int64)
    sums = pa._lib.BlockSums(*(pa._lib.ptr(a) for a in (lse, sw, suw, cnt)), None)
    nseg = pa._lib.ctypes.c_int64()
    L.pa_segment_count(40960, 1, 1, 10, pa._lib.ctypes.byref(nseg))
    assert nseg.value == 20
    segs = np.zeros(3 * nseg.value)
    segs[6::3] = -np.inf
    segs[0:6] = [0.0, 2.0, 4.0, 3.0, 1.0, -1.0]
    assert L.pa_combine_segments(40960, 1, 1, 10, pa._lib.ptr(segs), sums) == 0
    W, UW = pa.block_sums(lse, sw, suw)
    assert W[0] == pytest.approx(2.0 + np.exp(3.0))
    assert UW[0] == pytest.approx(4.0 - np.exp(3.0))
    assert cnt[0] == 4096 and np.all(W[1:] == 0)


def test_no_device_errors_are_status_codes(pa):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(pa._lib.PAError):
        pa._lib.Context(0)
    assert pa._lib.lib().pa_widom(None, None, None, None, None) == pa._lib.PA_ERR_ARG
    assert pa._lib.lib().pa_pose_host(16, 1, 1, 1, None, None) == pa._lib.PA_ERR_ARG
