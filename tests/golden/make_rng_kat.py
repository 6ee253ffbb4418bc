"""Writes rng_kat.json: known-answer vectors of the counter-based stream, from a pure-Python
restatement of splitmix64 (PureAdsorb.jl src/state.jl:225-230) and ChainRNG / next_bits /
unit_from_bits / mulhi64 (src/rng.jl:14-81), independent of the C++ oracle and the library.
Each case also carries the FP32 Shoemake quaternion of its draws 3..5 (src/rng.jl:126-129):
a = sqrt(1 - u1), b = sqrt(u1) and the four products, each rounded to FP32, with sinpi/cospi(2u)
correctly rounded to FP32 by mpmath (what Julia's Float32 sinpi/cospi return).

The reference's own tests hold no fixed draws (test/rng_tests.jl is statistical), so these
vectors are pinned by two independent restatements (this one and oracle.cpp) agreeing bit for
bit, and the library is checked against them.

Run: python tests/golden/make_rng_kat.py
"""
import json
import os
import struct

import mpmath as mp
import numpy as np

M = (1 << 64) - 1


def splitmix64(seed, index):
    z = (seed + index * 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def chain_key(chain_seed, cycle, move):
    return splitmix64(splitmix64(chain_seed, cycle), move)


def next_bits(key, draw):
    return splitmix64(key, draw)


def unit_f64(raw):
    return (raw >> 11) * 2.0**-53


def unit_f32_bits(raw):
    # (raw >> 40) * 2^-24 is exact in FP32; return the float32 bit pattern
    return struct.unpack("<I", struct.pack("<f", (raw >> 40) * 2.0**-24))[0]


def f32_nearest(v):
    """The FP32 value nearest to the mpmath number v (ties to even), zero as +0."""
    f = np.float32(float(v))
    cands = [np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))]
    best = min(range(3), key=lambda i: (abs(v - mp.mpf(float(cands[i]))), int(cands[i].view(np.uint32)) & 1))
    return cands[best] + np.float32(0)


def quat_f32_bits(raws):
    u1, u2, u3 = (np.float32((r >> 40) * 2.0**-24) for r in raws[3:6])
    a, b = np.sqrt(np.float32(1) - u1), np.sqrt(u1)
    c2, s2 = f32_nearest(mp.cospi(2 * mp.mpf(float(u2)))), f32_nearest(mp.sinpi(2 * mp.mpf(float(u2))))
    c3, s3 = f32_nearest(mp.cospi(2 * mp.mpf(float(u3)))), f32_nearest(mp.sinpi(2 * mp.mpf(float(u3))))
    q = [a * c2, b * s3, b * c3, a * s2]
    return [int(np.float32(x).view(np.uint32)) for x in q]


def mulhi64(a, b):
    return (a * b) >> 64


def main():
    mp.mp.dps = 50
    cases = []
    for seed in (0, 1, 42, 7, 0xDEADBEEF, M):
        for s in (0, 1, 2, 64):
            for k in (1, 2, 1000, 2**31 + 5):
                key = chain_key(splitmix64(seed, s), k, 0)
                raws = [next_bits(key, d) for d in range(6)]
                cases.append({"seed": str(seed), "s": s, "k": k, "raw": [str(r) for r in raws],
                              "u64": [unit_f64(r).hex() for r in raws], "u32_bits": [unit_f32_bits(r) for r in raws],
                              "quat_f32_bits": quat_f32_bits(raws)})
    mul = [{"a": str(a), "b": str(b), "hi": str(mulhi64(a, b))}
           for a, b in ((0, 0), (M, M), (1, M), (M, 1), (0x9E3779B97F4A7C15, 0xBF58476D1CE4E5B9),
                        (123456789123456789, 987654321987654321))]
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rng_kat.json"), "w") as fh:
        json.dump({"pose_stream": cases, "mulhi64": mul}, fh, indent=0)


if __name__ == "__main__":
    main()
