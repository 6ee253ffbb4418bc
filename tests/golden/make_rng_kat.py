"""Writes rng_kat.json: known-answer vectors of the counter-based stream, from a pure-Python
restatement of splitmix64 (PureAdsorb.jl src/state.jl:225-230) and ChainRNG / next_bits /
unit_from_bits / mulhi64 (src/rng.jl:14-81), independent of the C++ oracle and the library.

The reference's own tests hold no fixed draws (test/rng_tests.jl is statistical), so these
vectors are pinned by two independent restatements (this one and oracle.cpp) agreeing bit for
bit, and the library is checked against them.

Run: python tests/golden/make_rng_kat.py
"""
import json
import os
import struct

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


def mulhi64(a, b):
    return (a * b) >> 64


def main():
    cases = []
    for seed in (0, 1, 42, 7, 0xDEADBEEF, M):
        for s in (0, 1, 2, 64):
            for k in (1, 2, 1000, 2**31 + 5):
                key = chain_key(splitmix64(seed, s), k, 0)
                raws = [next_bits(key, d) for d in range(6)]
                cases.append({"seed": str(seed), "s": s, "k": k, "raw": [str(r) for r in raws],
                              "u64": [unit_f64(r).hex() for r in raws], "u32_bits": [unit_f32_bits(r) for r in raws]})
    mul = [{"a": str(a), "b": str(b), "hi": str(mulhi64(a, b))}
           for a, b in ((0, 0), (M, M), (1, M), (M, 1), (0x9E3779B97F4A7C15, 0xBF58476D1CE4E5B9),
                        (123456789123456789, 987654321987654321))]
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rng_kat.json"), "w") as fh:
        json.dump({"pose_stream": cases, "mulhi64": mul}, fh, indent=0)


if __name__ == "__main__":
    main()
