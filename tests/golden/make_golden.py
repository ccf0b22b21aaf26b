"""Generates tests/golden/rng_streams.json: RNG streams of common.wgsl:39-44
(seed(i, salt) at a frame index, then `random` draws) computed with exact
Python integer arithmetic and numpy float32 for the final u32 -> f32 step.

The salts are the reference's: 7 (VPL), 11/13 (candidates), 17/19
(temporal), 23/29 (spatial) — lighting.wgsl:53-99, vpl.wgsl:4.

    python tests/golden/make_golden.py
"""
import json
import os

import numpy as np


def stream(i, salt, frame, n):
    m = 0xFFFFFFFF
    s = (i * 1973 + frame * 9277 + salt * 26699 + 89173) & m
    states, bits = [], []
    for _ in range(n):
        s = (s * 747796405 + 2891336453) & m
        w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & m
        v = np.float32((w >> 22) ^ w) * np.float32(1.0 / 4294967296.0)
        states.append(s)
        bits.append(int(np.float32(v).view(np.uint32)))
    return states, bits


def main():
    cases = []
    for salt in (7, 11, 13, 17, 19, 23, 29):
        for i, frame in ((0, 0), (1, 0), (40959, 15), (2303999, 63), (123456, 7), (0xFFFFFFFF, 1)):
            st, bits = stream(i, salt, frame, 24)
            cases.append({"i": i, "salt": salt, "frame": frame, "states": st, "value_bits": bits})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rng_streams.json")
    with open(out, "w") as fh:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, fh)
    print(out, len(cases))


if __name__ == "__main__":
    main()
