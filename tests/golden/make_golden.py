"""Generates tests/golden/known_answers.json: known-answer vectors for the SPPM primitives.

The reference (alfazet/phosphor) ships no golden vectors and cannot be executed here, so these
values are derived from the reference's formulas by a second, independent restatement in plain
Python (exact integer arithmetic for the PCG stream and the grid key, numpy float32 for the
codecs, IEEE binary32 division for the cell coordinate).  The C++ oracle and the CUDA kernels are
both checked against this file.

    python tests/golden/make_golden.py
"""
import json
import math
from pathlib import Path

import numpy as np

M32 = 0xFFFFFFFF
f32 = np.float32


def pcg_seed(seed):  # include/common/random.h:16-24
    s = (0 * 747796405 + 2891336453) & M32
    s = (s + seed) & M32
    return (s * 747796405 + 2891336453) & M32


def random_u32(state):  # random.h:29-34
    old = state
    state = (state * 747796405 + 2891336453) & M32
    word = (((old >> ((old >> 28) + 4)) ^ old) * 277803737) & M32
    return word, state


def random_float(word):  # random.h:36: (f32)u32 / 4294967296.0f
    return float(f32(word) / f32(4294967296.0))


def encode_rgbe(p):  # include/device/encoding.h:10-29
    p = [f32(x) for x in p]
    m = max(p[0], max(p[1], p[2]))
    if m <= 0:
        return 0
    _, e = math.frexp(float(m))
    scale = f32(math.ldexp(1.0, e))
    r, g, b = (min(int(f32(f32(x / scale) * f32(256.0))), 255) for x in p)
    E = (e + 128) & M32
    return (r | (g << 8) | (b << 16) | (E << 24)) & M32


def decode_rgbe(w):  # encoding.h:31-39
    E = w >> 24
    if E == 0:
        return [0.0, 0.0, 0.0, 0.0]
    s = f32(math.ldexp(1.0, E - 136))
    return [float(f32(w & 0xFF) * s), float(f32((w >> 8) & 0xFF) * s), float(f32((w >> 16) & 0xFF) * s), 0.0]


def encode_oct(d):  # encoding.h:47-59 for an already unit-length direction
    x, y, z = (f32(c) for c in d[:3])
    n2 = f32(f32(f32(x * x) + f32(y * y)) + f32(z * z))
    ln = f32(np.sqrt(n2))
    x, y, z = f32(x / ln), f32(y / ln), f32(z / ln)
    l1 = f32(f32(abs(x) + abs(y)) + abs(z))
    nx, ny = f32(x / l1), f32(y / l1)
    if not z >= 0:
        sx = f32(1) if nx >= 0 else f32(-1)
        sy = f32(1) if ny >= 0 else f32(-1)
        nx, ny = f32(f32(1) - abs(ny)) * sx, f32(f32(1) - abs(nx)) * sy
    cl = lambda v: min(max(f32(f32(v * f32(0.5)) + f32(0.5)), f32(0)), f32(1))
    ux = int(f32(cl(nx) * f32(65535.0)))
    uy = int(f32(cl(ny) * f32(65535.0)))
    return ux | (uy << 16)


def get_hash(pos, origin, cell, g):  # include/common/photon_hash.h:21-37
    fs = [f32(f32(f32(p) - f32(o)) / f32(c)) for p, o, c in zip(pos, origin, cell)]
    if any(f < 0 for f in fs) or any(f >= f32(g) for f in fs):
        return 0
    x, y, z = (int(f) for f in fs)
    return (g * g * x + g * y + z + 1) & M32


def main():
    out = {"_about": "known answers derived from the reference formulas by tests/golden/make_golden.py"}
    pcg = {}
    for seed in [0, 1, 2, 42, 2137, 0xFFFFFFFF, 123456789]:
        st = pcg_seed(seed)
        words, floats = [], []
        for _ in range(8):
            w, st = random_u32(st)
            words.append(w)
            floats.append(random_float(w))
        pcg[str(seed)] = {"u32": words, "float": floats}
    out["pcg"] = pcg
    # a word that makes random_float round to exactly 1.0f (the reference's quirk)
    out["random_float_top"] = {"word": 0xFFFFFFFF, "float": random_float(0xFFFFFFFF)}
    powers = [[1.0, 0.5, 0.25], [2.9452431, 2.9452431, 2.9452431], [0.0, 0.0, 0.0], [1e-3, 2e-3, 5e-4],
              [7.5, 0.1, 0.0], [255.0, 128.0, 1.0], [0.999, 0.999, 0.999], [1e-30, 1e-31, 0.0]]
    out["rgbe"] = [{"power": p, "word": encode_rgbe(p), "decoded": decode_rgbe(encode_rgbe(p))} for p in powers]
    dirs = [[0, 0, 1], [0, 0, -1], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0],
            [0.57735026, 0.57735026, 0.57735026], [-0.57735026, 0.57735026, -0.57735026],
            [0.6, -0.8, 0.0], [0.0, 0.6, -0.8]]
    out["oct"] = [{"dir": d, "word": encode_oct(d)} for d in dirs]
    origin, cell, g = [-0.001, -0.001, -0.001], [0.02004, 0.02004, 0.02004], 50
    pts = [[0.5, 0.5, 0.5], [-0.001, -0.001, -0.001], [-0.0011, 0.5, 0.5], [1.0, 1.0, 1.0], [1.001, 0.5, 0.5],
           [0.01903, 0.5, 0.5], [0.019039998, 0.5, 0.5], [0.2, 0.999, 0.0], [0.0, 0.0, 0.0]]
    out["hash"] = {"origin": origin, "cell": cell, "grid_res": g,
                   "cases": [{"pos": p, "key": get_hash(p, origin, cell, g)} for p in pts]}
    path = Path(__file__).with_name("known_answers.json")
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
