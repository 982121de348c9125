"""The oracle against the known-answer vectors of tests/golden/known_answers.json (CPU only).

These pin the restatement of random.h, encoding.h and photon_hash.h:get_hash: the reference has
no golden vectors of its own, so the answers come from the independent restatement in
tests/golden/make_golden.py.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLD = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())


@pytest.mark.parametrize("seed", list(GOLD["pcg"].keys()))
def test_pcg_stream(seed):
    words, floats = O.pcg(int(seed), 8)
    assert words.tolist() == GOLD["pcg"][seed]["u32"]
    assert floats.tolist() == pytest.approx(GOLD["pcg"][seed]["float"], abs=0, rel=0)


def test_random_float_can_be_one():
    # (f32)0xFFFFFFFF rounds to 2^32, so random_float returns exactly 1.0f (random.h:36)
    assert GOLD["random_float_top"]["float"] == 1.0


def test_rgbe_known_answers():
    p = np.array([c["power"] + [0.0] for c in GOLD["rgbe"]], np.float32)
    words = O.encode_rgbe(p)
    assert words.tolist() == [c["word"] for c in GOLD["rgbe"]]
    dec = O.decode_rgbe(words)
    assert np.array_equal(dec, np.array([c["decoded"] for c in GOLD["rgbe"]], np.float32))


def test_oct_known_answers():
    d = np.array([c["dir"] + [0.0] for c in GOLD["oct"]], np.float32)
    assert O.encode_oct(d).tolist() == [c["word"] for c in GOLD["oct"]]


def test_oct_roundtrip_error_bound():
    rng = np.random.default_rng(3)
    v = rng.normal(size=(4096, 3)).astype(np.float32)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    d4 = np.concatenate([v, np.zeros((len(v), 1), np.float32)], axis=1)
    back = O.decode_oct(O.encode_oct(d4))[:, :3]
    ang = np.arccos(np.clip((back * v).sum(1), -1, 1))
    assert ang.max() < 1e-3  # 16-bit octahedral: well under a milliradian


def test_rgbe_relative_error_bound():
    rng = np.random.default_rng(5)
    p = rng.uniform(1e-4, 50.0, size=(4096, 3)).astype(np.float32)
    p4 = np.concatenate([p, np.zeros((len(p), 1), np.float32)], axis=1)
    back = O.decode_rgbe(O.encode_rgbe(p4))[:, :3]
    m = p.max(1, keepdims=True)
    assert np.all(np.abs(back - p) <= m / 128.0 + 1e-12)  # 8-bit shared-exponent mantissa, truncating


def test_get_hash_boundaries():
    h = GOLD["hash"]
    hd = np.zeros(12, np.float32)
    hd[0:3] = h["origin"]
    hd[4:7] = h["cell"]
    raw = bytearray(hd.tobytes())
    raw[32:36] = int(h["grid_res"]).to_bytes(4, "little")
    p = np.array([c["pos"] + [0.0] for c in h["cases"]], np.float32)
    assert O.get_hash(p, bytes(raw)).tolist() == [c["key"] for c in h["cases"]]
