"""Parity at the bench's own sizes (needs a GPU; the oracle takes seconds per round on the host).

bench.py times CUDA-graph replays of its workloads with the library's default tuning, two rounds in
flight per replay.  Here one such replay of the exact workload — the caustic Cornell box (149,862
triangles, 1024x1024, 2^20 photons, depth 12, grid 50, 16 samples) and the full atrium (262,898
triangles, 1920x1080, 2^22 photons, depth 16, grid 64) — is compared with the oracle, which the
reference build pins (tests/test_ref_pin.py): the SPPM state after the two rounds, and the second
round's hit points, per-path photon counts, canonical photons, cell keys, counts, starts and the
scatter permutation, all bit for bit.  These sizes reach what the small scenes cannot: slot
arrays of 12.6M and 67M entries, sort tiles sized by the stored count, two sets of round buffers.
"""
import numpy as np
import pytest

import bench
import oracle as O
import phosphor_b200 as P

pytestmark = pytest.mark.gpu

HP = ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT", "HP_EMISSION"]


def round_seeds(seed: int, n: int) -> list[int]:
    """The round seeds of Renderer::run (renderer.cpp:49,65): PCG stream of pcg_seed(seed)."""
    s = (2891336453 + seed) & 0xFFFFFFFF
    s = (s * 747796405 + 2891336453) & 0xFFFFFFFF
    out = []
    for _ in range(n):
        old = s
        s = (s * 747796405 + 2891336453) & 0xFFFFFFFF
        out.append((((old >> ((old >> 28) + 4)) ^ old) * 277803737) & 0xFFFFFFFF)
    return out


def same(name, got, want):
    got, want = np.ascontiguousarray(got), np.ascontiguousarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    eq = got.view(np.uint8).reshape(len(got), -1) == want.view(np.uint8).reshape(len(want), -1)
    bad = np.flatnonzero(~eq.all(axis=1))
    assert len(bad) == 0, f"{name}: {len(bad)} of {len(got)} rows differ, first {bad[:8]}"


@pytest.mark.parametrize("config", ["caustic", "atrium"])
def test_bench_workload_replay_equals_the_oracle(config):
    cfg = bench.CONFIGS[config]
    args = bench.make_args(cfg)
    scene = P.SceneData.generate(cfg["kind"], seed=1, width=args.width, height=args.height, detail=cfg["detail"])
    with P.Renderer(args) as r:
        r.set_scene(scene)
        assert r.tuning().pipeline_rounds == 2  # the bench's form
        r.iterate(2)
        got = {b: r.read(b) for b in ["FLUX", "PHOTON_WEIGHT", "RADIANCE", "EMIT_COUNT", "PHOTON_POS",
                                      "PHOTON_POWER", "PHOTON_DIR", "PHOTON_HASH", "CELL_COUNT", "CELL_START",
                                      "SORT_PERM"]}
        hp = np.stack([r.read(b) for b in HP], axis=1)
        inf = r.info()
    assert inf.stack_overflows == 0 and inf.error_flags == 0 and inf.rounds_done == 2
    o = O.Oracle(scene)
    st = o.render(args.params(), 2, prec=0)
    same("flux", got["FLUX"], st["flux"])
    same("photon weight", got["PHOTON_WEIGHT"], st["weight"])
    same("radiance", got["RADIANCE"], st["radiance"])
    seed2 = round_seeds(args.seed, 2)[1]
    same("hit points (second SPPM round)", hp, o.trace(args.width, args.height, seed2, args.direct_samples))
    counts, pos, power, dirs = o.emit(0, args.photons_per_round, args.max_photon_bounces, seed2)
    assert inf.n_photons == len(pos) == st["n_last"]
    same("per-path photon counts", got["EMIT_COUNT"], counts)
    same("photon positions", got["PHOTON_POS"][:len(pos)], pos)
    same("photon power", got["PHOTON_POWER"][:len(pos)], power)
    same("photon directions", got["PHOTON_DIR"][:len(pos)], dirs)
    keys, cell_counts = O.hash_photons(pos, bytes(inf.hash), inf.bucket_count)
    same("cell keys", got["PHOTON_HASH"][:len(pos)], keys)
    same("cell counts", got["CELL_COUNT"], cell_counts)
    starts = O.scan(cell_counts)
    same("cell starts", got["CELL_START"], starts)
    _, _, _, _, perm = O.scatter(pos, power, dirs, keys, starts)
    same("scatter permutation", got["SORT_PERM"][:len(pos)], perm)
    assert (st["weight"] > 0).mean() > 0.3
