"""One image over several GPUs: pixel-range camera passes, photon-path-range photon passes and one
photon all-gather per round (include/phx.h, phosphor_b200/csrc/engine_shard.cu).

CPU: two gloo ranks each emit their path range with the oracle and all-gather the photons; the
rank-order concatenation must be the oracle's single-process canonical photon list, bit for bit.
GPU (one device): three ranks emulated by three contexts on the same GPU, photons exchanged through
the host; every rank's pixels must equal a single-context render bit for bit.  No rank waits on
another inside a kernel, so running them one after another on one GPU is safe.  The NCCL transport
is run with one rank.
"""
import os
import socket

import numpy as np
import pytest

import oracle as O
import phosphor_b200 as P
from phosphor_b200 import _capi as A
from phosphor_b200.renderer import nccl_unique_id


def ranges(n: int, world: int):
    return [(n * r // world, n * (r + 1) // world) for r in range(world)]


def test_shard_ranges_partition():
    for n, w in [(1024 * 1024, 8), (4097, 3), (5, 5)]:
        rs = ranges(n, w)
        assert rs[0][0] == 0 and rs[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))


def _gloo_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        scene = P.SceneData.generate(A.PHX_SCENE_CAUSTIC, seed=2, width=32, height=32, detail=16)
        orc = O.Oracle(scene)
        e, seed = 1 << 12, 4242
        lo, hi = ranges(e, world)[rank]
        counts, pos, power, dirs = orc.emit(lo, hi, 8, seed, threads=2)
        parts = [None] * world
        dist.all_gather_object(parts, (counts, pos, power, dirs))
        cat = [np.concatenate([p[i] for p in parts]) for i in range(4)]
        full = orc.emit(0, e, 8, seed, threads=2)
        ok = all(np.array_equal(a, b) for a, b in zip(cat, full)) and len(full[1]) > 0
        out.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_photon_exchange_is_the_canonical_order_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: True, 1: True}


def _make():
    scene = P.SceneData.generate(A.PHX_SCENE_CAUSTIC, seed=2, width=48, height=40, detail=16)
    args = P.ArgsList(width=48, height=40, photons_per_round=1 << 13, max_photon_bounces=12, grid_res=50, seed=2,
                      direct_samples=8)
    return scene, args


@pytest.mark.gpu
def test_sharded_ranks_match_single_gpu_bit_for_bit():
    scene, args = _make()
    world, rounds = 3, 3
    single = P.Renderer(args)
    single.set_scene(scene)
    ranks = [P.Renderer(args) for _ in range(world)]
    for r, rr in enumerate(ranks):
        rr.set_scene(scene)
        rr.shard(r, world)
    with pytest.raises(A.PhxError) as e:
        ranks[0].round()
    assert e.value.code == A.PHX_E_STATE
    for _ in range(rounds):
        single.round()
        n = [rr.shard_begin() for rr in ranks]
        got = [rr.shard_get_photons(k) for rr, k in zip(ranks, n)]
        pos = np.concatenate([g[0] for g in got])
        pd = np.concatenate([g[1] for g in got])
        # the rank-order concatenation is the single GPU's canonical photon list
        assert np.array_equal(pos.view(np.uint32), single.read("PHOTON_POS").view(np.uint32))
        assert np.array_equal(pd[:, 0], single.read("PHOTON_POWER"))
        assert np.array_equal(pd[:, 1], single.read("PHOTON_DIR"))
        for rr in ranks:
            rr.shard_put_photons(pos, pd)
            rr.shard_end()
    npx = args.width * args.height
    for r, rr in enumerate(ranks):
        lo, hi = ranges(npx, world)[r]
        for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]:
            a = rr.read(buf).view(np.uint32)
            b = single.read(buf).view(np.uint32)
            assert np.array_equal(a[lo:hi], b[lo:hi]), (r, buf)
            assert not a[:lo].any() and not a[hi:].any(), (r, buf)
        assert rr.info().rounds_done == rounds
    for rr in ranks + [single]:
        rr.close()


@pytest.mark.gpu
def test_nccl_transport_one_rank():
    scene, args = _make()
    with P.Renderer(args) as a, P.Renderer(args) as b:
        a.set_scene(scene)
        b.set_scene(scene)
        a.shard(0, 1)
        a.shard_nccl(nccl_unique_id())
        for _ in range(3):
            a.shard_round()
            b.round()
        for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]:
            assert np.array_equal(a.read(buf).view(np.uint32), b.read(buf).view(np.uint32)), buf
