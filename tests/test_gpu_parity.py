"""Parity of the sm_100a kernels with the oracle, stage by stage and end to end (needs a GPU).

Every comparison runs the CUDA path through the C ABI (libphx.so) and the CPU restatement of the
reference (oracle/) on the same scene, seeds and inputs.  Integer results (cell keys, per-cell
counts, cell starts, the scatter permutation, photon codes) must be bit-exact; float results are
compared for exact equality first and must in any case agree within REL_TOL = 1e-4 relative.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import phosphor_b200 as P
from phosphor_b200 import _capi as A

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4  # float tolerance of the parity contract (hit points, photons, flux)

SCENES = {
    # name: (kind, detail, width, height, photons, max_bounces, grid_res)
    "cornell": (A.PHX_SCENE_CORNELL, 0, 64, 64, 1 << 14, 8, 50),
    "caustic": (A.PHX_SCENE_CAUSTIC, 0, 48, 40, 1 << 13, 12, 50),
    "atrium": (A.PHX_SCENE_ATRIUM, 16, 48, 27, 1 << 13, 16, 64),
}


def make(name, seed=1, **over):
    kind, detail, w, h, ph, mb, g = SCENES[name]
    scene = P.SceneData.generate(kind, seed=seed, width=w, height=h, detail=detail)
    args = P.ArgsList(width=w, height=h, photons_per_round=ph, max_photon_bounces=mb, grid_res=g, seed=seed,
                      direct_samples=16)
    for k, v in over.items():
        setattr(args, k, v)
    return scene, args


def assert_close(name, got, want, rel=REL_TOL):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    assert got.shape == want.shape, name
    exact = np.mean(got == want)
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-30)
    bad = (err > rel) & (np.abs(got - want) > 1e-30)
    assert not bad.any(), f"{name}: {bad.sum()} of {bad.size} values beyond {rel} (exact fraction {exact:.6f})"
    return exact


@pytest.mark.parametrize("name", list(SCENES))
def test_trace_rays_parity(name):
    scene, args = make(name)
    o = O.Oracle(scene)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        seed = 0x9E3779B9
        r.trace_rays(seed)
        got = np.stack([r.read(b) for b in ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT",
                                             "HP_EMISSION"]], axis=1)
        assert r.info().stack_overflows == 0
    want = o.trace(args.width, args.height, seed, args.direct_samples)
    exact = assert_close(f"{name} hit points", got, want)
    assert exact == 1.0, f"{name}: hit points not bit-exact ({exact})"
    assert (want[:, 5, 3] == 1.0).mean() > 0.3  # many pixels found a diffuse hit point


@pytest.mark.parametrize("name", list(SCENES))
def test_emit_photons_parity(name):
    scene, args = make(name)
    o = O.Oracle(scene)
    seed = 12345
    with P.Renderer(args) as r:
        r.set_scene(scene)
        n = r.emit_photons(seed)
        counts = r.read("EMIT_COUNT")
        pos, power, dirs = r.read("PHOTON_POS"), r.read("PHOTON_POWER"), r.read("PHOTON_DIR")
    ocounts, opos, opower, odir = o.emit(0, args.photons_per_round, args.max_photon_bounces, seed)
    assert n == len(opos) > 0
    assert np.array_equal(counts, ocounts)
    assert np.array_equal(power, opower)
    assert np.array_equal(dirs, odir)
    exact = assert_close(f"{name} photon positions", pos, opos)
    assert exact == 1.0


def inject_photons(r, pos, power, dirs):
    r.write("PHOTON_POS", np.ascontiguousarray(pos, np.float32))
    r.write("PHOTON_POWER", np.ascontiguousarray(power, np.uint32))
    r.write("PHOTON_DIR", np.ascontiguousarray(dirs, np.uint32))
    r.set_n_photons(len(pos))


@pytest.mark.parametrize("name", ["cornell", "caustic"])
def test_hash_scan_scatter_bit_exact(name):
    scene, args = make(name)
    o = O.Oracle(scene)
    _, pos, power, dirs = o.emit(0, args.photons_per_round, args.max_photon_bounces, 777)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        inject_photons(r, pos, power, dirs)
        r.hash_and_sort_photons()
        info = r.info()
        got = {b: r.read(b) for b in ["PHOTON_HASH", "CELL_COUNT", "CELL_START", "CELL_END", "SORTED_POS",
                                      "SORTED_POWER", "SORTED_DIR", "SORT_PERM"]}
    hd = bytes(info.hash)
    keys, counts = O.hash_photons(pos, hd, info.bucket_count)
    start = O.scan(counts)
    spos, spow, sdir, end, perm = O.scatter(pos, power, dirs, keys, start)
    assert np.array_equal(got["PHOTON_HASH"], keys)
    assert np.array_equal(got["CELL_COUNT"], counts)
    assert np.array_equal(got["CELL_START"], start)
    assert np.array_equal(got["CELL_END"], end)
    assert np.array_equal(got["SORT_PERM"], perm)
    assert np.array_equal(got["SORTED_POS"].view(np.uint32), spos.view(np.uint32))
    assert np.array_equal(got["SORTED_POWER"], spow)
    assert np.array_equal(got["SORTED_DIR"], sdir)
    # property: the permutation is the stable argsort of the keys
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))


@pytest.mark.parametrize("dist", ["uniform", "one_cell", "outside", "clustered"])
def test_sort_large_adversarial(dist):
    """3M photons on the largest grid (255^3 + 1 cells, 3 radix passes) against numpy."""
    scene, args = make("cornell", grid_res=255, photons_per_round=1 << 20, max_photon_bounces=4)
    rng = np.random.default_rng(11)
    n = 3_000_000
    if dist == "uniform":
        p = rng.uniform(-0.001, 1.001, size=(n, 3))
    elif dist == "one_cell":
        p = np.full((n, 3), 0.5)
    elif dist == "outside":
        p = rng.uniform(-0.001, 1.001, size=(n, 3))
        p[::3, 1] = 5.0  # a third of the photons outside the grid -> key 0
    else:
        p = 0.5 + 0.003 * rng.standard_normal(size=(n, 3))
    pos = np.concatenate([p, np.zeros((n, 1))], axis=1).astype(np.float32)
    power = rng.integers(0, 2**32, size=n, dtype=np.uint32)
    dirs = np.arange(n, dtype=np.uint32)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        inject_photons(r, pos, power, dirs)
        r.hash_and_sort_photons()
        info = r.info()
        keys_g = r.read("PHOTON_HASH")
        counts_g = r.read("CELL_COUNT")
        start_g = r.read("CELL_START")
        perm_g = r.read("SORT_PERM")
        sdir_g = r.read("SORTED_DIR")
    keys = O.get_hash(pos, bytes(info.hash))
    assert np.array_equal(keys_g, keys)
    counts = np.bincount(keys, minlength=info.bucket_count).astype(np.uint32)
    assert np.array_equal(counts_g, counts)
    start = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    assert np.array_equal(start_g, start)
    perm = np.argsort(keys, kind="stable").astype(np.uint32)
    assert np.array_equal(perm_g, perm)
    assert np.array_equal(sdir_g, dirs[perm])


@pytest.mark.parametrize("name", ["cornell", "caustic"])
def test_gather_parity(name):
    """gather_flux on identical inputs: hit points and sorted photons from the oracle, with a
    non-trivial SPPM state (radius already shrunk for some pixels)."""
    scene, args = make(name)
    o = O.Oracle(scene)
    hp = o.trace(args.width, args.height, 99, args.direct_samples)
    _, pos, power, dirs = o.emit(0, args.photons_per_round, args.max_photon_bounces, 99)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        inject_photons(r, pos, power, dirs)
        r.hash_and_sort_photons()
        info = r.info()
        rng = np.random.default_rng(4)
        npx = args.width * args.height
        flux = np.zeros((npx, 4), np.float32)
        r2 = (info.hash.cell_sizes.x * 0.5) ** 2 * 3
        flux[:, 3] = np.where(rng.uniform(size=npx) < 0.5, 0.0, r2 * rng.uniform(0.2, 1.0, size=npx))
        flux[:, :3] = rng.uniform(0, 1, size=(npx, 3))
        weight = rng.uniform(0, 5, size=npx).astype(np.float32)
        radiance = rng.uniform(0, 2, size=(npx, 4)).astype(np.float32)
        names = ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT", "HP_EMISSION"]
        for k, b in enumerate(names):
            r.write(b, hp[:, k, :])
        r.write("FLUX", flux)
        r.write("PHOTON_WEIGHT", weight)
        r.write("RADIANCE", radiance)
        r.gather_flux(0.7)
        gf, gw, gr = r.read("FLUX"), r.read("PHOTON_WEIGHT"), r.read("RADIANCE")
        hd = bytes(info.hash)
    keys, counts = O.hash_photons(pos, hd, info.bucket_count)
    start = O.scan(counts)
    spos, spow, sdir, end, _ = O.scatter(pos, power, dirs, keys, start)
    of, ow, orad = flux.copy(), weight.copy(), radiance.copy()
    O.gather(hp.reshape(npx, 24), spos, spow, sdir, start, end, hd, 0.7, of, ow, orad)
    assert (ow != weight).mean() > 0.2  # photons were found for many pixels
    for nm, g, w in (("flux", gf, of), ("weight", gw, ow), ("radiance", gr, orad)):
        exact = assert_close(nm, g, w)
        assert exact == 1.0, f"{nm} not bit-exact: {exact}"


@pytest.mark.parametrize("name", list(SCENES))
def test_rounds_end_to_end(name):
    """Three full SPPM rounds (plain per-pass form) against the oracle's Renderer::run."""
    scene, args = make(name)
    rounds = 3
    o = O.Oracle(scene)
    st = o.render(args.params(), rounds, prec=0)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        for _ in range(rounds):
            r.round()
        gf, gw, gr = r.read("FLUX"), r.read("PHOTON_WEIGHT"), r.read("RADIANCE")
        inf = r.info()
        img = r.image()
    assert inf.total_photons_emitted == st["total"]
    assert inf.n_photons == st["n_last"]
    for nm, g, w in (("flux", gf, st["flux"]), ("weight", gw, st["weight"]), ("radiance", gr, st["radiance"])):
        exact = assert_close(f"{name} {nm}", g, w)
        assert exact == 1.0, f"{name} {nm} not bit-exact: {exact}"
    oimg = O.image(st["flux"], st["radiance"], 0, args.exposure, False, st["total"], rounds)
    assert np.allclose(img.reshape(-1, 3), oimg, atol=1e-6)


@pytest.mark.parametrize("name", list(SCENES))
def test_kernel_forms_agree(name):
    """One-thread-per-item or lane-refill state-machine kernels, with the diffuse-hit NEE inline or
    deferred to the shadow wavefront: all four forms give identical bits."""
    scene, args = make(name)
    outs = []
    for persistent in (0, 1):
        for wavefront in (0, 1):
            with P.Renderer(args) as r:
                r.set_scene(scene)
                t = r.tuning()
                t.persistent, t.nee_wavefront = persistent, wavefront
                r.set_tuning(t)
                r.iterate(2)
                outs.append({b: r.read(b).view(np.uint32).copy() for b in
                             ["HP_POS", "HP_DIRECT", "HP_EMISSION", "HP_THROUGHPUT", "EMIT_COUNT", "PHOTON_POS",
                              "PHOTON_POWER", "FLUX", "RADIANCE"]})
    for o in outs[1:]:
        for b in o:
            assert np.array_equal(o[b], outs[0][b]), b


@pytest.mark.parametrize("sorted_pixels", [1, 0])
@pytest.mark.parametrize("name", list(SCENES))
def test_cooperative_gather_equals_the_per_thread_gather(name, sorted_pixels):
    """The warp-cooperative gather (records staged in shared memory per cell group) and the
    one-thread-per-pixel gather give identical bits, with the pixels grouped by cell or in plain
    order (where most warps need several cells per neighbour offset)."""
    scene, args = make(name)
    outs = []
    for coop in (0, 1):
        with P.Renderer(args) as r:
            r.set_scene(scene)
            t = r.tuning()
            t.gather_coop, t.gather_sorted = coop, sorted_pixels
            r.set_tuning(t)
            r.iterate(3)
            outs.append({b: r.read(b).view(np.uint32).copy() for b in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]})
    for b in outs[0]:
        assert np.array_equal(outs[0][b], outs[1][b]), b
    assert (outs[0]["PHOTON_WEIGHT"].view(np.float32) > 0).mean() > 0.1


def test_cooperative_gather_in_a_batch():
    """Lanes of one warp may belong to different scenes of a batch: cells are grouped by their
    global index, so the cooperative gather equals the per-thread one there too."""
    made = [make(n, photons_per_round=1 << 12) for n in ("cornell", "caustic", "atrium")]
    outs = []
    for coop in (0, 1):
        batch = P.Batch([s for s, _ in made], [a for _, a in made])
        t = batch.tuning()
        t.gather_coop = coop
        batch.set_tuning(t)
        batch.iterate(2, graph=True)
        outs.append([batch.read(i, "FLUX").view(np.uint32).copy() for i in range(3)])
        batch.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", list(SCENES))
def test_traversal_tree_does_not_change_results(name):
    """Traversing the reference median-split tree or binned-SAH trees with 1, 4 or 8 triangles per
    leaf, as 4-wide nodes or as child pairs, gives identical bits: closest hit, ties broken by the
    reference leaf rank."""
    scene, args = make(name)
    variants = [dict(flags=A.PHX_F_REFERENCE_BVH), dict(bvh_leaf_size=1), dict(bvh_leaf_size=4),
                dict(bvh_leaf_size=8), dict(flags=A.PHX_F_BINARY_BVH),
                dict(flags=A.PHX_F_BINARY_BVH, bvh_leaf_size=1)]
    outs = []
    for v in variants:
        a2 = make(name, **v)[1]
        with P.Renderer(a2) as r:
            r.set_scene(scene)
            r.iterate(2)
            inf = r.info()
            assert inf.stack_overflows == 0
            outs.append({b: r.read(b).view(np.uint32).copy() for b in ["HP_POS", "HP_NORMAL", "HP_DIRECT",
                                                                      "HP_EMISSION", "PHOTON_POS", "PHOTON_DIR",
                                                                      "FLUX", "RADIANCE"]})
    for o in outs[1:]:
        for b in o:
            assert np.array_equal(o[b], outs[0][b]), b


def test_graph_replay_equals_plain_rounds():
    scene, args = make("caustic")
    with P.Renderer(args) as a, P.Renderer(args) as b:
        a.set_scene(scene)
        b.set_scene(scene)
        for _ in range(4):
            a.round()
        b.iterate(2)
        b.iterate(2)
        for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE", "SORTED_POS", "CELL_START"]:
            assert np.array_equal(a.read(buf).view(np.uint32), b.read(buf).view(np.uint32)), buf
        assert a.info().total_photons_emitted == b.info().total_photons_emitted


def test_batch_equals_single_scenes():
    specs = [("cornell", dict(photons_per_round=1 << 13, sppm_alpha=0.62, seed=3)),
             ("caustic", dict(photons_per_round=1 << 12, sppm_alpha=0.75, seed=4)),
             ("atrium", dict(photons_per_round=1 << 12, sppm_alpha=0.7, seed=5))]
    made = [make(n, **kw) for n, kw in specs]
    rounds = 3
    batch = P.Batch([s for s, _ in made], [a for _, a in made])
    batch.iterate(rounds, graph=True)
    for i, (scene, args) in enumerate(made):
        with P.Renderer(args) as r:
            r.set_scene(scene)
            for _ in range(rounds):
                r.round()
            for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]:
                assert np.array_equal(batch.read(i, buf).view(np.uint32), r.read(buf).view(np.uint32)), (i, buf)
            assert np.array_equal(batch.read(i, "SORT_PERM"), r.read("SORT_PERM"))
    batch.close()


def test_batch_retired_scene_stops_and_others_continue():
    """A retired scene keeps its state and round count; the others go on exactly as alone."""
    specs = [("cornell", dict(photons_per_round=1 << 13, seed=3)),
             ("caustic", dict(photons_per_round=1 << 12, seed=4)),
             ("atrium", dict(photons_per_round=1 << 12, seed=5))]
    made = [make(n, **kw) for n, kw in specs]
    batch = P.Batch([s for s, _ in made], [a for _, a in made])
    batch.iterate(2, graph=True)
    batch.set_active(1, False)
    batch.iterate(3, graph=True)
    assert [batch.info(i).rounds_done for i in range(3)] == [5, 2, 5]
    for i, (scene, args) in enumerate(made):
        with P.Renderer(args) as r:
            r.set_scene(scene)
            r.iterate(2 if i == 1 else 5)
            for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]:
                assert np.array_equal(batch.read(i, buf).view(np.uint32), r.read(buf).view(np.uint32)), (i, buf)
    batch.set_active(1, True)
    batch.iterate(1, graph=True)
    assert batch.info(1).rounds_done == 3
    for i in range(3):
        batch.set_active(i, False)
    batch.iterate(2, graph=True)  # nothing active: no work, no error
    assert [batch.info(i).rounds_done for i in range(3)] == [6, 3, 6]
    batch.close()


def test_batch_with_scenes_sharing_warps():
    """Odd pixel counts at 16 samples per pixel: a scene's pixels and sample slots end inside a
    warp, so warps of every per-pixel and per-sample kernel straddle two scenes, and each scene
    alone ends with a partial warp; the batch still equals every scene alone."""
    made = []
    for kind, w, h, seed, detail in [(A.PHX_SCENE_CAUSTIC, 13, 11, 4, 0), (A.PHX_SCENE_CORNELL, 9, 7, 3, 0),
                                     (A.PHX_SCENE_ATRIUM, 15, 9, 5, 16), (A.PHX_SCENE_CAUSTIC, 7, 5, 6, 0)]:
        scene = P.SceneData.generate(kind, seed=seed, width=w, height=h, detail=detail)
        args = P.ArgsList(width=w, height=h, photons_per_round=1 << 12, max_photon_bounces=8, grid_res=16,
                          seed=seed, direct_samples=16)
        made.append((scene, args))
    batch = P.Batch([s for s, _ in made], [a for _, a in made])
    batch.iterate(3, graph=True)
    for i, (scene, args) in enumerate(made):
        with P.Renderer(args) as r:
            r.set_scene(scene)
            r.iterate(3)
            for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE", "HP_DIRECT", "HP_EMISSION"]:
                assert np.array_equal(batch.read(i, buf).view(np.uint32), r.read(buf).view(np.uint32)), (i, buf)
            assert r.info().stack_overflows == 0
    batch.close()


def test_material_change_recaptures_for_the_new_shadow_kind():
    """A scene whose every material blocks shadow rays replays graphs with the any-hit shadow
    kernel; making its water transmissive again (set_materials) must bring back the listing
    traversal for the next replays.  Graph replays before and after the change equal plain rounds
    (launched afresh each time) of a second context taken through the same changes, and both
    differ from the rounds the opaque water alone would give."""
    scene, args = make("caustic")
    view = scene.materials()
    glass = view.copy()
    water = int(np.argmax(glass["transmission"]))
    assert glass["transmission"][water] > 0.5
    opaque = glass.copy()
    opaque["transmission"][water] = 0.0
    bufs = ["FLUX", "PHOTON_WEIGHT", "RADIANCE", "HP_DIRECT", "HP_EMISSION"]
    view[:] = opaque
    try:
        a, b, c = P.Renderer(args), P.Renderer(args), P.Renderer(args)
        for r in (a, b, c):
            r.set_scene(scene)  # the scene's arrays are copied here
    finally:
        view[:] = glass
    try:
        a.iterate(2)
        for _ in range(2):
            b.round()
        c.iterate(5)
        a.set_materials(glass)
        b.set_materials(glass)
        a.iterate(3)
        for _ in range(3):
            b.round()
        for buf in bufs:
            assert np.array_equal(a.read(buf).view(np.uint32), b.read(buf).view(np.uint32)), buf
        assert any(not np.array_equal(a.read(buf).view(np.uint32), c.read(buf).view(np.uint32)) for buf in bufs)
        assert a.info().stack_overflows == 0
    finally:
        for r in (a, b, c):
            r.close()


PIPE_BUFS = ["FLUX", "PHOTON_WEIGHT", "RADIANCE", "HP_POS", "HP_DIRECT", "HP_EMISSION", "PHOTON_POS",
             "SORTED_POS", "SORT_PERM", "CELL_START"]


@pytest.mark.parametrize("name", ["caustic", "atrium"])
def test_pipelined_rounds_are_bit_identical(name):
    """Graph replays that capture k rounds at a time, with each round's passes on branches of their
    own and the gathers in order, give the bits of rounds replayed one by one: the SPPM state and
    the last round's hit points, photons and grid (k = 2, 3, 4; 7 rounds, which no k divides)."""
    scene, args = make(name)

    def run(k):
        with P.Renderer(args) as r:
            r.set_scene(scene)
            t = r.tuning()
            t.pipeline_rounds = k
            r.set_tuning(t)
            r.iterate(3)
            r.iterate(4)
            inf = r.info()
            return {b: r.read(b).view(np.uint32).copy() for b in PIPE_BUFS}, inf.rounds_done, inf.n_photons

    base = run(1)
    for k in (2, 3, 4):
        got = run(k)
        assert got[1:] == base[1:], k
        for b in PIPE_BUFS:
            assert np.array_equal(got[0][b], base[0][b]), (k, b)


def test_pipelined_batch_with_a_retired_scene():
    """The pipelined form on a batch, before and after a scene is retired, equals the scenes alone."""
    specs = [("cornell", dict(photons_per_round=1 << 13, seed=3)),
             ("caustic", dict(photons_per_round=1 << 12, seed=4)),
             ("atrium", dict(photons_per_round=1 << 12, seed=5))]
    made = [make(n, **kw) for n, kw in specs]
    batch = P.Batch([s for s, _ in made], [a for _, a in made])
    t = batch.tuning()
    t.pipeline_rounds, t.concurrent_passes = 2, 1
    batch.set_tuning(t)
    batch.iterate(4, graph=True)
    batch.set_active(1, False)
    batch.iterate(3, graph=True)
    assert [batch.info(i).rounds_done for i in range(3)] == [7, 4, 7]
    for i, (scene, args) in enumerate(made):
        with P.Renderer(args) as r:
            r.set_scene(scene)
            r.iterate(4 if i == 1 else 7)
            for buf in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]:
                assert np.array_equal(batch.read(i, buf).view(np.uint32), r.read(buf).view(np.uint32)), (i, buf)
    batch.close()


def test_autotune_keeps_state_and_results():
    """The autotuner renders trial rounds but restores state, seeds and counters, and the tuning it
    picks gives the same bits as the default one."""
    scene, args = make("caustic")
    with P.Renderer(args) as a, P.Renderer(args) as b:
        a.set_scene(scene)
        b.set_scene(scene)
        a.iterate(2)
        b.iterate(2)
        before = {k: a.read(k).view(np.uint32).copy() for k in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]}
        t = a.autotune(2)
        assert t.persistent in (0, 1) and t.nee_wavefront in (0, 1)
        assert a.info().rounds_done == 2 and a.info().total_photons_emitted == b.info().total_photons_emitted
        for k, v in before.items():
            assert np.array_equal(a.read(k).view(np.uint32), v), k
        a.iterate(3)
        b.iterate(3)
        for k in ["FLUX", "PHOTON_WEIGHT", "RADIANCE"]:
            assert np.array_equal(a.read(k).view(np.uint32), b.read(k).view(np.uint32)), k


def test_image_formation_matches_output_cpp():
    scene, args = make("cornell")
    with P.Renderer(args) as r:
        r.set_scene(scene)
        r.iterate(2)
        f, rad = r.read("FLUX"), r.read("RADIANCE")
        inf = r.info()
        for tm in (False, True):
            img = r.image(tonemap=tm)
            want = O.image(f, rad, 0, args.exposure, tm, inf.total_photons_emitted, inf.rounds_done)
            assert np.allclose(img.reshape(-1, 3), want, atol=1e-6)
        u8 = r.image_u8()
        assert u8.dtype == np.uint8 and u8.shape == (args.height, args.width, 3)


def _scene_from_arrays(tris, mats, lights, camera):
    """A scene over caller arrays; the emissive triangle list is the triangle array itself.  The
    light luminance prefix sum comes from the library's host helper and the UV transforms are zero
    (no material is textured), as the oracle reads both."""
    sc = A.Scene()
    sc.triangles = tris.ctypes.data_as(C.POINTER(A.Triangle))
    sc.n_triangles = len(tris)
    sc.materials = mats.ctypes.data_as(C.POINTER(A.Material))
    sc.n_materials = len(mats)
    uv = (A.UvTransformBlock * len(mats))()
    sc.uv_transforms = C.cast(uv, C.POINTER(A.UvTransformBlock))
    sc.emissive_triangles = tris.ctypes.data_as(C.POINTER(A.Triangle))
    sc.n_emissive_triangles = len(tris)
    sc.lights = lights.ctypes.data_as(C.POINTER(A.Light))
    sc.n_lights = len(lights)
    lum = np.zeros(max(len(lights), 1), np.float32)
    A.check(A.load().phx_lum_pref_sum(lights.ctypes.data_as(C.POINTER(A.Light)), len(lights),
                                      lum.ctypes.data_as(C.POINTER(C.c_float))))
    sc.lum_pref_sum = lum.ctypes.data_as(C.POINTER(C.c_float))
    sc.camera = camera
    return P.SceneData(sc, keep=(tris, mats, lights, uv, lum))


def test_no_photon_hit_is_a_status():
    """An emitter that faces away from all geometry stores nothing: the reference traps
    (renderer.cpp:117-118); here emit_photons returns PHX_E_NO_PHOTONS."""
    base = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=16, height=16)
    t = base.triangles()[:2].copy()  # the floor quad, y = 0, normal +y
    lt = t.copy()
    for k in ("v0", "v1", "v2"):
        lt[k]["y"] = -1.0  # light quad below the floor, facing down
    for k in ("n0", "n1", "n2"):
        lt[k]["y"] = -1.0
    tris = np.concatenate([t, lt])
    tris["mat_index"][:] = 0
    mats = base.materials()[:1].copy()
    lights = np.zeros(1, dtype=base.lights().dtype)
    lights[0] = base.lights()[0]
    aux = lights[0]["aux"]
    aux_u = np.array([0xFFFFFFFF, 2, 2], np.uint32).view(np.float32)
    aux["x"], aux["y"], aux["z"] = aux_u
    scene = _scene_from_arrays(tris, mats, lights, base.scene.camera)
    args = P.ArgsList(width=16, height=16, photons_per_round=4096, max_photon_bounces=4, grid_res=8)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        with pytest.raises(P.PhxError) as e:
            r.emit_photons(5)
        assert e.value.code == A.PHX_E_NO_PHOTONS


def _glass_panes_scene():
    """The Cornell box with three horizontal transmissive panes between the floor and the ceiling
    light: shadow rays from the floor cross three surfaces."""
    base = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=32, height=32)
    box = base.triangles().copy()
    panes = np.zeros(6, dtype=box.dtype)
    for q, y in enumerate((0.25, 0.5, 0.75)):
        corners = [(0.1, 0.1), (0.9, 0.1), (0.9, 0.9), (0.1, 0.9)]
        for k, tri in enumerate(((0, 1, 2), (0, 2, 3))):
            p = panes[2 * q + k]
            for v, c in zip(("v0", "v1", "v2"), tri):
                p[v]["x"], p[v]["y"], p[v]["z"] = corners[c][0], y, corners[c][1]
            for n in ("n0", "n1", "n2"):
                p[n]["y"] = 1.0
            p["mat_index"] = 4
    tris = np.concatenate([box, panes])
    mats = np.concatenate([base.materials(), base.materials()[:1]]).copy()
    glass = mats[4]
    glass["transmission"], glass["roughness"], glass["ior"] = 1.0, 0.1, 1.5
    glass["base_color"]["x"], glass["base_color"]["y"], glass["base_color"]["z"] = 0.9, 0.95, 0.9
    lights = base.lights().copy()
    light_tris = np.flatnonzero(tris["mat_index"] == 3)
    aux = np.array([lights[0]["aux"][c] for c in "xyzw"], np.float32).view(np.uint32)
    aux[1], aux[2] = light_tris[0], len(light_tris)  # emissive range within the triangle array
    for c, v in zip("xyzw", aux.view(np.float32)):
        lights[0]["aux"][c] = v
    return _scene_from_arrays(tris, mats, lights, base.scene.camera)


def _pcg_draw(v, k):
    """Draw k of the PCG stream pcg_seed(v) (random.h:16-34), as a u32."""
    m = 0xFFFFFFFF
    state = ((2891336453 + v) * 747796405 + 2891336453) & m
    for _ in range(k + 1):
        old = state
        state = (state * 747796405 + 2891336453) & m
    return (((old >> ((old >> 28) + 4)) ^ old) * 277803737) & m


@pytest.mark.parametrize("v", [37166213, 7983376])
def test_axis_aligned_photons(v):
    """A photon leaving a point light along -z or +z, its x and y direction components exactly
    zero: draw 1 of its stream (the unit-sphere sample's z, after the light choice) is 7 or
    2^32 - 86, so z = 2u - 1 rounds to -1 or +1.  The traversal's x and y slabs then use a finite
    stand-in for 1/0; the -z photon still finds the back wall of the box and the bounces after it,
    the +z one leaves through the open front, and every photon equals the oracle's."""
    t = 5
    w = _pcg_draw(v, 1)
    assert w < 64 or w >= (1 << 32) - 128
    base = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=16, height=16)
    tris = base.triangles()[:10].copy()  # the box without its ceiling light; back wall at z = 0
    mats = base.materials()[:3].copy()
    lights = np.zeros(1, dtype=base.lights().dtype)
    lights[0]["kind"] = A.PHX_LIGHT_POINT
    for c, x in zip("xyz", (0.3, 0.6, 0.5)):
        lights[0]["position"][c] = x
        lights[0]["power"][c] = 1.0
    scene = _scene_from_arrays(tris, mats, lights, base.scene.camera)
    args = P.ArgsList(width=16, height=16, photons_per_round=64, max_photon_bounces=4, grid_res=8, seed=1,
                      direct_samples=4)
    seed = (v - t) & 0xFFFFFFFF  # photon t's stream is pcg_seed(seed + t)
    o = O.Oracle(scene)
    ocounts, opos, opower, odir = o.emit(0, args.photons_per_round, args.max_photon_bounces, seed)
    first = int(np.sum(ocounts[:t]))
    if w < 64:  # straight at the back wall
        assert ocounts[t] >= 1 and np.array_equal(opos[first, :3], np.array([0.3, 0.6, 0.0], np.float32))
    else:
        assert ocounts[t] == 0
    with P.Renderer(args) as r:
        r.set_scene(scene)
        n = r.emit_photons(seed)
        assert n == len(opos)
        assert np.array_equal(r.read("EMIT_COUNT"), ocounts)
        assert np.array_equal(r.read("PHOTON_POWER"), opower)
        assert np.array_equal(r.read("PHOTON_DIR"), odir)
        assert np.array_equal(r.read("PHOTON_POS").view(np.uint32), np.asarray(opos, np.float32).view(np.uint32))
        assert r.info().stack_overflows == 0


def test_shadow_rays_through_several_transmissive_surfaces():
    """Shadow rays that cross more transmissive surfaces than one traversal lists go on with
    closest-hit queries past the listed ones; hit points (direct light included) stay bit-exact."""
    scene = _glass_panes_scene()
    args = P.ArgsList(width=40, height=40, photons_per_round=1 << 12, max_photon_bounces=8, grid_res=16,
                      direct_samples=16)
    o = O.Oracle(scene)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        seed = 0x51ED
        r.trace_rays(seed)
        got = np.stack([r.read(b) for b in ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT",
                                             "HP_EMISSION"]], axis=1)
        r.iterate(2)
        assert r.info().stack_overflows == 0
    want = o.trace(args.width, args.height, seed, args.direct_samples)
    assert assert_close("panes hit points", got, want) == 1.0
    diffuse = want[:, 5, 3] == 1.0
    assert diffuse.mean() > 0.3 and (want[diffuse, 4, :3] > 0).any()  # light reaches through the panes


def test_shadow_rays_through_a_textured_transmissive_pane():
    """Shadow rays crossing a transmissive surface whose base colour is a texture: the hit list of
    the shadow traversal keeps no barycentrics, so the crossing recomputes u, v for the texture
    lookup; hit points (direct light included) must stay bit-exact.  The scene is the textured
    Cornell box of the reference fixture with a horizontal pane of its textured, half-transmissive
    material between the floor and the light."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import ref_fixture as F
    case = next(c for c in F.load_cases() if c["name"] == "cornell_textured")
    arrays = {k[len("arr_"):]: v for k, v in case.items() if k.startswith("arr_")}
    base = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=16, height=16)
    dt = base.triangles().dtype
    tris = np.frombuffer(arrays["tris"].tobytes(), dtype=dt).copy()
    mats = np.frombuffer(arrays["mats"].tobytes(), dtype=base.materials().dtype)
    glass = [i for i, m in enumerate(mats) if m["transmission"] > 0.0 and m["diff_index"] != 0xFFFFFFFF]
    assert glass, "the textured fixture has a textured transmissive material"
    pane = np.zeros(2, dtype=dt)
    corners = [(0.1, 0.1), (0.9, 0.1), (0.9, 0.9), (0.1, 0.9)]
    for k, tri in enumerate(((0, 1, 2), (0, 2, 3))):
        p = pane[k]
        for v, uv, c in zip(("v0", "v1", "v2"), ("uv0", "uv1", "uv2"), tri):
            p[v]["x"], p[v]["y"], p[v]["z"] = corners[c][0], 0.55, corners[c][1]
            p[uv]["x"], p[uv]["y"] = corners[c][0] * 1.7, corners[c][1] * 0.8
        for n in ("n0", "n1", "n2"):
            p[n]["y"] = 1.0
        p["mat_index"] = glass[0]
    arrays["tris"] = np.frombuffer(np.concatenate([tris, pane]).tobytes(), np.uint8).copy()
    scene = F.ArrayScene(arrays)
    args = P.ArgsList(width=40, height=40, photons_per_round=1 << 12, max_photon_bounces=8, grid_res=16,
                      direct_samples=16)
    o = O.Oracle(scene)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        seed = 0x7A3E
        r.trace_rays(seed)
        got = np.stack([r.read(b) for b in ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT",
                                             "HP_EMISSION"]], axis=1)
    want = o.trace(args.width, args.height, seed, args.direct_samples)
    assert assert_close("textured pane hit points", got, want) == 1.0
    below = (want[:, 5, 3] == 1.0) & (want[:, 0, 1] < 0.5)  # diffuse hit points under the pane
    assert below.mean() > 0.1 and (want[below, 4, :3] > 0).any()  # light reaches them through it


def test_light_samples_with_varying_draws_and_few_samples():
    """Light samples are drawn where their shadow rays are traced, each from the RNG state advanced
    past the samples before it, when every light sample takes the same number of draws.  Two other
    forms remain and must give the same bits: lights whose samples take different draws (an area
    light and a point light: samples drawn by k_nee_sample and by the camera pass), and fewer than
    four samples per specular event (drawn by the camera pass)."""
    base = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=32, height=32)
    tris = base.triangles().copy()
    mats = base.materials().copy()
    mats[0]["metallic"], mats[0]["roughness"] = 0.3, 0.2  # specular events on the white walls
    lights = np.zeros(2, dtype=base.lights().dtype)
    lights[0] = base.lights()[0]
    aux = np.array([lights[0]["aux"][c] for c in "xyzw"], np.float32).view(np.uint32)
    light_tris = np.flatnonzero(tris["mat_index"] == 3)
    aux[1], aux[2] = light_tris[0], len(light_tris)
    for c, v in zip("xyzw", aux.view(np.float32)):
        lights[0]["aux"][c] = v
    lights[1]["kind"] = A.PHX_LIGHT_POINT
    for c, v in zip("xyzw", (0.3, 0.8, 0.4, 1.0)):
        lights[1]["position"][c] = v
    for c, v in zip("xyzw", (1.5, 1.2, 0.9, 0.0)):
        lights[1]["power"][c] = v
    mixed = _scene_from_arrays(tris, mats, lights, base.scene.camera)
    single = _scene_from_arrays(tris, mats, lights[:1].copy(), base.scene.camera)
    for scene, ds in ((mixed, 16), (single, 2), (mixed, 3)):
        args = P.ArgsList(width=40, height=40, photons_per_round=1 << 12, max_photon_bounces=8, grid_res=16,
                          direct_samples=ds)
        o = O.Oracle(scene)
        with P.Renderer(args) as r:
            r.set_scene(scene)
            seed = 0x5EED + ds
            r.trace_rays(seed)
            got = np.stack([r.read(b) for b in ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR",
                                                 "HP_DIRECT", "HP_EMISSION"]], axis=1)
            r.iterate(2)
            assert r.info().stack_overflows == 0
        want = o.trace(args.width, args.height, seed, args.direct_samples)
        assert assert_close(f"lights {len(scene.lights())} ds {ds}", got, want) == 1.0
        assert (want[:, 4, :3] > 0).any()


def test_state_and_argument_errors():
    scene, args = make("cornell")
    lib = A.load()
    with P.Renderer(args) as r:
        r.set_scene(scene)
        with pytest.raises(P.PhxError) as e:
            r.hash_and_sort_photons()
        assert e.value.code == A.PHX_E_STATE
        buf = np.zeros(4, np.float32)
        assert lib.phx_read_buffer(r.ctx, 99, buf.ctypes.data, 0, 16) == A.PHX_E_INVALID
        assert lib.phx_read_buffer(r.ctx, A.BUF["FLUX"], buf.ctypes.data, 10**9, 16) == A.PHX_E_INVALID
        assert lib.phx_set_n_photons(r.ctx, 2**31) == A.PHX_E_INVALID
        t = r.tuning()
        t.trace_block = 33
        assert lib.phx_set_tuning(r.ctx, C.byref(t)) == A.PHX_E_INVALID


def test_lookback_wait_gives_up_with_a_status():
    """Failure detection without a fault: a scan whose tile 0 never publishes must time out,
    report PHX_E_TIMEOUT and leave the device usable."""
    lib = A.load()
    flags = C.c_uint32()
    assert lib.phx_selftest_lookback_timeout(0, 1 << 16, C.byref(flags)) == A.PHX_E_TIMEOUT
    assert flags.value & 1
    scene, args = make("cornell")  # the context still works afterwards
    with P.Renderer(args) as r:
        r.set_scene(scene)
        r.iterate(1)
        assert r.info().error_flags == 0
