"""phx_scan_noalloc, the exclusive scan whose scratch is a static device array (needs a GPU).

The scan is checked against the cell starts phx_hash_sort computes with the round's own scan
(which the parity tests pin to the oracle), twice in a row on the same static scratch, and
against numpy at its maximum size.  Integer results must be bit-exact (tolerance 0).
"""
import numpy as np
import pytest
import torch

import phosphor_b200 as P
from phosphor_b200 import _capi as A

MAX_N = 1 << 24


def scan(lib, inp: torch.Tensor, out: torch.Tensor, total: torch.Tensor) -> None:
    stream = torch.cuda.current_stream().cuda_stream
    A.check(lib.phx_scan_noalloc(inp.data_ptr(), out.data_ptr(), inp.numel(), total.data_ptr(), stream))


def test_rejects_sizes_beyond_its_static_scratch():
    lib = A.load()
    buf = np.zeros(1, np.uint32)  # never touched: the size check comes first
    rc = lib.phx_scan_noalloc(buf.ctypes.data, buf.ctypes.data, MAX_N + 1, None, 0)
    assert rc == A.PHX_E_INVALID
    assert "maximum" in lib.phx_last_error().decode()


@pytest.mark.gpu
def test_matches_the_rounds_cell_starts_twice_in_a_row():
    lib = A.load()
    scene = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=5, width=64, height=48)
    args = P.ArgsList(width=64, height=48, photons_per_round=1 << 15, max_photon_bounces=8, grid_res=100, seed=5)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        r.trace_rays(0x1234567)
        r.emit_photons(0x89ABCDE)
        r.hash_and_sort_photons()
        counts = r.read("CELL_COUNT")
        starts = r.read("CELL_START")
        ends = r.read("CELL_END")
    assert counts.size > 4096 * 3 and counts.sum() > 0
    inp = torch.from_numpy(counts.view(np.int32)).cuda()
    for _ in range(2):
        out = torch.full_like(inp, -1)
        total = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        scan(lib, inp, out, total)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), starts)
        assert int(total.cpu().numpy().view(np.uint32)[0]) == int(ends[-1])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 4095, 4097, MAX_N])
def test_matches_numpy_up_to_the_maximum(n):
    lib = A.load()
    rng = np.random.default_rng(n)
    host = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    want = (np.cumsum(host, dtype=np.uint64) - host).astype(np.uint32)  # exclusive, mod 2^32
    inp = torch.from_numpy(host.view(np.int32)).cuda()
    out = torch.full_like(inp, -1)
    total = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        scan(lib, inp, out, total)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
        want_total = int(host.astype(np.uint64).sum() & 0xFFFFFFFF)
        assert int(total.cpu().numpy().view(np.uint32)[0]) == want_total
