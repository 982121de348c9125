"""phx_render, the C++ host over the C ABI: flag handling (CPU) and a small render (GPU)."""
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CLI = ROOT / "phosphor_b200" / "phx_render"


@pytest.fixture(scope="module", autouse=True)
def cli_built():
    from phosphor_b200.build import build_cli
    build_cli()


def run(*args, timeout=120):
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=timeout)


def read_png(path: Path) -> np.ndarray:
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n = int.from_bytes(data[pos:pos + 4], "big")
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h = int.from_bytes(body[:4], "big"), int.from_bytes(body[4:8], "big")
        elif tag == b"IDAT":
            idat += body
        crc = int.from_bytes(data[pos + 8 + n:pos + 12 + n], "big")
        assert crc == zlib.crc32(tag + body) & 0xFFFFFFFF
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 3 * w + 1)
    assert np.all(rows[:, 0] == 0)
    return rows[:, 1:].reshape(h, w, 3)


def test_help_and_bad_flags():
    r = run("--help")
    assert r.returncode == 1 and "--sppm-rounds" in r.stderr
    r = run("--max-bounces", "0")
    assert r.returncode == 1 and "out of range" in r.stderr
    r = run("--grid-res", "256")
    assert r.returncode == 1
    r = run("--scene", "sponza")
    assert r.returncode == 1 and "--scene" in r.stderr
    r = run("--bogus")
    assert r.returncode == 1 and "unknown flag" in r.stderr


@pytest.mark.gpu
def test_cli_render_writes_the_device_image(tmp_path):
    out = tmp_path / "render"
    r = run("--scene", "cornell", "-w", "64", "-h", "48", "-p", "8192", "--max-bounces", "8", "--grid-res", "50",
            "--sppm-rounds", "5", "--snapshots", "--seed", "3", "-o", str(out))
    assert r.returncode == 0, r.stderr
    assert "Mphotons/s" in r.stdout
    files = sorted(p.name for p in out.glob("*.png"))
    assert files == ["000001.png", "000002.png", "000004.png", "000005.png"]
    img = read_png(out / "000005.png")
    assert img.shape == (48, 64, 3)
    # the same render through the Python binding gives the same 8-bit image
    import phosphor_b200 as P
    args = P.ArgsList(width=64, height=48, photons_per_round=8192, max_photon_bounces=8, grid_res=50, seed=3)
    scene = P.SceneData.generate(0, seed=3, width=64, height=48)
    with P.Renderer(args) as rr:
        rr.set_scene(scene)
        rr.iterate(5)
        assert np.array_equal(rr.image_u8(), img)


def test_missing_model_file_is_an_error(tmp_path):
    r = run("-m", str(tmp_path / "none.glb"))
    assert r.returncode == 1 and "cannot read" in r.stderr


@pytest.mark.gpu
def test_cli_renders_a_gltf_scene(tmp_path):
    """-m renders a .glb through phx_scene_load_gltf; the image equals the Python binding's render
    of the same loaded scene."""
    import math

    import phosphor_b200 as P
    from gltf_writer import Gltf
    g = Gltf()
    quad = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]], np.float32)
    idx = np.array([0, 2, 1, 0, 3, 2], np.uint16)
    floor = g.material(pbrMetallicRoughness={"baseColorFactor": [0.8, 0.7, 0.6, 1.0], "metallicFactor": 0.0})
    g.node(mesh=g.mesh([{"attributes": {"POSITION": g.accessor(quad)}, "indices": g.accessor(idx, 5123),
                         "material": floor}]))
    lamp = g.light(type="point", color=[1.0, 1.0, 1.0], intensity=3000.0)
    g.node(extensions={"KHR_lights_punctual": {"light": lamp}}, translation=[0.5, 0.8, 0.5])
    q = [math.sin(-0.6 / 2), 0.0, 0.0, math.cos(-0.6 / 2)]  # look down 0.6 rad
    g.node(camera=g.camera(0.8, 1.0), translation=[0.5, 0.9, 2.0], rotation=q)
    g.write_glb(tmp_path / "floor.glb")
    out = tmp_path / "render"
    r = run("-m", str(tmp_path / "floor.glb"), "-w", "48", "-h", "40", "-p", "8192", "--max-bounces", "4",
            "--grid-res", "32", "--sppm-rounds", "3", "--seed", "5", "-o", str(out))
    assert r.returncode == 0, r.stderr
    img = read_png(out / "000003.png")
    scene = P.SceneData.load_gltf(tmp_path / "floor.glb", width=48, height=40)
    args = P.ArgsList(width=48, height=40, photons_per_round=8192, max_photon_bounces=4, grid_res=32, seed=5)
    with P.Renderer(args) as rr:
        rr.set_scene(scene)
        rr.iterate(3)
        assert np.array_equal(rr.image_u8(), img)
    assert img.mean() > 1.0
