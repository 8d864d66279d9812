"""The reference-side adapter on the GPU: a frame drawn through the reference engine's renderer
interface (splatkit::SplatRenderer::draw, SplatRenderer.h:134, as CudaSplatRenderer implements it
over the C ABI; tests/adapter/draw_through_renderer.cpp) is the frame the C ABI draws for the same
cloud and camera, byte for byte, uploaded as one world or as tiles of a slab
(createSlab / uploadTile, SplatRenderer.h:91-103).

The adapter program is compiled where the reference's headers are (the build step) and carried
with the repository; the test skips when it was never built."""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
PROGRAM = ROOT / "tests" / "adapter" / "_bin" / "draw_through_renderer"
W, H = 480, 320


def write_input(path: Path, cloud: sk.Cloud, view, proj, eye, tiles: int):
    header = np.array([cloud.count, cloud.sh_degree, W, H, tiles], np.uint32)
    parts = [header.tobytes(), np.asarray(view, np.float32).tobytes(),
             np.asarray(proj, np.float32).tobytes(), np.asarray(eye, np.float32).tobytes()]
    for a in (cloud.positions, cloud.covariances, cloud.colors, cloud.alphas):
        parts.append(np.ascontiguousarray(a, np.float32).tobytes())
    if cloud.sh_degree:
        parts.append(np.ascontiguousarray(cloud.sh, np.float32).tobytes())
    path.write_bytes(b"".join(parts))


@pytest.mark.skipif(not PROGRAM.exists(), reason="the adapter program was not built (no reference headers)")
@pytest.mark.parametrize("tiles", [0, 3])
def test_a_frame_through_the_engine_interface_is_the_c_abi_frame(tmp_path, cuda_device, tiles):
    cloud = synthetic.random_cloud(60_000, seed=61, sh_degree=2)
    view, eye = skcam.orbit_view(23)
    proj = skcam.perspective(math.radians(60.0), W / H, 0.05, 200.0)
    write_input(tmp_path / "in.bin", cloud, view, proj, eye, tiles)
    run = subprocess.run([str(PROGRAM), str(tmp_path / "in.bin"), str(tmp_path / "out.rgba")],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    print(run.stdout.strip())
    got = np.frombuffer((tmp_path / "out.rgba").read_bytes(), np.uint8).reshape(H, W, 4)
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA8) as r:
        r.apply_render_policy(sk.Policy())  # RenderPolicy{}
        r.upload_world(cloud, cloud.sh_degree)
        r.draw(sk.Frame(view, proj, eye, [(0, cloud.count)], cloud.sh_degree))
        want = r.read_image(sk.FORMAT_RGBA8)
        drawn = r.stats()["draw_count"]
    assert f"drawn={drawn} " in run.stdout
    assert got.tobytes() == want.tobytes()
