"""Part-label styling and the reveal glow in the cull (SplatVisibility.metal:69-85,
SplatProjection.metalh:177-189): the oracle pinned to the reference's known answer (CPU), then the
CUDA path bit-exact against the oracle on a labelled cloud with a reveal band (GPU)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

from test_oracle_golden import ref_camera
from scenes import half_bits, unit_cov_splats

IDENTITY = ((1.0, 1.0, 1.0), 0.0, 1.0, 1.0)


def palette_array(entries):
    out = np.zeros((10, 8), np.float32)
    out[:, 0:3], out[:, 4], out[:, 5] = 1.0, 1.0, 1.0
    for i, (tint, amount, brightness, opacity) in enumerate(entries):
        out[i, 0:3], out[i, 3], out[i, 4], out[i, 5] = tint, amount, brightness, opacity
    return out


def test_tinted_label_known_answer(oracle):
    # MetalVisibilityPassTest.mm:568-627: label 65535 -> state 1 -> tint (0, 1, 0), amount 1
    splats = unit_cov_splats([[0, 0, -5]])
    cam = ref_camera(oracle)
    plain_keys, plain = oracle.visibility(cam, splats, None, 0, 0, 32, [(0, 1)])
    labels = np.array([65535], np.uint16)
    states = np.zeros(65536, np.uint32)
    identity_keys, identical = oracle.visibility(
        cam, splats, None, 0, 0, 32, [(0, 1)], parts=(labels, palette_array([IDENTITY]), states))
    assert identical.tobytes() == plain.tobytes()
    states[65535] = 1
    pal = palette_array([IDENTITY, ((0.0, 1.0, 0.0), 1.0, 1.0, 1.0)])
    _, styled = oracle.visibility(cam, splats, None, 0, 0, 32, [(0, 1)], parts=(labels, pal, states))
    assert len(styled) == 1
    assert int(styled["color0"][0]) == half_bits(1.0) << 16


def test_transparent_style_drops_and_unknown_label_is_unstyled(oracle):
    splats = unit_cov_splats([[0, 0, -5], [0.5, 0, -5], [-0.5, 0, -5]])
    cam = ref_camera(oracle)
    _, plain = oracle.visibility(cam, splats, None, 0, 0, 32, [(0, 3)])
    labels = np.array([0, 1, 7], np.uint16)  # label 7 has no state
    pal = palette_array([IDENTITY, ((1.0, 0.0, 0.0), 0.5, 1.0, 0.001)])
    _, styled = oracle.visibility(cam, splats, None, 0, 0, 32, [(0, 3)],
                                  parts=(labels, pal, np.array([0, 1], np.uint32)))
    assert list(styled["index"]) == [0, 2]
    assert styled.tobytes() == plain[[0, 2]].tobytes()


@pytest.mark.gpu
def test_labelled_cloud_with_reveal_band_matches_the_oracle(oracle, cuda_device):
    cloud = synthetic.random_cloud(60_000, seed=21, sh_degree=1, half_extent=6.0)
    rng = np.random.default_rng(22)
    labels = rng.integers(0, 9, cloud.count).astype(np.uint16)  # labels 6..8 have no state
    entries = [IDENTITY, ((1.0, 0.2, 0.1), 0.6, 1.3, 1.0), ((0.0, 0.0, 1.0), 1.0, 0.5, 0.4),
               ((0.3, 0.9, 0.3), 0.25, 1.0, 0.02), ((1.0, 1.0, 1.0), 0.0, 2.0, 1.0)]
    states = np.array([0, 1, 2, 3, 4, 1], np.uint32)
    w, h = 320, 240
    view, eye = skcam.orbit_view(9, radius=12.0)
    proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0)
    frame = sk.Frame(view, proj, eye, [(0, cloud.count)], 1, reveal_level=1.5, reveal_band=3.0,
                     reveal_tint_amount=0.7, reveal_brightness_boost=0.5, reveal_tint=(1.0, 0.6, 0.1))
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA32F)
    r.apply_render_policy(sk.Policy(sort_depth_bits=16))
    r.upload_world(cloud, 1)
    r.upload_labels(labels[:20_000])
    r.upload_labels(labels[20_000:], offset=20_000)
    r.set_part_styles(entries, states)
    r.draw(frame)
    keys, projected = r.read_visible()
    order = r.read_order()
    image = r.read_image(sk.FORMAT_RGBA32F)
    r.close()

    cam = oracle.camera(view, proj, eye, w, h, 1.0)
    cam.reveal[0], cam.reveal[1], cam.reveal[2], cam.reveal[3] = 1.5, 3.0, 0.7, 0.5
    cam.revealTint[0], cam.revealTint[1], cam.revealTint[2] = 1.0, 0.6, 0.1
    stride = sk.sh_device_stride(1)
    okeys, oproj = oracle.visibility(cam, sk.pack_splats(cloud), sk.pack_sh(cloud, 1, stride),
                                     stride, 1, 16, [(0, cloud.count)], threads=8,
                                     parts=(labels, palette_array(entries), states))
    assert np.array_equal(keys, okeys)
    assert projected.tobytes() == oproj.tobytes()
    assert np.array_equal(order, oracle.stable_argsort(okeys))
    ref = oracle.composite(oproj, oracle.stable_argsort(okeys), w, h, precision=64)
    assert np.abs(image[..., :3] - ref[..., :3]).max() <= 1.0 / 255.0
