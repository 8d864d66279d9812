"""The residency slab (SplatRenderer::createSlab / uploadTile, SplatRenderer.h:91-103; the Metal
world's slab, metal/world/MetalWorld.mm:65-100): tiles uploaded into a fixed-capacity slab at
chosen offsets and drawn through per-tile ranges (the multi-range visibility of
SplatVisibility.metal:30-37,61-67) give the frame the same cloud gives uploaded flat: the same
keys, projected records (up to each record's source index, which is its slab position), depth
order and image, bit for bit."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

pytestmark = pytest.mark.gpu

W, H = 640, 480


def part(cloud: sk.Cloud, begin: int, end: int) -> sk.Cloud:
    return sk.Cloud(cloud.positions[begin:end], cloud.covariances[begin:end], cloud.colors[begin:end],
                    cloud.alphas[begin:end], cloud.sh_degree,
                    None if cloud.sh is None else cloud.sh[begin:end])


def frame_of(ranges, degree):
    view, eye = skcam.orbit_view(17)
    proj = skcam.perspective(math.radians(60.0), W / H, 0.05, 200.0)
    return sk.Frame(view, proj, eye, ranges, degree)


def draw(r, frame):
    r.draw(frame)
    keys, projected = r.read_visible()
    return keys, projected, r.read_order(), r.read_image(sk.FORMAT_RGBA32F), r.stats()


@pytest.mark.parametrize("bits", [16, 32])
def test_tiles_in_a_slab_draw_like_the_flat_cloud(cuda_device, bits):
    cloud = synthetic.random_cloud(90_000, seed=41, sh_degree=3)
    cuts = [0, 25_000, 61_000, 90_000]               # three tiles of the cloud
    offsets = [7, 40_000, 120_000]                   # their places in the slab, with gaps
    capacity = 160_000
    policy = sk.Policy(sort_depth_bits=bits)
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F) as flat:
        flat.apply_render_policy(policy)
        flat.upload_world(cloud, 3)
        want = draw(flat, frame_of([(0, cloud.count)], 3))
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F) as slab:
        slab.apply_render_policy(policy)
        slab.create_slab(capacity, 3)
        assert slab.world() == (capacity, 3)
        for k, offset in enumerate(offsets):
            slab.upload_tile(offset, part(cloud, cuts[k], cuts[k + 1]))
        ranges = [(offsets[k], cuts[k + 1] - cuts[k]) for k in range(3)]
        got = draw(slab, frame_of(ranges, 3))
    keys, projected, order, image, stats = got
    wkeys, wprojected, worder, wimage, wstats = want
    assert stats["device_error"] == 0 and len(keys) == len(wkeys) > 0
    assert np.array_equal(keys, wkeys)
    # a survivor's source index is its slab position: tile k's record j sits at offsets[k] + j
    source = wprojected["index"].astype(np.int64)
    tile = np.searchsorted(cuts, source, side="right") - 1
    expected_index = np.asarray(offsets, np.int64)[tile] + source - np.asarray(cuts, np.int64)[tile]
    assert np.array_equal(projected["index"].astype(np.int64), expected_index)
    for name in projected.dtype.names:  # every other field bit for bit
        if name != "index":
            assert projected[name].tobytes() == wprojected[name].tobytes(), name
    assert np.array_equal(order, worder)
    assert image.tobytes() == wimage.tobytes()


def test_a_tile_uploaded_again_replaces_its_records(cuda_device):
    a = synthetic.random_cloud(20_000, seed=42, sh_degree=1)
    b = synthetic.random_cloud(20_000, seed=43, sh_degree=1)
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F) as flat:
        flat.upload_world(b, 1)
        want = draw(flat, frame_of([(0, b.count)], 1))
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F) as slab:
        slab.create_slab(50_000, 1)
        slab.upload_tile(1000, a)
        first = draw(slab, frame_of([(1000, a.count)], 1))
        slab.upload_tile(1000, b)
        got = draw(slab, frame_of([(1000, b.count)], 1))
        with pytest.raises(sk.SplatError) as err:   # past the capacity: nothing is written
            slab.upload_tile(40_000, b)
        assert err.value.status == sk.SK_E_INVALID
        again = draw(slab, frame_of([(1000, b.count)], 1))
    assert not np.array_equal(first[0], got[0])
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[2], want[2])
    assert got[3].tobytes() == want[3].tobytes()
    assert again[3].tobytes() == want[3].tobytes()
