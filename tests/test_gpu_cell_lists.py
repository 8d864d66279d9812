"""Cell lists written in place (binning.cu launchCellLists) against the stable (cell, splat) sort
they replace on targets of up to 4096 binning cells: the same front-to-back list per cell, the
same instance count and the same image. Cases: a 1080p frame, an odd target, the 4096-cell limit,
splats whose boxes exceed 64 cells (walked by the whole warp) with an instance overflow that
regrows the buffers, consecutive frames on one renderer, and a frame with no survivors."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic


def draw_lists(cloud, frames, w, h, mode):
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA32F)
    r.set_binning(mode)
    r.upload_world(cloud, cloud.sh_degree)
    out = []
    for frame in frames:
        r.draw(frame)
        ranges, values = r.read_tile_lists()
        out.append((ranges, values, r.read_image(sk.FORMAT_RGBA32F), r.stats()["instances"]))
    r.close()
    return out


def frames_for(cloud, w, h, steps, radius=15.0):
    out = []
    for step in steps:
        view, eye = skcam.orbit_view(step, radius=radius)
        proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0)
        out.append(sk.Frame(view, proj, eye, [(0, cloud.count)], cloud.sh_degree))
    return out


def assert_same_lists(direct, sorted_):
    for (ra, va, ia, na), (rb, vb, ib, nb) in zip(direct, sorted_):
        assert na == nb
        assert len(va) == len(vb) == na
        assert np.array_equal(va, vb)
        nonempty = rb[:, 1] > rb[:, 0]
        assert np.array_equal(ra[nonempty], rb[nonempty])
        assert np.all(ra[~nonempty, 0] == ra[~nonempty, 1])
        assert np.array_equal(ia, ib)


@pytest.mark.gpu
@pytest.mark.parametrize("n,w,h,log_scale", [
    (200_000, 1920, 1080, -3.0),
    (60_000, 333, 97, -1.5),
    (120_000, 2048, 2048, -2.5),   # 64 x 64 = 4096 cells, the largest direct target
    (6_000, 640, 480, 1.0),        # boxes of more than 64 cells; the first draw overflows
])
def test_direct_lists_equal_the_sorted_lists(cuda_device, n, w, h, log_scale):
    cloud = synthetic.random_cloud(n, seed=31, sh_degree=1, log_scale_mean=log_scale)
    frames = frames_for(cloud, w, h, (3, 40, 41))
    direct = draw_lists(cloud, frames, w, h, "auto")
    assert_same_lists(direct, draw_lists(cloud, frames, w, h, "sorted"))
    assert direct[0][3] > 0
    if log_scale > 0:
        assert direct[0][3] > 8 * n  # more than the first reservation: the frame was redrawn


@pytest.mark.gpu
def test_frame_without_survivors_has_empty_lists(cuda_device):
    cloud = synthetic.random_cloud(10_000, seed=5, sh_degree=0, half_extent=2.0)
    view, eye = skcam.orbit_view(0, radius=15.0)
    proj = skcam.perspective(math.radians(60.0), 4 / 3, 0.05, 1.0)  # far plane before the cloud
    frame = sk.Frame(view, proj, eye, [(0, cloud.count)], 0)
    (ranges, values, image, count), = draw_lists(cloud, [frame], 640, 480, "auto")
    assert count == 0 and len(values) == 0
    assert np.all(ranges[:, 0] == ranges[:, 1])
