"""captureNextFrame (sk_capture_next_frame / sk_wait_capture): captures taken one frame behind the
draws, copied while the next frame renders, hold exactly the images sk_read_image gives for the
same frames; a frame redrawn after an overflow of its lists is captured as redrawn; misuse is
rejected; the timing modes draw the same pixels."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic


def frames_for(cloud, w, h, steps):
    out = []
    for step in steps:
        view, eye = skcam.orbit_view(step, radius=15.0)
        proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0)
        out.append(sk.Frame(view, proj, eye, [(0, cloud.count)], cloud.sh_degree))
    return out


def read_back(cloud, frames, w, h, fmt):
    r = sk.Renderer(w, h, image_format=fmt)
    r.upload_world(cloud, cloud.sh_degree)
    out = []
    for f in frames:
        r.draw(f)
        out.append(r.read_image(fmt).copy())
    r.close()
    return out


def pinned_image(w, h, fmt):
    if fmt == sk.FORMAT_RGBA32F:
        return torch.empty((h, w, 4), dtype=torch.float32, pin_memory=True).numpy()
    return torch.empty((h, w, 4), dtype=torch.uint8, pin_memory=True).numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [sk.FORMAT_RGBA8, sk.FORMAT_RGBA32F])
def test_captures_one_frame_behind_equal_read_image(cuda_device, fmt):
    w, h = 640, 480
    cloud = synthetic.random_cloud(200_000, seed=41, sh_degree=1)
    frames = frames_for(cloud, w, h, range(0, 60, 7))
    r = sk.Renderer(w, h, image_format=fmt)
    r.upload_world(cloud, 1)
    buffers = [pinned_image(w, h, fmt) for _ in range(2)]
    captured, previous = [], None
    for k, f in enumerate(frames):
        ticket = r.capture_next_frame(buffers[k % 2])
        r.draw(f)
        if previous is not None:
            captured.append(r.wait_capture(previous).copy())
        previous = ticket
    captured.append(r.wait_capture(previous).copy())
    # a plain readback on the same renderer after captures: the last drawn frame
    r.draw(frames[2])
    last = r.read_image(fmt).copy()
    r.close()
    expected = read_back(cloud, frames, w, h, fmt)
    for got, want in zip(captured, expected):
        assert np.array_equal(got, want)
    assert np.array_equal(last, expected[2])


@pytest.mark.gpu
def test_capture_of_a_redrawn_frame(cuda_device):
    # boxes of many cells: the first draw overflows the first list reservation and is redrawn
    w, h = 640, 480
    cloud = synthetic.random_cloud(6_000, seed=31, sh_degree=1, log_scale_mean=1.0)
    frames = frames_for(cloud, w, h, (3, 40))
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    r.upload_world(cloud, 1)
    buf = pinned_image(w, h, sk.FORMAT_RGBA8)
    got = []
    for f in frames:
        t = r.capture_next_frame(buf)
        r.draw(f)
        got.append(r.wait_capture(t).copy())
    assert r.stats()["instances"] > 8 * cloud.count
    r.close()
    for g, want in zip(got, read_back(cloud, frames, w, h, sk.FORMAT_RGBA8)):
        assert np.array_equal(g, want)


@pytest.mark.gpu
def test_capture_misuse_is_rejected(cuda_device):
    w, h = 320, 240
    cloud = synthetic.random_cloud(20_000, seed=5, sh_degree=0)
    (frame,) = frames_for(cloud, w, h, (0,))
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    r.upload_world(cloud, 0)
    lib = sk.library()
    import ctypes
    t = ctypes.c_uint64()
    small = np.empty((h, w, 2), np.uint8)
    assert lib.sk_capture_next_frame(r._h, small.ctypes.data, small.nbytes, sk.FORMAT_RGBA8,
                                     ctypes.byref(t)) == sk.SK_E_INVALID
    buf = np.empty((h, w, 4), np.uint8)
    assert lib.sk_capture_next_frame(r._h, buf.ctypes.data, buf.nbytes, sk.FORMAT_RGBA32F,
                                     ctypes.byref(t)) == sk.SK_E_INVALID
    ticket = r.capture_next_frame(buf)
    with pytest.raises(sk.SplatError):  # one capture waits for the next frame at a time
        r.capture_next_frame(np.empty((h, w, 4), np.uint8))
    with pytest.raises(sk.SplatError):  # its frame is not drawn yet
        r.wait_capture(ticket)
    r.resize(2 * w, 2 * h)  # the target outgrows the buffer before the frame is drawn
    r.draw(frame)
    with pytest.raises(sk.SplatError):
        r.wait_capture(ticket)
    assert lib.sk_wait_capture(r._h, 12345) == sk.SK_E_INVALID
    # the renderer keeps working
    r.draw(frame)
    assert r.read_image(sk.FORMAT_RGBA8).shape == (2 * h, 2 * w, 4)
    r.close()


@pytest.mark.gpu
def test_two_frames_in_flight_with_an_overflow(cuda_device):
    # three draws without a wait: the first overflows its lists while the second is queued, so
    # both are drawn again before the third takes the first one's slot
    w, h = 640, 480
    cloud = synthetic.random_cloud(6_000, seed=31, sh_degree=1, log_scale_mean=1.0)
    frames = frames_for(cloud, w, h, (3, 40, 41))
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    r.upload_world(cloud, 1)
    buffers = [pinned_image(w, h, sk.FORMAT_RGBA8) for _ in frames]
    tickets = []
    for f, b in zip(frames, buffers):
        tickets.append(r.capture_next_frame(b))
        r.draw(f)
    got = [r.wait_capture(t).copy() for t in tickets]
    last = r.read_image(sk.FORMAT_RGBA8).copy()
    stats = r.stats()
    r.close()
    want = read_back(cloud, frames, w, h, sk.FORMAT_RGBA8)
    for g, expected in zip(got, want):
        assert np.array_equal(g, expected)
    assert np.array_equal(last, want[-1])
    assert stats["submitted_frames"] == stats["completed_frames"] == len(frames)


@pytest.mark.gpu
def test_timing_modes_draw_the_same_image(cuda_device):
    # sk_set_timing: 1 per-stage events and fragment counts, 2 the frame's own pair, 0 nothing;
    # none of them changes a pixel
    w, h = 640, 480
    cloud = synthetic.random_cloud(100_000, seed=8, sh_degree=1)
    (frame,) = frames_for(cloud, w, h, (12,))
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    r.upload_world(cloud, 1)
    images, stats = {}, {}
    for mode in (True, "frame", False):
        r.set_timing(mode)
        r.draw(frame)
        images[mode] = r.read_image(sk.FORMAT_RGBA8).copy()
        stats[mode] = r.stats()
    r.close()
    assert np.array_equal(images[True], images["frame"])
    assert np.array_equal(images[True], images[False])
    assert stats[True]["gpu_ms"] > 0 and stats[True]["composite_ms"] > 0
    assert stats[True]["fragments"] > 0
    assert stats["frame"]["gpu_ms"] > 0 and stats["frame"]["composite_ms"] == 0
    for mode in (True, "frame", False):
        assert stats[mode]["draw_count"] == stats[True]["draw_count"]


@pytest.mark.gpu
def test_overlapped_frames_equal_frames_drawn_alone(cuda_device):
    # draws without a wait alternate between the two frame slots, each on its own stream with its
    # own scratch and image: every frame's image equals the one drawn alone, and the read-backs
    # after the last draw give that frame's survivors, records and order
    w, h = 640, 480
    cloud = synthetic.random_cloud(150_000, seed=12, sh_degree=2)
    frames = frames_for(cloud, w, h, range(0, 50, 5))
    alone = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    alone.upload_world(cloud, 2)
    want = []
    for f in frames:
        alone.draw(f)
        keys, projected = alone.read_visible()
        want.append((alone.read_image(sk.FORMAT_RGBA8).copy(), keys, projected, alone.read_order()))
    alone.close()
    r = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    r.upload_world(cloud, 2)
    buffers = [pinned_image(w, h, sk.FORMAT_RGBA8) for _ in frames]
    tickets = []
    for f, b in zip(frames, buffers):
        tickets.append(r.capture_next_frame(b))
        r.draw(f)
    got = [r.wait_capture(t).copy() for t in tickets]
    keys, projected = r.read_visible()
    order = r.read_order()
    for g, expected in zip(got, want):
        assert np.array_equal(g, expected[0])
    assert np.array_equal(keys, want[-1][1]) and projected.tobytes() == want[-1][2].tobytes()
    assert np.array_equal(order, want[-1][3])
    # plain draws in flight (no captures): the image and read-backs are the last frame's
    for k in (3, 4, 7):
        r.draw(frames[k])
    assert np.array_equal(r.read_image(sk.FORMAT_RGBA8), want[7][0])
    keys, projected = r.read_visible()
    assert np.array_equal(keys, want[7][1]) and np.array_equal(r.read_order(), want[7][3])
    stats = r.stats()
    r.close()
    assert stats["submitted_frames"] == stats["completed_frames"] == len(frames) + 3


@pytest.mark.gpu
def test_a_lod_world_after_overlapped_flat_frames_reads_back_its_own_frames(cuda_device):
    # flat frames in flight on both slots, then a LOD world (one slot): its cut, survivors, order
    # and image are a fresh renderer's, not what the second slot's scratch last held
    w, h = 320, 240
    flat = synthetic.random_cloud(60_000, seed=3, sh_degree=1)
    cloud = synthetic.clustered_cloud(24, 400, seed=5, half_extent=8.0, rms=1.0)
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min, cloud.bounds_max = pos.min(axis=0), pos.max(axis=0)
    tree = sk.build_lod_tree(cloud)
    used = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    used.upload_world(flat, 1)
    for f in frames_for(flat, w, h, range(0, 30, 5)):
        used.draw(f)
    fresh = sk.Renderer(w, h, image_format=sk.FORMAT_RGBA8)
    for r in (used, fresh):
        r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
        r.upload_lod_world(tree, 0, 100_000)
    for step in (0, 7, 13):
        view, eye = skcam.orbit_view(step, radius=12.0)
        frame = sk.Frame(view, skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0), eye, [], 0)
        got = []
        for r in (used, fresh):
            r.draw(frame)
            cut, _ = r.read_cut()
            keys, projected = r.read_visible()
            got.append((cut, keys, projected.tobytes(), r.read_order(), r.read_image(sk.FORMAT_RGBA8)))
        (cut, keys, projected, order, image), want = got
        assert len(cut) > 0 and len(keys) > 0
        assert np.array_equal(cut, want[0]) and np.array_equal(keys, want[1])
        assert projected == want[2] and np.array_equal(order, want[3])
        assert np.array_equal(image, want[4])
    used.close()
    fresh.close()
