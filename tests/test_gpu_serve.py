"""The continuous-batching server (sk_server_*): every request's image equals its plain frame,
alone and in a mix of scenes and sizes, and admission sheds what cannot fit.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

SIZES = [(320, 240), (640, 480), (256, 144), (480, 480)]


def request_frames(scenes, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        s = int(rng.integers(0, len(scenes)))
        w, h = SIZES[int(rng.integers(0, len(SIZES)))]
        view, eye = skcam.orbit_view(int(rng.integers(0, 120)), radius=float(rng.uniform(8, 16)))
        proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0)
        out.append((s, sk.Frame(view, proj, eye, [(0, scenes[s][1].count)], 3), w, h))
    return out


def plain_image(renderer, frame, w, h):
    renderer.resize(w, h)
    renderer.draw(frame)
    return renderer.read_image(sk.FORMAT_RGBA8).copy(), renderer.stats()["draw_count"]


@pytest.fixture(scope="module")
def scenes(cuda_device):
    out = []
    for n, seed in ((60_000, 11), (150_000, 12), (20_000, 13)):
        cloud = synthetic.random_cloud(n, seed=seed, sh_degree=3)
        r = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
        r.apply_render_policy(sk.Policy(sort_depth_bits=16))
        r.upload_world(cloud, 3)
        out.append((r, cloud))
    yield out
    for r, _ in out:
        r.close()


def serve(scenes, frames, arrival_us, **config):
    with sk.Server(lanes=2, max_batch_views=8, **config) as server:
        ids = [server.add_scene(r) for r, _ in scenes]
        assert ids == list(range(len(scenes)))
        images = [sk.HostImage(w, h) for _, _, w, h in frames]
        requests = [sk.Request(s, f, w, h, img) for (s, f, w, h), img in zip(frames, images)]
        done = server.replay(requests, arrival_us)
    return done, images


@pytest.mark.gpu
def test_every_request_equals_its_plain_frame_in_the_mix(scenes):
    frames = request_frames(scenes, 40, seed=5)
    arrivals = np.cumsum(np.random.default_rng(6).exponential(300.0, len(frames)))  # ~3300 req/s
    done, images = serve(scenes, frames, arrivals)
    batched = 0
    for (s, f, w, h), c, img in zip(frames, done, images):
        assert c["status"] == sk.SK_OK
        assert c["latency_ms"] >= c["queue_ms"] >= 0.0
        want, visible = plain_image(scenes[s][0], f, w, h)
        assert c["visible"] == visible
        assert np.array_equal(img.array, want)
        batched += c["batch_views"] > 1
    assert batched > 0  # arrivals overlapped and were batched together


@pytest.mark.gpu
def test_a_request_is_the_same_alone_and_in_the_mix(scenes):
    frames = request_frames(scenes, 12, seed=8)
    mixed, mixed_images = serve(scenes, frames, [0.0] * len(frames))
    for k in (0, 5, 11):
        alone, alone_images = serve(scenes, [frames[k]], [0.0])
        assert alone[0]["status"] == mixed[k]["status"] == sk.SK_OK
        assert alone[0]["visible"] == mixed[k]["visible"]
        assert np.array_equal(alone_images[0].array, mixed_images[k].array)


@pytest.mark.gpu
def test_admission_sheds_what_cannot_fit(scenes):
    (r, cloud) = scenes[1]
    frames = request_frames(scenes, 6, seed=9)
    # a budget that holds the scenes but not one request of the largest scene
    budget = sum(sk.world_bytes(c.count, 3, 0) for _, c in scenes) + 52 * 100_000
    done, _ = serve(scenes, frames, [0.0] * len(frames), memory_budget=budget)
    for (s, _, w, h), c in zip(frames, done):
        fits = 52 * scenes[s][1].count + 4 * w * h <= 52 * 100_000
        assert c["status"] == (sk.SK_OK if fits else sk.SK_E_ADMISSION), (s, w, h)


# ---- LOD scenes ------------------------------------------------------------------------------
LOD_W, LOD_H = 480, 320


def lod_frame(x, w=LOD_W, h=LOD_H):
    eye = np.array([x, 1.7, 35.0], np.float32)
    view = skcam.look_at_view(eye, (x * 0.5, 0.0, 0.0))
    proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 400.0)
    return sk.Frame(view, proj, eye, [], 0)


@pytest.fixture(scope="module")
def lod_trees(cuda_device):
    trees = []
    for seed in (71, 72):
        cloud = synthetic.clustered_cloud(40, 600, seed=seed, half_extent=25.0)
        trees.append(sk.build_lod_tree(cloud))
    return trees


def lod_renderer(tree, policy):
    r = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
    r.apply_render_policy(policy)
    r.upload_lod_world(tree, 0, 4_000_000)
    return r


@pytest.mark.gpu
def test_lod_scene_requests_equal_their_plain_frames(lod_trees, cuda_device):
    """LOD scenes beside a flat one: each request's cut is selected on the server's lane and its
    image equals the plain frame of the scene's own context."""
    policy = sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16)
    flat_cloud = synthetic.random_cloud(30_000, seed=73, sh_degree=0)
    flat = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
    flat.apply_render_policy(policy)
    flat.upload_world(flat_cloud, 0)
    scenes = [(lod_renderer(t, policy), None) for t in lod_trees] + [(flat, flat_cloud)]
    rng = np.random.default_rng(74)
    frames = []
    for i in range(24):
        s = int(rng.integers(0, 3))
        w, h = SIZES[int(rng.integers(0, len(SIZES)))]
        f = lod_frame(float(rng.uniform(-30, 30)), w, h)
        if s == 2:
            f = sk.Frame(f.view, f.proj, f.camera_position, [(0, flat_cloud.count)], 0)
        frames.append((s, f, w, h))
    arrivals = np.cumsum(rng.exponential(200.0, len(frames)))
    try:
        done, images = serve(scenes, frames, arrivals)
        batched = 0
        for (s, f, w, h), c, img in zip(frames, done, images):
            assert c["status"] == sk.SK_OK
            want, visible = plain_image(scenes[s][0], f, w, h)
            assert c["visible"] == visible > 0
            assert np.array_equal(img.array, want)
            batched += c["batch_views"] > 1
        assert batched > 0
    finally:
        for r, _ in scenes:
            r.close()


@pytest.mark.gpu
def test_a_lod_scene_keeps_its_threshold_across_requests(lod_trees, cuda_device):
    """A splat limit that binds: the scene's adaptive threshold rises request after request
    (LodThreshold.h:27-36), fed by each completed request's cut. Served one at a time, the
    requests draw exactly the frames the scene's own context draws for the same camera path."""
    tree = lod_trees[0]
    leaves = tree.leaf_count
    policy = sk.Policy(lod_error_pixels=0.5, lod_splat_limit=leaves // 6, sort_depth_bits=16)
    served_scene = lod_renderer(tree, policy)
    plain = lod_renderer(tree, policy)
    frames = [(0, lod_frame(-20.0 + 2.0 * k), LOD_W, LOD_H) for k in range(12)]
    try:
        with sk.Server(lanes=1, max_batch_views=1) as server:
            server.add_scene(served_scene)
            images = [sk.HostImage(LOD_W, LOD_H) for _ in frames]
            requests = [sk.Request(0, f, w, h, img) for (_, f, w, h), img in zip(frames, images)]
            done = server.replay(requests, [0.0] * len(frames))
        thresholds = []
        for (_, f, w, h), c, img in zip(frames, done, images):
            assert c["status"] == sk.SK_OK
            want, visible = plain_image(plain, f, w, h)
            thresholds.append(plain.stats()["lod_pixels"])
            assert c["visible"] == visible
            assert np.array_equal(img.array, want)
        assert thresholds[-1] > thresholds[0] > 0.5  # the limit bound and the threshold rose
        assert served_scene.stats()["lod_pixels"] == pytest.approx(thresholds[-1])
    finally:
        served_scene.close()
        plain.close()
