"""The batched multi-view path (sk_batch_*) against the plain per-frame path, view by view.

A batch runs every stage once over all its views (several worlds, several target sizes; the cell
lists in place by one launch per pass over all views, or for targets above 4096 cells by one sort
over all views) with the plain
frame's arithmetic, so each view's image and survivor count must equal what sk_draw
gives for that view with 16-bit depth keys — bit for bit, not just within tolerance.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

SIZES = [(320, 240), (640, 480), (200, 150), (333, 177), (512, 512)]


def proj_for(width, height):
    return skcam.perspective(math.radians(60.0), width / height, 0.05, 200.0)


def plain(renderer, frame, width, height):
    renderer.resize(width, height)
    renderer.draw(frame)
    image = renderer.read_image(sk.FORMAT_RGBA8)
    return image.copy(), renderer.stats()["draw_count"]


@pytest.fixture(scope="module")
def worlds(cuda_device):
    a = synthetic.random_cloud(120_000, seed=3, sh_degree=3)
    b = synthetic.random_cloud(40_000, seed=4, sh_degree=3, half_extent=6.0)
    rs = []
    for cloud in (a, b):
        r = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
        r.apply_render_policy(sk.Policy(sort_depth_bits=16))
        r.upload_world(cloud, 3)
        rs.append((r, cloud))
    yield rs
    for r, _ in rs:
        r.close()


def views_for(worlds, count, start_frame=0, ranges=None):
    out = []
    for i in range(count):
        r, cloud = worlds[i % len(worlds)]
        w, h = SIZES[i % len(SIZES)]
        view, eye = skcam.orbit_view(start_frame + 11 * i, radius=15.0 if i % 2 == 0 else 9.0)
        rng = ranges[i] if ranges else [(0, cloud.count)]
        out.append(sk.BatchView(r, sk.Frame(view, proj_for(w, h), eye, rng, 3), w, h))
    return out


def check_against_plain(batch, ticket, views):
    for i, v in enumerate(views):
        want, want_visible = plain(v.renderer, v.frame, v.width, v.height)
        got = batch.read_image(ticket, i)
        assert batch.view_visible(ticket, i) == want_visible, f"view {i}"
        assert np.array_equal(got, want), (
            f"view {i}: {np.count_nonzero(got != want)} channels differ, "
            f"max {np.abs(got.astype(int) - want.astype(int)).max()}")


@pytest.mark.gpu
def test_batch_of_two_worlds_and_five_sizes_equals_plain_frames(worlds):
    views = views_for(worlds, 10)
    with sk.Batch(lanes=2, max_views=16) as batch:
        ticket = batch.submit(views)
        batch.wait(ticket)
        stats = batch.stats(ticket)
        assert stats["views"] == 10 and stats["device_error"] == 0
        assert stats["visible"] == sum(batch.view_visible(ticket, i) for i in range(10))
        check_against_plain(batch, ticket, views)


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [False, True])
def test_batch_with_a_view_above_the_direct_cell_limit(worlds, graphs):
    # 2560 x 2048 is 80 x 64 = 5120 binning cells, above the 4096 that lists are written in place
    # for: the whole batch takes the sorted path (emission + stable sort of (cell, splat))
    views = views_for(worlds, 3)
    r, cloud = worlds[0]
    view, eye = skcam.orbit_view(23, radius=15.0)
    views.insert(1, sk.BatchView(r, sk.Frame(view, proj_for(2560, 2048), eye, [(0, cloud.count)], 3),
                                 2560, 2048))
    with sk.Batch(lanes=1, max_views=8, use_graphs=graphs) as batch:
        for _ in range(2 if graphs else 1):  # with graphs: captured, then replayed
            ticket = batch.submit(views)
            batch.wait(ticket)
            check_against_plain(batch, ticket, views)


@pytest.mark.gpu
def test_submissions_in_flight_on_two_lanes(worlds):
    first = views_for(worlds, 4, start_frame=5)
    second = views_for(worlds, 6, start_frame=40,
                       ranges=[[(1000, 30_000)], [(0, 40_000)], [(5, 100_000)], [(0, 20_000)],
                               [(0, 120_000)], [(7, 3)]])
    with sk.Batch(lanes=2, max_views=8) as batch:
        t1 = batch.submit(first)
        t2 = batch.submit(second)  # runs while the first may still be on the device
        batch.wait(t2)
        batch.wait(t1)
        check_against_plain(batch, t1, first)
        check_against_plain(batch, t2, second)
        # a third submission reuses the first lane: its ticket is gone
        t3 = batch.submit(first)
        with pytest.raises(sk.SplatError):
            batch.wait(t1)
        check_against_plain(batch, t3, first)


@pytest.mark.gpu
def test_lanes_grow_while_the_other_lane_draws(worlds):
    # lane buffers grow stream-ordered: each submission is larger than anything its lane held
    # and is enqueued while the other lane's submission is still on the device; all stay exact
    with sk.Batch(lanes=2, max_views=16) as batch:
        tickets, submitted = [], []
        for k, count in enumerate((2, 6, 12, 16)):
            views = views_for(worlds, count, start_frame=20 * k)
            tickets.append(batch.submit(views))
            submitted.append(views)
            if k >= 1:  # the previous submission, on the other lane, before its lane is reused
                check_against_plain(batch, tickets[k - 1], submitted[k - 1])
        check_against_plain(batch, tickets[-1], submitted[-1])


@pytest.mark.gpu
def test_graph_replay_with_new_cameras(worlds):
    with sk.Batch(lanes=1, max_views=8, use_graphs=True) as batch:
        for start in (0, 17, 33):  # same worlds and sizes: captured once, replayed twice
            views = views_for(worlds, 5, start_frame=start)
            ticket = batch.submit(views)
            check_against_plain(batch, ticket, views)


@pytest.mark.gpu
def test_instance_overflow_grows_and_redraws(cuda_device):
    # few large splats close to the camera: far more tile instances than the first guess
    cloud = synthetic.random_cloud(3000, seed=9, sh_degree=3, half_extent=2.0, log_scale_mean=-0.7,
                                   log_scale_std=0.2)
    r = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
    r.apply_render_policy(sk.Policy(sort_depth_bits=16))
    r.upload_world(cloud, 3)
    view, eye = skcam.orbit_view(3, radius=6.0)
    views = [sk.BatchView(r, sk.Frame(view, proj_for(640, 480), eye, [(0, 3000)], 3), 640, 480)]
    with sk.Batch(lanes=1, max_views=4) as batch:
        ticket = batch.submit(views)
        stats = batch.stats(ticket)
        assert stats["instances"] > 4 * 3000
        check_against_plain(batch, ticket, views)
    r.close()


@pytest.mark.gpu
def test_batch_rejects_what_it_cannot_draw(worlds, cuda_device):
    (ra, a), _ = worlds
    low = sk.Renderer(64, 64)
    low.upload_world(synthetic.random_cloud(1000, seed=1, sh_degree=1), 1)
    view, eye = skcam.orbit_view(0)
    with sk.Batch(lanes=1, max_views=2) as batch:
        mixed = [sk.BatchView(ra, sk.Frame(view, proj_for(64, 64), eye, [(0, a.count)], 3), 64, 64),
                 sk.BatchView(low, sk.Frame(view, proj_for(64, 64), eye, [(0, 1000)], 3), 64, 64)]
        with pytest.raises(sk.SplatError) as info:
            batch.submit(mixed)
        assert info.value.status == sk.SK_E_INVALID
        with pytest.raises(sk.SplatError):
            batch.submit(mixed[:1] * 3)  # more than max_views
        with pytest.raises(sk.SplatError):
            batch.submit([sk.BatchView(ra, sk.Frame(view, proj_for(64, 64), eye, [(0, a.count + 1)], 3),
                                       64, 64)])
        with pytest.raises(sk.SplatError):
            batch.apply_render_policy(sk.Policy(sort_depth_bits=32))
        ok = batch.submit(mixed[:1])
        batch.wait(ok)
    low.close()


@pytest.mark.gpu
def test_every_tuning_draws_the_same_images_and_the_tuner_picks_one(worlds):
    views = views_for(worlds, 6, start_frame=21)
    with sk.Batch(lanes=2, max_views=8) as batch:
        for sorted_lists in (0, 1):
            for balanced in (0, 1):
                for tile_keys in (2048, 4096, 6144):
                    batch.set_tuning(balanced, tile_keys, 1, sorted_lists)
                    ticket = batch.submit(views)
                    check_against_plain(batch, ticket, views)
        chosen = batch.autotune(views)
        assert chosen["sorted_lists"] in (0, 1)
        assert chosen["sort_tile_keys"] in (2048, 4096, 6144)
        assert chosen["emission_balanced"] in (0, 1) and 1 <= chosen["lanes"] <= 2
        assert chosen["gpu_ms"] > 0 and chosen["views_per_s"] > 0
        ticket = batch.submit(views)
        check_against_plain(batch, ticket, views)


@pytest.mark.gpu
def test_lod_views_select_their_cuts_in_the_batch(cuda_device):
    """Views of two LOD worlds and a flat one in one submission, graphs asked for (a batch with
    LOD views runs its stages directly): each LOD view's cut is selected on the batch's stream
    with its context's threshold and the view equals sk_draw's frame of that context."""
    policy = sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16)
    renderers = []
    for seed in (81, 82):
        tree = sk.build_lod_tree(synthetic.clustered_cloud(30, 500, seed=seed, half_extent=20.0))
        r = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
        r.apply_render_policy(policy)
        r.upload_lod_world(tree, 0, 4_000_000)
        renderers.append(r)
    flat_cloud = synthetic.random_cloud(25_000, seed=83, sh_degree=0)
    flat = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8)
    flat.apply_render_policy(policy)
    flat.upload_world(flat_cloud, 0)
    views = []
    for i in range(9):
        w, h = SIZES[i % len(SIZES)]
        eye = np.array([-20.0 + 5.0 * i, 2.0, 30.0], np.float32)
        view = skcam.look_at_view(eye, (0.0, 0.0, 0.0))
        if i % 3 == 2:
            frame = sk.Frame(view, proj_for(w, h), eye, [(0, flat_cloud.count)], 0)
            views.append(sk.BatchView(flat, frame, w, h))
        else:
            views.append(sk.BatchView(renderers[i % 3], sk.Frame(view, proj_for(w, h), eye, [], 0), w, h))
    try:
        with sk.Batch(lanes=2, max_views=16, use_graphs=True) as batch:
            for _ in range(2):  # the second submission reuses the lane's LOD buffers
                ticket = batch.submit(views)
                batch.wait(ticket)
                assert batch.stats(ticket)["device_error"] == 0
            check_against_plain(batch, ticket, views)
    finally:
        for r in renderers + [flat]:
            r.close()
