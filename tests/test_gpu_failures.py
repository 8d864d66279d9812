"""The error paths, made to fire through the test hooks of include/splatkit_b200_testing.h without
faulting, trapping or hanging the GPU:

  - a bounded device wait that runs out (a depth-sort tile that never publishes its look-back
    status words): the frame reports SK_E_TIMEOUT and the next frame on the same context is right;
  - a failed upload (device allocations made to fail on the host) keeps the previous world,
    transactionally, as the reference's renderer does (MetalFrameCompute.mm:113-139), and does not
    latch the context;
  - a failed CUDA call (a faked status) latches the context failed for good, like the reference's
    failure latch (MetalFrameLoop.h:51-55; SplatEngine.cpp:517-536): every later call returns
    SK_E_DEVICE, while another context keeps drawing."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

pytestmark = pytest.mark.gpu

W, H = 320, 240
CUDA_ERROR_LAUNCH_FAILURE = 719  # cudaErrorLaunchFailure, faked: no kernel fails


def frame_of(cloud, k=5, degree=None):
    view, eye = skcam.orbit_view(k)
    proj = skcam.perspective(math.radians(60.0), W / H, 0.05, 200.0)
    return sk.Frame(view, proj, eye, [(0, cloud.count)], cloud.sh_degree if degree is None else degree)


def test_a_wait_that_runs_out_fails_one_frame_and_the_next_is_right(cuda_device):
    cloud = synthetic.random_cloud(120_000, seed=51, sh_degree=1)  # ~90k survivors: ~22 sort tiles
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F) as r:
        r.apply_render_policy(sk.Policy(sort_depth_bits=32))
        r.upload_world(cloud, 1)
        r.draw(frame_of(cloud))
        want_order, want_image = r.read_order(), r.read_image(sk.FORMAT_RGBA32F)
        assert r.stats()["device_error"] == 0 and len(want_order) > 5 * 4096
        r.testing_withhold_sort_status(3)
        r.draw(frame_of(cloud))
        with pytest.raises(sk.SplatError) as err:
            r.wait_idle()
        assert err.value.status == sk.SK_E_TIMEOUT
        assert r.stats()["device_error"] != 0
        assert not r.gpu_failed()
        # the same context draws the next frame right
        r.draw(frame_of(cloud))
        r.wait_idle()
        assert r.stats()["device_error"] == 0
        assert np.array_equal(r.read_order(), want_order)
        assert r.read_image(sk.FORMAT_RGBA32F).tobytes() == want_image.tobytes()


def test_a_failed_upload_keeps_the_previous_world(cuda_device):
    small = synthetic.random_cloud(30_000, seed=52, sh_degree=0)
    large = synthetic.random_cloud(200_000, seed=53, sh_degree=0)
    with sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F) as r:
        r.upload_world(small, 0)
        r.draw(frame_of(small))
        want = r.read_image(sk.FORMAT_RGBA32F)
        try:
            sk.testing_fail_device_allocations(1)
            with pytest.raises(sk.SplatError) as err:
                r.upload_world(large, 0)
        finally:
            sk.testing_fail_device_allocations(0)
        assert err.value.status == sk.SK_E_OOM
        assert not r.gpu_failed()
        assert r.world() == (small.count, 0)
        r.draw(frame_of(small))
        assert r.read_image(sk.FORMAT_RGBA32F).tobytes() == want.tobytes()
        # and the upload succeeds once memory is there
        r.upload_world(large, 0)
        assert r.world() == (large.count, 0)
        r.draw(frame_of(large))
        assert r.stats()["device_error"] == 0 and r.read_image(sk.FORMAT_RGBA32F).any()


def test_a_failed_call_latches_the_context(cuda_device):
    cloud = synthetic.random_cloud(20_000, seed=54, sh_degree=0)
    with sk.Renderer(W, H) as failing, sk.Renderer(W, H) as other:
        for r in (failing, other):
            r.upload_world(cloud, 0)
        failing.testing_fail_next_check(CUDA_ERROR_LAUNCH_FAILURE)
        with pytest.raises(sk.SplatError) as err:
            failing.draw(frame_of(cloud))
            failing.wait_idle()
        assert err.value.status == sk.SK_E_DEVICE
        assert failing.gpu_failed()
        for call in (lambda: failing.draw(frame_of(cloud)), failing.wait_idle,
                     lambda: failing.upload_world(cloud, 0), lambda: failing.resize(64, 64)):
            with pytest.raises(sk.SplatError) as again:
                call()
            assert again.value.status == sk.SK_E_DEVICE
        # the latch is the context's: another context keeps drawing
        other.draw(frame_of(cloud))
        assert other.read_image().any() and not other.gpu_failed()
