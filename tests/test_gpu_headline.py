"""Parity at the benchmark's own workload: the 1M-splat SH3 scene (PCG64 seed 0) at 1920x1080 on
the 120-frame orbit (radius 15 m, 3 degrees per frame), frames 0, 37 and 90, with 16- and
32-bit depth keys, through the C ABI exactly as bench.py draws it. Survivors, depth keys,
projected records and the depth order are bit-exact against the oracle (its restatement of
SplatProjection.metalh:78-141 and SplatVisibility.metal:16-106, and a stable sort, the
reference's own sort oracle in MetalRadixSortTest.mm:58-62); the image is within 1/255 per
channel of the FP64 composite of SplatRaster.metal:27-44 / MetalSplatPipeline.mm:46-71,153-161,
with PSNR >= 50 dB.

Also pinned against the oracle here: a 3840x2160 target (more than 4096 binning cells, so the
cell lists take the stable-sort path) and a 2560x1440 one, which the serving mix draws."""
from __future__ import annotations

import math
import os
import time

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

from scenes import psnr

pytestmark = pytest.mark.gpu

TOL = 1.0 / 255.0  # image tolerance, max abs per channel
MIN_PSNR = 50.0    # dB against the FP64 composite
SPLATS, SH = 1_000_000, 3
THREADS = os.cpu_count() or 1


def orbit(frame, width, height):
    view, eye = skcam.orbit_view(frame, radius=15.0, degrees_per_frame=3.0)
    proj = skcam.perspective(math.radians(60.0), width / height, 0.05, 200.0)
    return view, proj, eye


@pytest.fixture(scope="module")
def scene():
    cloud = synthetic.random_cloud(SPLATS, seed=0, sh_degree=SH)
    return cloud, sk.pack_splats(cloud), sk.pack_sh(cloud, SH)


def draw(r, cloud, view, proj, eye):
    r.draw(sk.Frame(view, proj, eye, [(0, cloud.count)], SH))
    keys, projected = r.read_visible()
    order = r.read_order()
    image = r.read_image(sk.FORMAT_RGBA32F)
    return keys, projected, order, image, r.stats()


def check(oracle, scene, r, frame, bits, width, height, label):
    cloud, packed, sh = scene
    view, proj, eye = orbit(frame, width, height)
    t0 = time.perf_counter()
    keys, projected, order, image, stats = draw(r, cloud, view, proj, eye)
    t1 = time.perf_counter()
    cam = oracle.camera(view, proj, eye, width, height, 1.0)
    okeys, oproj = oracle.visibility(cam, packed, sh, sk.sh_device_stride(SH), SH, bits,
                                     [(0, cloud.count)], threads=THREADS)
    oorder = oracle.stable_argsort(okeys)
    oimage = oracle.composite(oproj, oorder, width, height, threads=THREADS)
    t2 = time.perf_counter()
    assert stats["device_error"] == 0, label
    assert len(keys) == len(okeys) > 0, label
    assert np.array_equal(keys, okeys), label
    assert projected.tobytes() == oproj.tobytes(), label
    assert np.array_equal(order, oorder), label
    err = float(np.abs(image.astype(np.float64) - oimage).max())
    p = psnr(image[..., :3], oimage[..., :3])
    print(f"{label}: visible {len(keys)}, list entries {stats['instances']}, max abs "
          f"{err * 255:.3f}/255, PSNR {p:.1f} dB (gpu {t1 - t0:.2f} s, oracle {t2 - t1:.2f} s on "
          f"{THREADS} threads)")
    assert err <= TOL, label
    assert p >= MIN_PSNR, label


@pytest.mark.parametrize("bits", [16, 32])
def test_headline_frames_match_the_oracle(oracle, scene, cuda_device, bits):
    cloud = scene[0]
    with sk.Renderer(1920, 1080, image_format=sk.FORMAT_RGBA32F) as r:
        r.apply_render_policy(sk.Policy(sort_depth_bits=bits))
        r.upload_world(cloud, SH)
        for frame in (0, 37, 90):
            check(oracle, scene, r, frame, bits, 1920, 1080, f"1M SH3 1080p frame {frame} {bits}-bit")


@pytest.mark.parametrize("width,height", [(3840, 2160), (2560, 1440)])
def test_large_targets_match_the_oracle(oracle, scene, cuda_device, width, height):
    """3840x2160 has 8160 binning cells: its lists come from the stable sort of (cell, splat)
    pairs, which no smaller target takes; 2560x1440 has 3680 and is written in place."""
    cloud = scene[0]
    with sk.Renderer(width, height, image_format=sk.FORMAT_RGBA32F) as r:
        r.apply_render_policy(sk.Policy(sort_depth_bits=16))
        r.upload_world(cloud, SH)
        check(oracle, scene, r, 11, 16, width, height, f"1M SH3 {width}x{height} frame 11")
