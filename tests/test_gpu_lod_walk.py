"""The LOD workload at full size: 6M leaves (2000 clusters of 3000 splats), the tree built by the
reference's own builder and selection data (LodTree.cpp:308-330, LodSelection.cpp:47-133,
compiled into oracle/_ref), walked at 1920x1080 with a 1.5 px error. The cut, the survivors' keys
and records and the depth order are bit-exact against the oracle, and one frame's image is within
1/255 of the FP64 composite. The same cloud built into a tree on the GPU
(sk_build_lod_tree_device) gives the reference tree's layout and the same cut on every one of the
300 walk frames."""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

from scenes import psnr, tree_from_reference

W, H, FRAMES = 1920, 1080, 300
TOL = 1.0 / 255.0
MIN_PSNR = 50.0
THREADS = os.cpu_count() or 1


def walk_frame(i):
    x = -90.0 + 180.0 * i / (FRAMES - 1)
    eye = np.array([x, 1.7, 0.0], np.float32)
    view = skcam.look_at_view(eye, (x + 10.0, 1.7, 0.0))
    proj = skcam.perspective(math.radians(60.0), W / H, 0.05, 400.0)
    return view, proj, eye


def walk_cloud():
    cloud = synthetic.clustered_cloud(2000, 3000, seed=0)
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min, cloud.bounds_max = pos.min(axis=0), pos.max(axis=0)
    return cloud


@pytest.fixture(scope="module")
def walk_tree(reference):
    return reference.build_lod_tree(walk_cloud())


@pytest.mark.gpu
def test_walk_cuts_and_orders_match_the_oracle(oracle, walk_tree, cuda_device):
    d = walk_tree
    tree = tree_from_reference(d)
    r = sk.Renderer(W, H, image_format=sk.FORMAT_RGBA32F)
    r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
    r.upload_lod_world(tree, 0, 4_000_000)
    packed = sk.pack_splats(tree.nodes)
    for i in (0, 100, 200):
        view, proj, eye = walk_frame(i)
        r.draw(sk.Frame(view, proj, eye, [], 0))
        cut, stats = r.read_cut()
        keys, projected = r.read_visible()
        order = r.read_order()
        assert r.stats()["device_error"] == 0
        cam = oracle.camera(view, proj, eye, W, H, 1.0)
        ocut, _ = oracle.lod_select(cam, d["clusters"], d["leaves"], d["depth"] + 1,
                                    min(4_000_000, d["leaf_count"]), 1.5, 4.0, True)
        assert len(cut) > 10_000
        assert np.array_equal(cut, ocut), f"frame {i}"
        okeys, oproj = oracle.visibility(cam, packed, None, 0, 0, 16, indices=ocut, threads=THREADS)
        assert np.array_equal(keys, okeys), f"frame {i}"
        assert projected.tobytes() == oproj.tobytes(), f"frame {i}"
        oorder = oracle.stable_argsort(okeys)
        assert np.array_equal(order, oorder), f"frame {i}"
        if i == 100:
            image = r.read_image(sk.FORMAT_RGBA32F)
            oimage = oracle.composite(oproj, oorder, W, H, threads=THREADS)
            err = float(np.abs(image.astype(np.float64) - oimage).max())
            p = psnr(image[..., :3], oimage[..., :3])
            print(f"walk frame {i}: cut {len(cut)}, visible {len(keys)}, max abs {err * 255:.3f}/255, "
                  f"PSNR {p:.1f} dB")
            assert err <= TOL and p >= MIN_PSNR
    r.close()


@pytest.mark.gpu
def test_device_tree_build_gives_the_reference_layout_and_cuts(walk_tree, cuda_device):
    """The same 6M-leaf cloud built on the GPU: the layout (child ranges) is the reference
    builder's exactly and node attributes agree within a few ulp; drawn along the whole 300-frame
    walk, each frame's cut (node indices in emission order) equals the reference tree's."""
    d = walk_tree
    gpu = sk.build_lod_tree(walk_cloud())
    assert gpu.leaf_count == d["leaf_count"] and len(gpu.layout) == len(d["layout"])
    np.testing.assert_array_equal(gpu.layout["child_start"], d["layout"]["child_start"])
    np.testing.assert_array_equal(gpu.layout["child_count"], d["layout"]["child_count"])
    pos = np.asarray(gpu.nodes.positions, np.float64)
    ref_pos = d["positions"].astype(np.float64)
    same = np.all(pos == ref_pos, axis=1)
    worst = float(np.abs(pos - ref_pos).max())
    print(f"device tree: {same.mean() * 100:.2f}% of node positions bit-equal, worst {worst:.2e} m")
    np.testing.assert_allclose(pos, ref_pos, rtol=0, atol=1e-4)
    np.testing.assert_array_equal(gpu.clusters["leaf_count"], d["clusters"]["leaf_count"])
    np.testing.assert_array_equal(gpu.leaves, d["leaves"])
    ref_tree = tree_from_reference(d)
    renderers = []
    for tree in (ref_tree, gpu):
        r = sk.Renderer(W, H, image_format=sk.FORMAT_RGBA8)
        r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
        r.upload_lod_world(tree, 0, 4_000_000)
        renderers.append(r)
    differing = []
    for i in range(FRAMES):
        view, proj, eye = walk_frame(i)
        cuts = []
        for r in renderers:
            r.draw(sk.Frame(view, proj, eye, [], 0))
            cuts.append(r.read_cut()[0])
        if not np.array_equal(cuts[0], cuts[1]):
            differing.append(i)
    for r in renderers:
        r.close()
    print(f"walk: {FRAMES - len(differing)} of {FRAMES} cuts identical")
    assert not differing, differing
