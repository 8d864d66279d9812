"""The LOD workload at full size: 6M leaves (2000 clusters of 3000 splats), the tree built on the
host (the reference builder's tree bit for bit), walked at 1920x1080 with a 1.5 px error. The cut,
the survivors' keys and records and the depth order are bit-exact against the oracle."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

W, H, FRAMES = 1920, 1080, 300


def walk_frame(i):
    x = -90.0 + 180.0 * i / (FRAMES - 1)
    eye = np.array([x, 1.7, 0.0], np.float32)
    view = skcam.look_at_view(eye, (x + 10.0, 1.7, 0.0))
    proj = skcam.perspective(math.radians(60.0), W / H, 0.05, 400.0)
    return view, proj, eye


@pytest.fixture(scope="module")
def walk_tree(cuda_device):
    cloud = synthetic.clustered_cloud(2000, 3000, seed=0)
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min, cloud.bounds_max = pos.min(axis=0), pos.max(axis=0)
    return sk.build_lod_tree(cloud)


@pytest.mark.gpu
def test_walk_cuts_and_orders_match_the_oracle(oracle, walk_tree):
    tree = walk_tree
    depth = sk.lod_depth(tree.layout, tree.leaf_count)
    r = sk.Renderer(W, H, image_format=sk.FORMAT_RGBA8)
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
        ocut, _ = oracle.lod_select(cam, tree.clusters, tree.leaves, depth + 1,
                                    min(4_000_000, tree.leaf_count), 1.5, 4.0, True)
        assert len(cut) > 10_000
        assert np.array_equal(cut, ocut), f"frame {i}"
        okeys, oproj = oracle.visibility(cam, packed, None, 0, 0, 16, indices=ocut, threads=16)
        assert np.array_equal(keys, okeys), f"frame {i}"
        assert projected.tobytes() == oproj.tobytes(), f"frame {i}"
        assert np.array_equal(order, oracle.stable_argsort(okeys)), f"frame {i}"
    r.close()


@pytest.mark.gpu
def test_device_tree_build_has_the_host_layout(walk_tree):
    """The same 6M-leaf tree built on the GPU (sk_build_lod_tree_device): the layout is the host
    builder's exactly, attributes to a few ulp."""
    cloud = synthetic.clustered_cloud(2000, 3000, seed=0)
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min, cloud.bounds_max = pos.min(axis=0), pos.max(axis=0)
    gpu = sk.build_lod_tree(cloud, device=True)
    host = walk_tree
    assert gpu.leaf_count == host.leaf_count and len(gpu.layout) == len(host.layout)
    np.testing.assert_array_equal(gpu.layout["child_start"], host.layout["child_start"])
    np.testing.assert_array_equal(gpu.layout["child_count"], host.layout["child_count"])
    np.testing.assert_allclose(gpu.nodes.positions, host.nodes.positions, rtol=1e-4, atol=1e-3)
    np.testing.assert_allclose(gpu.layout["size"], host.layout["size"], rtol=1e-3, atol=1e-5)
    np.testing.assert_array_equal(gpu.clusters["leaf_count"], host.clusters["leaf_count"])
    np.testing.assert_array_equal(gpu.leaves, host.leaves)
