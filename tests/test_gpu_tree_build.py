"""The LOD tree built on the GPU (sk_build_lod_tree_device) against the reference's own builder
(LodTree.cpp:17-344, compiled into oracle/_ref) given the same bounds: the same layout exactly,
node attributes within a few ulp (the device's acos/cos and powf are not the host library's),
the same selection structure, and a drawn image within 2/255."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

from scenes import tree_from_reference

pytestmark = pytest.mark.gpu


def bounded(cloud):
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min = pos.min(axis=0) - 0.25
    cloud.bounds_max = pos.max(axis=0) + 0.25
    return cloud


def duplicated(n: int, copies: int, seed: int):
    """Every splat repeated `copies` times: ranges of one Morton key that merge at the depth limit."""
    base = synthetic.random_cloud(n, seed=seed, sh_degree=1, half_extent=3.0)
    rep = lambda a: None if a is None else np.repeat(np.asarray(a), copies, axis=0)
    return sk.Cloud(rep(base.positions), rep(base.covariances), rep(base.colors), rep(base.alphas),
                    sh_degree=1, sh=rep(base.sh))


# every cloud carries bounds: the reference builder takes a cloud's bounds as they are
CLOUDS = {
    "random_sh3": lambda: bounded(synthetic.random_cloud(20000, seed=21, sh_degree=3, half_extent=4.0)),
    "random_sh0": lambda: bounded(synthetic.random_cloud(7000, seed=22, sh_degree=0, half_extent=9.0)),
    "clustered_80k": lambda: bounded(synthetic.clustered_cloud(80, 1000, seed=14, half_extent=50.0)),
    "duplicates": lambda: bounded(duplicated(500, 40, seed=23)),
    "one": lambda: bounded(synthetic.random_cloud(1, seed=24, sh_degree=2)),
    "two": lambda: bounded(synthetic.random_cloud(2, seed=25, sh_degree=2)),
}


def assert_same_tree(gpu: sk.LodTree, host: sk.LodTree):
    """host: the reference builder's tree."""
    assert gpu.leaf_count == host.leaf_count
    assert len(gpu.layout) == len(host.layout)
    np.testing.assert_array_equal(gpu.layout["child_start"], host.layout["child_start"])
    np.testing.assert_array_equal(gpu.layout["child_count"], host.layout["child_count"])
    # attributes: relative 1e-4 of each array's scale (a few ulp through the merges)
    for name in ("positions", "covariances", "colors", "alphas"):
        a = np.asarray(getattr(gpu.nodes, name), np.float64)
        b = np.asarray(getattr(host.nodes, name), np.float64)
        scale = max(np.abs(b).max(), 1e-30)
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-5 * scale, err_msg=name)
    np.testing.assert_allclose(gpu.layout["size"], host.layout["size"], rtol=1e-4,
                               atol=1e-5 * float(np.abs(host.layout["size"]).max()))
    np.testing.assert_array_equal(gpu.layout["position"], gpu.nodes.positions)
    if host.nodes.sh is None:
        assert gpu.nodes.sh is None
    else:
        scale = float(np.abs(host.nodes.sh).max())
        np.testing.assert_allclose(gpu.nodes.sh, host.nodes.sh, rtol=1e-4, atol=1e-5 * scale)
    # leaves copy their splat unchanged
    leaf = host.layout["child_count"] == 0
    assert gpu.nodes.positions[leaf].tobytes() == host.nodes.positions[leaf].tobytes()
    assert gpu.nodes.alphas[leaf].tobytes() == host.nodes.alphas[leaf].tobytes()


@pytest.mark.parametrize("name", sorted(CLOUDS))
@pytest.mark.parametrize("depth,leaves", [(0, 0), (6, 8), (3, 64), (2, 2)])
def test_device_build_matches_the_reference_build(reference, name, depth, leaves, cuda_device):
    cloud = CLOUDS[name]()
    d = reference.build_lod_tree(cloud, octree_depth=depth, cluster_leaves=leaves)
    ref = tree_from_reference(d)
    gpu = sk.build_lod_tree(cloud, octree_depth=depth, cluster_leaves=leaves)
    assert_same_tree(gpu, ref)
    assert sk.lod_depth(gpu.layout, gpu.leaf_count) == d["depth"]
    assert len(gpu.clusters) == len(d["clusters"])
    for field in ("node", "child_start", "child_count", "leaf_start", "leaf_count", "subtree_leaves"):
        np.testing.assert_array_equal(gpu.clusters[field], d["clusters"][field], err_msg=field)
    np.testing.assert_array_equal(gpu.leaves, d["leaves"])


def test_device_built_tree_draws_like_the_reference_tree(reference, cuda_device):
    cloud = bounded(synthetic.clustered_cloud(60, 800, seed=31, half_extent=20.0))
    ref = tree_from_reference(reference.build_lod_tree(cloud))
    gpu = sk.build_lod_tree(cloud)
    view = skcam.look_at_view(np.array([0.0, 5.0, 45.0], np.float32), (0.0, 0.0, 0.0))
    proj = skcam.perspective(math.radians(60.0), 320 / 240, 0.05, 400.0)
    images = []
    for tree in (ref, gpu):
        r = sk.Renderer(320, 240, image_format=sk.FORMAT_RGBA8)
        r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
        r.upload_lod_world(tree, 0, 100_000)
        r.draw(sk.Frame(view, proj, np.array([0.0, 5.0, 45.0], np.float32), [], 0))
        assert r.stats()["device_error"] == 0
        images.append(r.read_image().astype(np.int32))
        r.close()
    assert np.abs(images[0] - images[1]).max() <= 2
    assert images[0].any()


def test_tree_arrays_are_read_only_views_that_keep_the_tree_alive(cuda_device):
    import gc
    import weakref
    tree = sk.build_lod_tree(bounded(synthetic.random_cloud(5000, seed=11, sh_degree=2, half_extent=4.0)))
    expected = tree.nodes.positions.copy()
    owner = weakref.ref(tree.layout.base._owner)
    assert not tree.nodes.positions.flags["OWNDATA"]
    assert not tree.nodes.positions.flags["WRITEABLE"]  # the memory is the library's
    positions = tree.nodes.positions
    del tree
    gc.collect()
    assert owner() is not None  # one view is left
    np.testing.assert_array_equal(positions, expected)
    del positions
    gc.collect()
    assert owner() is None  # freed with the last view
