"""The host LOD tree builder (sk_build_lod_tree, subtrees built on all host threads) and .lodsplat
writer against the reference's own
builder and writer: the same tree, selection data and file, bit for bit (CPU only)."""
from __future__ import annotations

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import synthetic

from scenes import hierarchy_cloud


def bounded(cloud):
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min = pos.min(axis=0) - 0.25
    cloud.bounds_max = pos.max(axis=0) + 0.25
    return cloud


CLOUDS = {
    "grid": lambda: hierarchy_cloud(),
    "random_sh2": lambda: bounded(synthetic.random_cloud(5000, seed=11, sh_degree=2, half_extent=4.0)),
    "random_sh3": lambda: bounded(synthetic.random_cloud(3000, seed=12, sh_degree=3, half_extent=2.0)),
    "clustered": lambda: bounded(synthetic.clustered_cloud(12, 400, seed=13, half_extent=30.0)),
    # enough leaves for hundreds of subtrees built on separate threads
    "clustered_80k": lambda: bounded(synthetic.clustered_cloud(80, 1000, seed=14, half_extent=50.0)),
    # edge cases: a root that is its one splat, a root of two, every splat repeated (one Morton
    # key per run, merged at the depth limit). Bounds given, as a loader gives them: the
    # reference builder takes the cloud's bounds as they are (zero when unset), this build the
    # positions' own box when none are passed.
    "one": lambda: bounded(synthetic.random_cloud(1, seed=24, sh_degree=2)),
    "two": lambda: bounded(synthetic.random_cloud(2, seed=25, sh_degree=2)),
    "duplicates": lambda: bounded(repeated(synthetic.random_cloud(300, seed=23, sh_degree=1, half_extent=3.0), 40)),
}


def repeated(cloud, copies: int):
    rep = lambda a: None if a is None else np.repeat(np.asarray(a), copies, axis=0)
    return sk.Cloud(rep(cloud.positions), rep(cloud.covariances), rep(cloud.colors), rep(cloud.alphas),
                    sh_degree=cloud.sh_degree, sh=rep(cloud.sh))


def assert_tree_equals(ours: sk.LodTree, ref: dict):
    n = len(ref["layout"])
    assert len(ours.layout) == n and ours.leaf_count == ref["leaf_count"]
    assert ours.layout.tobytes() == np.ascontiguousarray(ref["layout"]).tobytes()
    for name, got in (("positions", ours.nodes.positions), ("covariances", ours.nodes.covariances),
                      ("colors", ours.nodes.colors), ("alphas", ours.nodes.alphas)):
        assert np.asarray(got, np.float32).tobytes() == np.asarray(ref[name], np.float32).tobytes(), name
    if ref["sh"] is None:
        assert ours.nodes.sh is None
    else:
        assert ours.nodes.sh.tobytes() == np.asarray(ref["sh"], np.float32).tobytes()
    if ref["clusters"] is not None and len(ref["clusters"]):
        assert ours.clusters.tobytes() == np.ascontiguousarray(ref["clusters"]).tobytes()
        np.testing.assert_array_equal(ours.leaves, ref["leaves"])


@pytest.mark.parametrize("name", sorted(CLOUDS))
@pytest.mark.parametrize("depth,leaves", [(0, 0), (6, 8), (3, 64)])
def test_builder_matches_the_reference_builder(reference, name, depth, leaves):
    cloud = CLOUDS[name]()
    ours = sk.build_lod_tree(cloud, octree_depth=depth, cluster_leaves=leaves)
    ref = reference.build_lod_tree(cloud, octree_depth=depth, cluster_leaves=leaves)
    assert_tree_equals(ours, ref)
    assert sk.lod_depth(ours.layout, ours.leaf_count) == ref["depth"]


@pytest.mark.parametrize("selection", [True, False])
def test_written_file_is_the_reference_file(reference, tmp_path, selection):
    cloud = CLOUDS["random_sh2"]()
    ref = reference.write_lodsplat(cloud, tmp_path / "ref.lodsplat", selection=selection)
    ours = sk.build_lod_tree(cloud, selection=selection)
    sk.write_lodsplat(ours, tmp_path / "ours.lodsplat")
    assert (tmp_path / "ours.lodsplat").read_bytes() == (tmp_path / "ref.lodsplat").read_bytes()
    with pytest.raises(sk.SplatError):  # never overwrites
        sk.write_lodsplat(ours, tmp_path / "ours.lodsplat")
    assert ref["depth"] == sk.lodsplat_header((tmp_path / "ours.lodsplat").read_bytes())["depth"]


def test_tree_arrays_are_views_that_keep_the_tree_alive():
    import gc
    import weakref
    cloud = CLOUDS["random_sh2"]()
    tree = sk.build_lod_tree(cloud)
    expected = tree.nodes.positions.copy()
    owner = weakref.ref(tree.layout.base._owner)
    assert not tree.nodes.positions.flags["OWNDATA"]
    positions = tree.nodes.positions
    del tree
    gc.collect()
    assert owner() is not None  # one view is left
    np.testing.assert_array_equal(positions, expected)
    del positions
    gc.collect()
    assert owner() is None  # freed with the last view


def test_selection_of_a_tree_split_over_host_threads_is_the_reference_selection(reference):
    """~540k nodes: the selection structure is ranked in several host-thread slices of the layout
    (and of the clusters); clusters, leaf references and layout stay the reference's bit for bit."""
    cloud = bounded(synthetic.clustered_cloud(160, 3000, seed=15, half_extent=60.0))
    ours = sk.build_lod_tree(cloud)
    ref = reference.build_lod_tree(cloud)
    assert len(ours.layout) > 4 * 65536 and len(ours.clusters) > 2 * 16384
    assert_tree_equals(ours, ref)
