"""LOD selection data (sk_build_lod_selection, host/selection.cpp) and the .lodsplat writer
(sk_write_lodsplat) against the reference's own buildLodSelectionData (LodSelection.cpp:47-133)
and writeLodSplat (LodFile.cpp:425-458), on trees the reference's builder made: the same
clusters, leaf references and file, bit for bit (CPU only)."""
from __future__ import annotations

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import synthetic

from scenes import hierarchy_cloud, layout_tree, tree_from_reference, uniform_nodes


def bounded(cloud):
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min = pos.min(axis=0) - 0.25
    cloud.bounds_max = pos.max(axis=0) + 0.25
    return cloud


def repeated(cloud, copies: int):
    rep = lambda a: None if a is None else np.repeat(np.asarray(a), copies, axis=0)
    return sk.Cloud(rep(cloud.positions), rep(cloud.covariances), rep(cloud.colors), rep(cloud.alphas),
                    sh_degree=cloud.sh_degree, sh=rep(cloud.sh))


CLOUDS = {
    "grid": lambda: hierarchy_cloud(),
    "random_sh1": lambda: bounded(synthetic.random_cloud(4000, seed=10, sh_degree=1, half_extent=4.0)),
    "random_sh2": lambda: bounded(synthetic.random_cloud(5000, seed=11, sh_degree=2, half_extent=4.0)),
    "random_sh3": lambda: bounded(synthetic.random_cloud(3000, seed=12, sh_degree=3, half_extent=2.0)),
    "clustered": lambda: bounded(synthetic.clustered_cloud(12, 400, seed=13, half_extent=30.0)),
    # edge cases: a root that is its one splat, a root of two, every splat repeated (one Morton
    # key per run, merged at the depth limit)
    "one": lambda: bounded(synthetic.random_cloud(1, seed=24, sh_degree=2)),
    "two": lambda: bounded(synthetic.random_cloud(2, seed=25, sh_degree=2)),
    "duplicates": lambda: bounded(repeated(synthetic.random_cloud(300, seed=23, sh_degree=1, half_extent=3.0), 40)),
}


def without_selection(d: dict) -> sk.LodTree:
    return tree_from_reference({**d, "clusters": np.zeros(0, sk.LOD_CLUSTER_DTYPE),
                                "leaves": np.zeros(0, np.uint32)})


def assert_selection_is_the_reference_selection(d: dict):
    clusters, leaves = sk.build_lod_selection(without_selection(d))
    assert len(clusters) == len(d["clusters"]) and len(leaves) == len(d["leaves"])
    for field in ("node", "child_start", "child_count", "leaf_start", "leaf_count", "subtree_leaves"):
        np.testing.assert_array_equal(clusters[field], d["clusters"][field], err_msg=field)
    np.testing.assert_array_equal(leaves, d["leaves"])
    assert clusters.tobytes() == d["clusters"].tobytes()


@pytest.mark.parametrize("name", sorted(CLOUDS))
@pytest.mark.parametrize("depth,leaves", [(0, 0), (6, 8), (3, 64)])
def test_selection_matches_the_reference_selection(reference, name, depth, leaves):
    d = reference.build_lod_tree(CLOUDS[name](), octree_depth=depth, cluster_leaves=leaves)
    assert_selection_is_the_reference_selection(d)


def test_selection_of_hand_made_trees(reference):
    """Trees the builder would not make: a chain, a wide root of 513 leaves, a root of one leaf."""
    cases = [
        (layout_tree(5, lambda i: (1, 2) if i == 0 else ((3, 2) if i == 2 else (0, 0))), 3),
        (layout_tree(514, lambda i: (1, 513) if i == 0 else (0, 0)), 513),
        (layout_tree(7, lambda i: (i + 1, 1) if i < 3 else ((4, 3) if i == 3 else (0, 0))), 3),
    ]
    for lay, leaf_count in cases:
        d = reference.make_tree(uniform_nodes(len(lay)), lay, leaf_count)
        assert_selection_is_the_reference_selection(d)


def test_selection_refuses_a_layout_that_is_not_breadth_first(reference):
    lay = layout_tree(5, lambda i: (1, 2) if i == 0 else ((3, 2) if i == 2 else (0, 0)))
    lay[0]["child_start"] = 2
    with pytest.raises(sk.SplatError) as err:
        sk.build_lod_selection(sk.LodTree(uniform_nodes(5), lay, 3))
    assert err.value.status == sk.SK_E_INVALID


def test_selection_of_a_tree_split_over_host_threads_is_the_reference_selection(reference):
    """~540k nodes: the topology is ranked in several host-thread slices of the layout (and of the
    clusters), the levels' clusters finished on several threads; clusters and leaf references stay
    the reference's bit for bit."""
    d = reference.build_lod_tree(bounded(synthetic.clustered_cloud(160, 3000, seed=15, half_extent=60.0)))
    assert len(d["layout"]) > 4 * 65536 and len(d["clusters"]) > 2 * 16384
    assert_selection_is_the_reference_selection(d)


@pytest.mark.parametrize("selection", [True, False])
def test_written_file_is_the_reference_file(reference, tmp_path, selection):
    cloud = CLOUDS["random_sh2"]()
    d = reference.write_lodsplat(cloud, tmp_path / "ref.lodsplat", selection=selection)
    ours = tree_from_reference(d)
    ours.nodes.bounds_min, ours.nodes.bounds_max = cloud.bounds_min, cloud.bounds_max
    sk.write_lodsplat(ours, tmp_path / "ours.lodsplat")
    assert (tmp_path / "ours.lodsplat").read_bytes() == (tmp_path / "ref.lodsplat").read_bytes()
    with pytest.raises(sk.SplatError):  # never overwrites
        sk.write_lodsplat(ours, tmp_path / "ours.lodsplat")
    assert d["depth"] == sk.lodsplat_header((tmp_path / "ours.lodsplat").read_bytes())["depth"]
