"""The CPU oracle against the reference's own known-answer tests (CPU only).

Each case rebuilds a scene from the reference's Metal tests and checks the oracle reproduces
the expected answer those tests assert. This pins the oracle before any GPU result is
compared with it."""
from __future__ import annotations

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam

from scenes import (hierarchy_cloud, identity, layout_tree, leaves_under, lod_camera,
                    three_splats, tree_from_reference, uniform_nodes, unit_cov_splats)


def ref_camera(oracle, view=None, proj=None, width=1000, height=1000, minpx=0.0, focal=500.0,
               tan=1.0, cam_pos=(0, 0, 0)):
    """The visibility tests' hand-set uniform: focal 500, tanHalfFov 1 over 1000 px
    (MetalVisibilityPassTest.mm:110-121)."""
    view = identity() if view is None else view
    proj = skcam.perspective(1.0, 1.0, 0.1, 100.0) if proj is None else proj
    cam = oracle.camera(view, proj, cam_pos, width, height, minpx)
    cam.focal[0] = cam.focal[1] = focal
    cam.tanHalfFov[0] = cam.tanHalfFov[1] = tan
    return cam


def visible_sorted(oracle, cam, splats, ranges, key_bits=32, sh=None, degree=0, stride=0):
    keys, proj = oracle.visibility(cam, splats, sh, stride, degree, key_bits, ranges)
    order = oracle.stable_argsort(keys)
    return keys, proj, order


# ---- visibility (MetalVisibilityPassTest.mm) ----------------------------------------------
def test_culls_and_orders_ranges_front_to_back(oracle):
    # :205-263
    positions = [[0, 0, -10], [0, 0, 5], [0, 0, -2], [50, 0, -1], [0, 0, -5], [0, 0, -3]]
    splats = unit_cov_splats(positions)
    cam = ref_camera(oracle)
    keys, proj, order = visible_sorted(oracle, cam, splats, [(0, 3), (3, 2)])
    assert len(keys) == 3
    assert list(proj["index"][order]) == [2, 4, 0]


def test_drops_subpixel_gaussian(oracle):
    # :265-300
    splats = unit_cov_splats([[0, 0, -2], [0, 0, -2]])
    splats["cov"][1] = [np.float16(1e-8).view(np.uint16), np.uint32(np.float16(1e-8).view(np.uint16)) << 16,
                        np.uint32(np.float16(1e-8).view(np.uint16)) << 16]
    cam = ref_camera(oracle, minpx=0.5)
    keys, _, _ = visible_sorted(oracle, cam, splats, [(0, 2)])
    assert len(keys) == 1


@pytest.mark.parametrize("cutoff,kept", [(0.5, 1), (1.0, 0)])
def test_keeps_only_splats_at_or_over_cutoff(oracle, cutoff, kept):
    # :302-333: sigma 0.3 px at depth 20, 2.5 sigma quad = 0.75 px footprint
    splats = unit_cov_splats([[0, 0, -20]], variance=1.44e-4)
    cam = ref_camera(oracle, minpx=cutoff)
    keys, _, _ = visible_sorted(oracle, cam, splats, [(0, 1)])
    assert len(keys) == kept


def test_keeps_edge_crossing_quad_and_culls_transparent(oracle):
    # :335-372
    cam = ref_camera(oracle)
    edge = 2.0 / float(cam.proj[0])
    cases = [(1.25 * edge, 0.3, 0xFFFFFFFF), (1.25 * edge, 0.05, 0xFFFFFFFF),
             (0.0, 0.1, 0x00FFFFFF), (0.0, 0.1, 0xFFFFFFFF)]
    splats = np.concatenate([unit_cov_splats([[c, 0, -2]], rgba8=r, variance=s * s)
                             for c, s, r in cases])
    keys, proj, _ = visible_sorted(oracle, cam, splats, [(0, 4)])
    assert sorted(proj["index"]) == [0, 3]


def test_culls_by_footprint_and_depth_planes_and_caps_radius(oracle):
    # :374-423
    cam = ref_camera(oracle, minpx=1.0)
    two = 0x40000000
    cases = [(-2.0, 0.0024, 0xFFFFFFFF, 0), (-2.0, 0.0008, 0xFFFFFFFF, 0),
             (-0.05, 0.1, 0xFFFFFFFF, 0), (-150.0, 1.0, 0xFFFFFFFF, 0),
             (-2.0, 0.1, 0x00000000, two), (-2.0, 1.6, 0xFFFFFFFF, 0)]
    splats = np.concatenate([unit_cov_splats([[0, 0, z]], rgba8=r, variance=s * s, lod_alpha=l)
                             for z, s, r, l in cases])
    keys, proj, _ = visible_sorted(oracle, cam, splats, [(0, 6)])
    assert sorted(proj["index"]) == [0, 4, 5]
    huge = proj[proj["index"] == 5][0]
    assert abs(float(huge["radius"]) - 512.0 / 400.0) <= 0.02


def test_sixteen_bit_keys_quantize_relative_depth(oracle):
    # :427-493
    z_near = 0.05
    proj = skcam.perspective(1.0, 1.0, z_near, 200.0)
    view = identity()
    view[14] = -10
    depths = [150, 2.0002, 2.0001, 0.4003, 0.4002, 0.06, 199, 250, -1]
    splats = unit_cov_splats([[0, 0, 10 - d] for d in depths])
    cam = ref_camera(oracle, view=view, proj=proj, cam_pos=(0, 0, 10))
    expected = [5, 4, 3, 1, 2, 0, 6]

    def rel_key(depth):
        bits = lambda f: int(np.array([f], np.float32).view(np.uint32)[0])  # noqa: E731
        return min((bits(depth) - bits(z_near)) >> 11, 65535)

    for indexed in (False, True):
        if indexed:
            keys, pr = oracle.visibility(cam, splats, None, 0, 0, 16, indices=np.arange(9))
        else:
            keys, pr = oracle.visibility(cam, splats, None, 0, 0, 16, [(0, 9)])
        order = oracle.stable_argsort(keys)
        assert len(keys) == 7
        assert list(pr["index"][order]) == expected
        sk_sorted = np.sort(keys)
        for i in range(7):
            assert abs(int(sk_sorted[i]) - rel_key(depths[expected[i]])) <= 1
        assert sk_sorted[1] < sk_sorted[2]
        assert sk_sorted[3] == sk_sorted[4]
        assert sk_sorted[6] < 65535


def test_compacts_simd_tails(oracle):
    # :495-537: every third splat behind the camera
    positions = np.zeros((513, 3), np.float32)
    positions[:, 2] = -2
    positions[::3, 2] = 2
    splats = unit_cov_splats(positions)
    cam = ref_camera(oracle)
    for n in (1, 31, 32, 33, 255, 256, 257, 513, 0):
        keys, proj = oracle.visibility(cam, splats, None, 0, 0, 32, [(0, n)] if n else [])
        assert len(keys) == n - (n + 2) // 3
        assert all(i % 3 != 0 for i in proj["index"])
        assert len(set(proj["index"])) == len(keys)


# ---- frame compute (MetalFrameComputeTest.mm) --------------------------------------------
@pytest.mark.parametrize("bits", [32, 16])
def test_flat_world_orders_front_to_back(oracle, reference, bits):
    # :168-214: three splats -> {2, 0, 1}
    cloud = three_splats()
    packed = reference.pack_splats(cloud)
    proj = skcam.perspective(1.0, 1.0, 0.1, 100.0)
    cam = oracle.camera(identity(), proj, (0, 0, 0), 64, 64, 1.0)
    keys, pr = oracle.visibility(cam, packed, None, 0, 0, bits, [(0, 3)])
    order = oracle.stable_argsort(keys)
    assert list(pr["index"][order]) == [2, 0, 1]


# ---- sort (MetalRadixSortTest.mm:81-140) --------------------------------------------------
def ref_pairs(oracle, n, mask, seed):
    return oracle.mt19937(seed, n) & np.uint32(mask)


@pytest.mark.parametrize("n,mask,seed", [(1000003, 0xFFFFFFFF, 1), (70000, 0x7, 2),
                                         (4096, 0xFFFFFFFF, 4), (17, 0xFFFFFFFF, 3)])
def test_radix_matches_stable_sort(oracle, n, mask, seed):
    keys = ref_pairs(oracle, n, mask, seed)
    expected = oracle.stable_argsort(keys)
    assert np.array_equal(expected, np.argsort(keys, kind="stable"))
    bits = 16 if mask <= 0xFFFF else 32
    assert np.array_equal(oracle.radix_argsort(keys, bits, threads=4), expected)


def test_two_pass_keys_with_ties_and_tails(oracle):
    for n in (0, 1, 31, 32, 33, 4095, 4096, 4097, 1000003):
        keys = ref_pairs(oracle, n, 0xFFFF, 16)
        if n > 1:
            keys[0], keys[-1] = 65535, 0
        expected = oracle.stable_argsort(keys)
        assert np.array_equal(oracle.radix_argsort(keys, 16, threads=3), expected)
        assert np.array_equal(oracle.radix_argsort(keys, 32, threads=2), expected)


# ---- LOD selection (MetalLodSelectionTest.mm) ---------------------------------------------
def lod_cam(oracle, distance=0.0):
    view, proj, pos = lod_camera(distance)
    cam = oracle.camera(view, proj, pos, 1000, 1000, 0.0)
    cam.focal[0] = cam.focal[1] = 500.0
    cam.tanHalfFov[0] = cam.tanHalfFov[1] = 1.0
    return cam


@pytest.fixture(scope="module")
def hierarchy(reference):
    return reference.build_lod_tree(hierarchy_cloud(), octree_depth=6)


def select(oracle, tree, cam, capacity, pixel_limit, color_weight=4.0, cull=True):
    capacity = min(capacity, 4000000, tree["leaf_count"])
    return oracle.lod_select(cam, tree["clusters"], tree["leaves"], tree["depth"] + 1, capacity,
                             pixel_limit, color_weight, cull)


def test_budget_cuts_cover_every_leaf_once(oracle, hierarchy):
    # :80-102
    for budget in (1, 7, 31, 32, 33, 64, 257, 400, 515):
        cut, _ = select(oracle, hierarchy, lod_cam(oracle), budget, 0.0)
        again, _ = select(oracle, hierarchy, lod_cam(oracle), budget, 0.0)
        assert np.array_equal(cut, again)
        assert 0 < len(cut) <= budget
        represented = []
        for node in cut:
            leaves_under(hierarchy["layout"], int(node), represented)
        assert len(represented) == hierarchy["leaf_count"]
        assert len(set(represented)) == hierarchy["leaf_count"]
        if budget == 515:
            assert len(cut) == 515


def test_distance_changes_cut(oracle, hierarchy):
    # :104-134
    near, _ = select(oracle, hierarchy, lod_cam(oracle), 400, 1.0)
    far, _ = select(oracle, hierarchy, lod_cam(oracle, 1000000.0), 400, 1.0)
    assert len(near) > 1 and len(far) == 1


def test_color_variation_refines(oracle, reference):
    # :249-275
    lay = np.zeros(7, sk.LOD_NODE_DTYPE)
    spec = [((0, 0, -2), 2, 1, 2), ((-0.7, 0, -2), 0.1, 3, 2), ((0.7, 0, -2), 1.8, 5, 2),
            ((-0.8, 0, -2), 0.1, 0, 0), ((-0.6, 0, -2), 0.1, 0, 0), ((0.6, 0, -2), 0.1, 0, 0),
            ((0.8, 0, -2), 0.1, 0, 0)]
    for i, (p, s, cs, cc) in enumerate(spec):
        lay[i] = (p, s, cs, cc)
    nodes = sk.Cloud(lay["position"], np.tile([0.01, 0, 0, 0.01, 0, 0.01], (7, 1)),
                     np.ones((7, 3)), np.full(7, 0.5))
    nodes.colors[5, 0] = 0
    nodes.colors[6, 1] = 0
    tree = reference.make_tree(nodes, lay, 4)
    cut, stats = oracle.lod_select(lod_cam(oracle, 100.0), tree["clusters"], tree["leaves"],
                                   tree["depth"] + 1, 4, 1.0, 4.0, False)
    assert set(cut.tolist()) == {1, 5, 6}
    assert stats[4] == 0 and stats[5] == 3


def test_packets_and_capacity_pressure(oracle, hierarchy):
    # :277-291
    cut, stats = select(oracle, hierarchy, lod_cam(oracle), 515, 0.0, cull=False)
    assert len(cut) == 515 and stats[4] == 0 and stats[5] == len(hierarchy["clusters"])
    cut, stats = select(oracle, hierarchy, lod_cam(oracle), 33, 0.0, cull=False)
    assert len(cut) <= 33 and stats[4] > 0


def test_empty_view_and_single_leaf_root(oracle, hierarchy, reference):
    # :293-307
    cut, _ = select(oracle, hierarchy, lod_cam(oracle, -100.0), 515, 0.0)
    assert len(cut) == 0
    one = sk.Cloud([[0, 0, -2]], [[0.001, 0, 0, 0.001, 0, 0.001]], [[1, 1, 1]], [0.5])
    tree = reference.build_lod_tree(one)
    cut, _ = select(oracle, tree, lod_cam(oracle), 1, 1.0)
    assert cut.tolist() == [0]


@pytest.mark.parametrize("capacity", [20000, 32768])
def test_cross_block_scan(oracle, reference, capacity):
    # :309-342: a complete binary tree over 32768 leaves
    count = 32768
    nodes_n = 2 * count - 1
    lay = layout_tree(nodes_n, lambda i: (2 * i + 1, 2) if i < count - 1 else (0, 0))
    tree = reference.make_tree(uniform_nodes(nodes_n), lay, count)
    cut, stats = oracle.lod_select(lod_cam(oracle), tree["clusters"], tree["leaves"],
                                   tree["depth"] + 1, capacity, 0.0, 4.0, False)
    assert len(cut) == capacity
    represented = []
    for node in cut:
        leaves_under(lay, int(node), represented)
    assert len(represented) == count and len(set(represented)) == count
    if capacity == count:
        assert stats[4] == 0 and stats[5] == count - 1
    else:
        assert stats[4] > 0


def test_each_round_emits_after_previous(oracle, reference):
    # :346-366
    lay = layout_tree(5, lambda i: (1, 2) if i == 0 else ((3, 2) if i == 2 else (0, 0)))
    tree = reference.make_tree(uniform_nodes(5), lay, 3)
    cut, stats = oracle.lod_select(lod_cam(oracle), tree["clusters"], tree["leaves"],
                                   tree["depth"] + 1, 3, 0.0, 4.0, False)
    assert cut.tolist() == [1, 3, 4] and stats[5] == 2


def test_large_leaf_packet(oracle, reference):
    # :368-393
    lay = layout_tree(514, lambda i: (1, 513) if i == 0 else (0, 0))
    tree = reference.make_tree(uniform_nodes(514), lay, 513)
    cut, stats = oracle.lod_select(lod_cam(oracle), tree["clusters"], tree["leaves"],
                                   tree["depth"] + 1, 513, 0.0, 4.0, True)
    assert cut.tolist() == list(range(1, 514)) and stats[5] == 1 and stats[4] == 0
    cut, stats = oracle.lod_select(lod_cam(oracle), tree["clusters"], tree["leaves"],
                                   tree["depth"] + 1, 512, 0.0, 4.0, True)
    assert cut.tolist() == [0] and stats[4] == 1


# ---- raster (MetalSplatPipelineTest.mm) ---------------------------------------------------
def draw_one(oracle, reference, cloud, size=64, bits=32):
    packed = reference.pack_splats(cloud)
    proj = skcam.perspective(1.0, 1.0, 0.1, 100.0)
    cam = oracle.camera(identity(), proj, (0, 0, 0), size, size, 1.0)
    keys, pr = oracle.visibility(cam, packed, None, 0, 0, bits, [(0, cloud.count)])
    order = oracle.stable_argsort(keys)
    return oracle.composite(pr, order, size, size)


def test_nearer_splat_wins(oracle, reference):
    # :173-192
    cloud = sk.Cloud([[0, 0, -2.5], [0, 0, -1.8]], [[0.05, 0, 0, 0.05, 0, 0.05]] * 2,
                     [[0, 1, 0], [1, 0, 0]], [1, 1])
    img = draw_one(oracle, reference, cloud)
    r, g = img[32, 32, 0] * 255, img[32, 32, 1] * 255
    assert r > 150 and g < 80


@pytest.mark.parametrize("alpha,coverage", [(0.5, 0.5 * 0.991), (0.1, 0.1 * 0.991), (4.0, 1.0)])
def test_analytic_blend_over_background(oracle, reference, alpha, coverage):
    # :197-232: colour = coverage * c + (1 - coverage) * bg within 1/255 at the centre pixel
    colour, bg = (0.6, 0.2, 0.4), (0.05, 0.05, 0.08)
    cloud = sk.Cloud([[0, 0, -2.5]], [[0.05, 0, 0, 0.05, 0, 0.05]], [colour], [alpha])
    img = draw_one(oracle, reference, cloud)
    for c in range(3):
        expected = coverage * colour[c] + (1 - coverage) * bg[c]
        assert abs(img[32, 32, c] - expected) * 255 <= 1.0


def test_background_alone(oracle):
    # :113-129
    img = oracle.composite(np.zeros(0, sk.PROJECTED_DTYPE), np.zeros(0, np.uint32), 64, 64)
    assert np.allclose(img[32, 32, :3] * 255, [12.75, 12.75, 20.4], atol=1e-3)
    assert [round(v) for v in img[32, 32, :3] * 255] == [13, 13, 20]
