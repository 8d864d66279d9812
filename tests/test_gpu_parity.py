"""GPU parity through the C ABI: the CUDA path against the CPU oracle and the reference's
known answers. Cull, keys, projected records, the depth order and the LOD cut must be
bit-exact; images must be within 1/255 per channel (max abs) of the FP64 composite, with
the PSNR printed and bounded below."""
from __future__ import annotations

import math

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

from scenes import (hierarchy_cloud, identity, layout_tree, leaves_under, lod_camera, psnr,
                    three_splats, tree_from_reference, uniform_nodes)

pytestmark = pytest.mark.gpu

TOL = 1.0 / 255.0  # image tolerance, max abs per channel
MIN_PSNR = 50.0    # dB against the FP64 composite


def square_proj(near=0.1, far=100.0):
    """A projection whose P00 = P11 = 1: over a 1000 px square it gives focal 500 px and
    tanHalfFov 1, the hand-set uniform of the reference's visibility tests."""
    p = skcam.perspective(1.0, 1.0, near, far)
    p[0] = p[5] = 1.0
    return p


def render(cloud, view, proj, campos, width, height, ranges=None, sh_degree=None, bits=32,
           policy=None, fmt=sk.FORMAT_RGBA32F):
    r = sk.Renderer(width, height, image_format=fmt)
    pol = policy or sk.Policy(sort_depth_bits=bits, subpixel_threshold=0.0)
    r.apply_render_policy(pol)
    r.upload_world(cloud, 3)
    degree = cloud.sh_degree if sh_degree is None else sh_degree
    r.draw(sk.Frame(view, proj, campos, ranges if ranges is not None else [(0, cloud.count)], degree))
    keys, projected = r.read_visible()
    order = r.read_order()
    image = r.read_image(fmt)
    stats = r.stats()
    r.close()
    return keys, projected, order, image, stats


def oracle_frame(oracle, cloud, view, proj, campos, width, height, ranges=None, degree=None,
                 bits=32, minpx=0.0, threads=8, composite=True):
    degree = cloud.sh_degree if degree is None else degree
    packed = sk.pack_splats(cloud)
    stride = sk.sh_device_stride(degree)
    sh = sk.pack_sh(cloud, degree) if degree else None
    cam = oracle.camera(view, proj, campos, width, height, minpx)
    keys, pr = oracle.visibility(cam, packed, sh, stride, degree, bits,
                                 ranges if ranges is not None else [(0, cloud.count)], threads=threads)
    order = oracle.stable_argsort(keys)
    image = oracle.composite(pr, order, width, height, threads=threads) if composite else None
    return keys, pr, order, image


def assert_frame_parity(gpu, ref, image_check=True, label=""):
    keys, projected, order, image, stats = gpu
    okeys, oproj, oorder, oimage = ref
    assert len(keys) == len(okeys), label
    assert np.array_equal(keys, okeys), label
    assert projected.tobytes() == oproj.tobytes(), label
    assert np.array_equal(order, oorder), label
    assert stats["device_error"] == 0
    if image_check:
        err = np.abs(image.astype(np.float64) - oimage.astype(np.float64)).max()
        p = psnr(image[..., :3], oimage[..., :3])
        print(f"{label}: visible {len(keys)}, max abs {err * 255:.3f}/255, PSNR {p:.1f} dB")
        assert err <= TOL, label
        assert p >= MIN_PSNR, label


# ---- the reference's visibility known answers (MetalVisibilityPassTest.mm) -----------------
def test_culls_and_orders_ranges_front_to_back(oracle, cuda_device):
    positions = [[0, 0, -10], [0, 0, 5], [0, 0, -2], [50, 0, -1], [0, 0, -5], [0, 0, -3]]
    cloud = sk.Cloud(positions, [[1, 0, 0, 1, 0, 1]] * 6, [[1, 1, 1]] * 6, [1.0] * 6)
    ranges = [(0, 3), (3, 2)]
    gpu = render(cloud, identity(), square_proj(), (0, 0, 0), 1000, 1000, ranges)
    assert list(gpu[1]["index"][gpu[2]]) == [2, 4, 0]
    assert_frame_parity(gpu, oracle_frame(oracle, cloud, identity(), square_proj(), (0, 0, 0),
                                          1000, 1000, ranges))


def test_footprint_depth_planes_and_radius_cap(oracle, cuda_device):
    cases = [(-2.0, 0.0024, 1.0), (-2.0, 0.0008, 1.0), (-0.05, 0.1, 1.0), (-150.0, 1.0, 1.0),
             (-2.0, 0.1, 2.0), (-2.0, 1.6, 1.0)]
    cloud = sk.Cloud([[0, 0, z] for z, _, _ in cases],
                     [[s * s, 0, 0, s * s, 0, s * s] for _, s, _ in cases],
                     [[1, 1, 1]] * 6, [a for _, _, a in cases])
    pol = sk.Policy(sort_depth_bits=32, subpixel_threshold=1.0)
    gpu = render(cloud, identity(), square_proj(), (0, 0, 0), 1000, 1000, policy=pol)
    assert sorted(gpu[1]["index"]) == [0, 4, 5]
    huge = gpu[1][gpu[1]["index"] == 5][0]
    assert abs(float(huge["radius"]) - 512.0 / 400.0) <= 0.02
    assert_frame_parity(gpu, oracle_frame(oracle, cloud, identity(), square_proj(), (0, 0, 0),
                                          1000, 1000, minpx=1.0))


def test_sixteen_bit_keys_order(oracle, cuda_device):
    z_near = 0.05
    proj = square_proj(z_near, 200.0)
    view = identity()
    view[14] = -10
    depths = [150, 2.0002, 2.0001, 0.4003, 0.4002, 0.06, 199, 250, -1]
    cloud = sk.Cloud([[0, 0, 10 - d] for d in depths], [[1, 0, 0, 1, 0, 1]] * 9, [[1, 1, 1]] * 9,
                     [1.0] * 9)
    gpu = render(cloud, view, proj, (0, 0, 10), 1000, 1000, bits=16)
    assert list(gpu[1]["index"][gpu[2]]) == [5, 4, 3, 1, 2, 0, 6]
    assert_frame_parity(gpu, oracle_frame(oracle, cloud, view, proj, (0, 0, 10), 1000, 1000,
                                          bits=16))


def test_compacts_tails_in_source_order(oracle, cuda_device):
    positions = np.zeros((513, 3), np.float32)
    positions[:, 2] = -2
    positions[::3, 2] = 2
    cloud = sk.Cloud(positions, np.tile([1, 0, 0, 1, 0, 1], (513, 1)), np.ones((513, 3)),
                     np.ones(513))
    r = sk.Renderer(1000, 1000)
    r.apply_render_policy(sk.Policy(sort_depth_bits=32, subpixel_threshold=0.0))
    r.upload_world(cloud, 0)
    for n in (1, 31, 32, 33, 255, 256, 257, 513, 0):
        r.draw(sk.Frame(identity(), square_proj(), (0, 0, 0), [(0, n)] if n else []))
        keys, projected = r.read_visible()
        assert len(keys) == n - (n + 2) // 3
        # source order: survivors appear in increasing index
        assert np.all(np.diff(projected["index"].astype(np.int64)) > 0)
        assert all(i % 3 for i in projected["index"])
    r.close()


@pytest.mark.parametrize("bits", [32, 16])
def test_three_splats_front_to_back(oracle, cuda_device, bits):
    # MetalFrameComputeTest.mm:168-214
    cloud = three_splats()
    proj = skcam.perspective(1.0, 1.0, 0.1, 100.0)
    gpu = render(cloud, identity(), proj, (0, 0, 0), 64, 64, bits=bits)
    assert list(gpu[1]["index"][gpu[2]]) == [2, 0, 1]
    assert_frame_parity(gpu, oracle_frame(oracle, cloud, identity(), proj, (0, 0, 0), 64, 64,
                                          bits=bits))


def test_invalid_ranges_encode_nothing(cuda_device):
    cloud = three_splats()
    r = sk.Renderer(64, 64)
    r.upload_world(cloud, 0)
    for ranges in ([(2, 5)], [(3, 1)], [(0, 2), (0, 2)]):
        with pytest.raises(sk.SplatError) as err:
            r.draw(sk.Frame(identity(), skcam.perspective(1, 1, 0.1, 100), (0, 0, 0), ranges))
        assert err.value.status == sk.SK_E_INVALID
    assert r.stats()["submitted_frames"] == 0
    r.close()


# ---- raster (MetalSplatPipelineTest.mm) ----------------------------------------------------
def test_nearer_splat_wins_and_background(cuda_device):
    cloud = sk.Cloud([[0, 0, -2.5], [0, 0, -1.8]], [[0.05, 0, 0, 0.05, 0, 0.05]] * 2,
                     [[0, 1, 0], [1, 0, 0]], [1, 1])
    r = sk.Renderer(64, 64)
    r.upload_world(cloud, 0)
    r.draw(sk.Frame(identity(), skcam.perspective(1, 1, 0.1, 100), (0, 0, 0), [(0, 2)]))
    bgra = r.read_image(sk.FORMAT_BGRA8)
    assert bgra[32, 32, 2] > 150 and bgra[32, 32, 1] < 80
    r.draw(sk.Frame(identity(), skcam.perspective(1, 1, 0.1, 100), (0, 0, 0), []))
    bgra = r.read_image(sk.FORMAT_BGRA8)
    assert list(bgra[32, 32]) == [20, 13, 13, 255]
    r.close()


@pytest.mark.parametrize("alpha,coverage", [(0.5, 0.5 * 0.991), (0.1, 0.1 * 0.991), (4.0, 1.0)])
def test_analytic_blend(cuda_device, alpha, coverage):
    colour, bg = (0.6, 0.2, 0.4), (0.05, 0.05, 0.08)
    cloud = sk.Cloud([[0, 0, -2.5]], [[0.05, 0, 0, 0.05, 0, 0.05]], [colour], [alpha])
    r = sk.Renderer(64, 64)
    r.upload_world(cloud, 0)
    r.draw(sk.Frame(identity(), skcam.perspective(1, 1, 0.1, 100), (0, 0, 0), [(0, 1)]))
    bgra = r.read_image(sk.FORMAT_BGRA8)
    for c in range(3):
        expected = coverage * colour[c] + (1 - coverage) * bg[c]
        assert abs(float(bgra[32, 32, 2 - c]) - expected * 255) <= 1.0
    r.close()


# ---- randomized scenes at the benchmark distributions ---------------------------------------
@pytest.mark.parametrize("bits", [32, 16])
def test_small_scene_sh0_parity(oracle, cuda_device, bits):
    # the 100k-splat SH0 single-frame workload at 1280x720, camera at the cube edge
    cloud = synthetic.random_cloud(100_000, seed=0, sh_degree=0)
    proj = skcam.perspective(math.radians(60), 1280 / 720, 0.05, 200.0)
    view = skcam.look_at_view((0, 0, 10), (0, 0, 0))
    gpu = render(cloud, view, proj, (0, 0, 10), 1280, 720, bits=bits,
                 policy=sk.Policy(sort_depth_bits=bits))
    ref = oracle_frame(oracle, cloud, view, proj, (0, 0, 10), 1280, 720, bits=bits, minpx=1.0)
    assert_frame_parity(gpu, ref, label=f"100k SH0 {bits}-bit")


@pytest.mark.parametrize("frame", [0, 37, 90])
def test_sh3_orbit_parity(oracle, cuda_device, frame):
    cloud = synthetic.random_cloud(120_000, seed=1, sh_degree=3)
    view, eye = skcam.orbit_view(frame)
    proj = skcam.perspective(math.radians(60), 640 / 480, 0.05, 200.0)
    pol = sk.Policy(sort_depth_bits=32)
    gpu = render(cloud, view, proj, eye, 640, 480, policy=pol)
    ref = oracle_frame(oracle, cloud, view, proj, eye, 640, 480, minpx=1.0)
    assert_frame_parity(gpu, ref, label=f"120k SH3 orbit {frame}")


def test_lower_sh_degree_frame_and_multi_ranges(oracle, cuda_device):
    cloud = synthetic.random_cloud(50_000, seed=2, sh_degree=3)
    view, eye = skcam.orbit_view(11)
    proj = skcam.perspective(math.radians(60), 1.0, 0.05, 200.0)
    ranges = [(100, 20000), (30000, 5000), (0, 50), (45000, 5000)]
    for degree in (1, 2):
        gpu = render(cloud, view, proj, eye, 320, 320, ranges=ranges, sh_degree=degree,
                     policy=sk.Policy(sort_depth_bits=16))
        ref = oracle_frame(oracle, cloud, view, proj, eye, 320, 320, ranges=ranges,
                           degree=degree, bits=16, minpx=1.0)
        assert_frame_parity(gpu, ref, label=f"SH{degree} ranges")


# ---- the sort component (MetalRadixSortTest.mm:81-140) --------------------------------------
def gpu_argsort(keys: np.ndarray, bits: int, capacity=None, stale=None):
    import torch

    n = len(keys)
    capacity = max(n, 1) if capacity is None else capacity
    dev = torch.device("cuda")
    k = torch.from_numpy(np.ascontiguousarray(keys).view(np.int32).copy()).to(dev) if n else \
        torch.zeros(1, dtype=torch.int32, device=dev)
    count = torch.tensor([n], dtype=torch.int32, device=dev)
    order = torch.full((capacity,), -1 if stale is None else stale, dtype=torch.int64,
                       device=dev).to(torch.int32)
    ws = torch.zeros(sk.sort_workspace_bytes(capacity), dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    before = k.clone()
    sk.radix_argsort_device(k.data_ptr(), count.data_ptr(), capacity, bits, order.data_ptr(),
                            ws.data_ptr(), ws.numel(), err.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(k, before)  # keys are read only
    return order.cpu().numpy().view(np.uint32)[:n]


def test_sort_random_keys_like_stable_sort(oracle, cuda_device):
    keys = oracle.mt19937(1, 1000003)
    assert np.array_equal(gpu_argsort(keys, 32), oracle.stable_argsort(keys))


def test_sort_keeps_order_of_equal_keys(oracle, cuda_device):
    keys = oracle.mt19937(2, 70000) & np.uint32(0x7)
    assert np.array_equal(gpu_argsort(keys, 32), oracle.stable_argsort(keys))
    assert np.array_equal(gpu_argsort(keys, 16), oracle.stable_argsort(keys))


def test_sort_ignores_stale_order_buffer(oracle, cuda_device):
    keys = oracle.mt19937(6, 70000) & np.uint32(0xFFFF)
    for bits in (16, 32):
        assert np.array_equal(gpu_argsort(keys, bits, stale=0x0EADBEEF), oracle.stable_argsort(keys))


def test_sort_small_empty_and_block_sizes(oracle, cuda_device):
    for n in (0, 1, 17, 31, 32, 33, 4095, 4096, 4097, 1000003):
        keys = oracle.mt19937(16, n) & np.uint32(0xFFFF)
        if n > 1:
            keys[0], keys[-1] = 65535, 0
        expected = oracle.stable_argsort(keys)
        assert np.array_equal(gpu_argsort(keys, 16), expected), n
        assert np.array_equal(gpu_argsort(keys, 32), expected), n
    keys = oracle.mt19937(3, 17)
    assert np.array_equal(gpu_argsort(keys, 32, capacity=64), oracle.stable_argsort(keys))


def test_sort_count_is_clamped_to_capacity(oracle, cuda_device):
    import torch

    keys = oracle.mt19937(9, 5000)
    dev = torch.device("cuda")
    k = torch.from_numpy(keys.view(np.int32).copy()).to(dev)
    count = torch.tensor([10_000], dtype=torch.int32, device=dev)  # more than the capacity
    order = torch.zeros(4096, dtype=torch.int32, device=dev)
    ws = torch.zeros(sk.sort_workspace_bytes(4096), dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    sk.radix_argsort_device(k.data_ptr(), count.data_ptr(), 4096, 32, order.data_ptr(),
                            ws.data_ptr(), ws.numel(), err.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = order.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, oracle.stable_argsort(keys[:4096]))


# ---- LOD cut (MetalLodSelectionTest.mm) ----------------------------------------------------
def lod_frame(distance=0.0):
    view, _, pos = lod_camera(distance)
    return view, square_proj(0.1, 1000000.0), pos


def gpu_cut(tree: sk.LodTree, budget, policy: sk.Policy, distance=0.0, frustum=True):
    r = sk.Renderer(1000, 1000)
    policy.enable_frustum_culling = frustum
    r.apply_render_policy(policy)
    r.upload_lod_world(tree, 0, budget)
    view, proj, pos = lod_frame(distance)
    r.draw(sk.Frame(view, proj, pos, [], 0))
    cut, stats = r.read_cut()
    keys, projected = r.read_visible()
    order = r.read_order()
    st = r.stats()
    r.close()
    return cut, stats, keys, projected, order, st


def oracle_cut(oracle, tree_dict, budget, pixel_limit, distance=0.0, cull=True):
    view, proj, pos = lod_frame(distance)
    cam = oracle.camera(view, proj, pos, 1000, 1000, 0.0)
    cap = min(budget, 4000000, tree_dict["leaf_count"])
    return oracle.lod_select(cam, tree_dict["clusters"], tree_dict["leaves"],
                             tree_dict["depth"] + 1, cap, pixel_limit, 4.0, cull)


@pytest.fixture(scope="module")
def hierarchy(reference):
    return reference.build_lod_tree(hierarchy_cloud(), octree_depth=6)


def test_lod_cuts_match_oracle_for_every_budget(oracle, hierarchy, cuda_device):
    tree = tree_from_reference(hierarchy)
    for budget in (1, 7, 31, 32, 33, 64, 257, 400, 515):
        for limit in (0.0, 1.0):
            cut, stats, *_ , st = gpu_cut(tree, budget, sk.Policy(lod_error_pixels=limit or 1e-6))
            # the policy cannot say 0 px; the oracle gets the same threshold
            ocut, ostats = oracle_cut(oracle, hierarchy, budget, limit or 1e-6)
            assert np.array_equal(cut, ocut), (budget, limit)
            assert np.array_equal(stats, ostats), (budget, limit)
            represented = []
            for node in cut:
                leaves_under(hierarchy["layout"], int(node), represented)
            assert sorted(represented) == sorted(set(represented))
            assert len(represented) == hierarchy["leaf_count"]
            assert st["device_error"] == 0


def test_lod_selection_built_on_upload_matches(oracle, hierarchy, cuda_device):
    tree = tree_from_reference({**hierarchy, "clusters": np.zeros(0, sk.LOD_CLUSTER_DTYPE),
                                "leaves": np.zeros(0, np.uint32)})
    cut, stats, *_ = gpu_cut(tree, 400, sk.Policy(lod_error_pixels=1.0))
    ocut, ostats = oracle_cut(oracle, hierarchy, 400, 1.0)
    assert np.array_equal(cut, ocut) and np.array_equal(stats, ostats)


def test_lod_distance_changes_cut(oracle, hierarchy, cuda_device):
    tree = tree_from_reference(hierarchy)
    near = gpu_cut(tree, 400, sk.Policy(lod_error_pixels=1.0))[0]
    far = gpu_cut(tree, 400, sk.Policy(lod_error_pixels=1.0), distance=1000000.0)[0]
    assert len(near) > 1 and len(far) == 1
    assert len(gpu_cut(tree, 515, sk.Policy(lod_error_pixels=1.0), distance=-100.0)[0]) == 0


def test_lod_small_trees(oracle, reference, cuda_device):
    cases = [
        (layout_tree(5, lambda i: (1, 2) if i == 0 else ((3, 2) if i == 2 else (0, 0))), 5, 3, 3,
         [1, 3, 4]),
        (layout_tree(514, lambda i: (1, 513) if i == 0 else (0, 0)), 514, 513, 513,
         list(range(1, 514))),
        (layout_tree(514, lambda i: (1, 513) if i == 0 else (0, 0)), 514, 513, 512, [0]),
    ]
    for lay, nodes, leaves, budget, expected in cases:
        d = reference.make_tree(uniform_nodes(nodes), lay, leaves)
        cut, stats, *_ = gpu_cut(tree_from_reference(d), budget, sk.Policy(lod_error_pixels=1e-6),
                                 frustum=False)
        ocut, ostats = oracle_cut(oracle, d, budget, 1e-6, cull=False)
        assert cut.tolist() == expected
        assert np.array_equal(cut, ocut) and np.array_equal(stats, ostats)


@pytest.mark.parametrize("budget", [20000, 32768])
def test_lod_cross_block_scan(oracle, reference, cuda_device, budget):
    count = 32768
    lay = layout_tree(2 * count - 1, lambda i: (2 * i + 1, 2) if i < count - 1 else (0, 0))
    d = reference.make_tree(uniform_nodes(2 * count - 1), lay, count)
    cut, stats, *_ = gpu_cut(tree_from_reference(d), budget, sk.Policy(lod_error_pixels=1e-6),
                             frustum=False)
    ocut, ostats = oracle_cut(oracle, d, budget, 1e-6, cull=False)
    assert len(cut) == budget
    assert np.array_equal(cut, ocut) and np.array_equal(stats, ostats)


def test_lod_world_culls_and_sorts_only_the_cut(oracle, reference, cuda_device):
    cloud = synthetic.clustered_cloud(clusters=40, per_cluster=500, seed=3, half_extent=20.0)
    d = reference.build_lod_tree(cloud)
    tree = tree_from_reference(d)
    r = sk.Renderer(480, 270)
    r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=32))
    r.upload_lod_world(tree, 0, 4_000_000)
    proj = skcam.perspective(math.radians(60), 480 / 270, 0.05, 200.0)
    for x in (-30.0, 0.0, 25.0):
        view = skcam.look_at_view((x, 1.7, 30.0), (x + 10.0, 1.7, 0.0))
        r.draw(sk.Frame(view, proj, (x, 1.7, 30.0), [], 0))
        cut, stats = r.read_cut()
        keys, projected = r.read_visible()
        order = r.read_order()
        cam = oracle.camera(view, proj, (x, 1.7, 30.0), 480, 270, 1.0)
        # the threshold in use for this frame (it adapts between frames)
        ocut, ostats = oracle.lod_select(cam, d["clusters"], d["leaves"], d["depth"] + 1,
                                         min(4_000_000, d["leaf_count"]), 1.5, 4.0, True)
        assert np.array_equal(cut, ocut)
        packed = sk.pack_splats(tree.nodes)
        okeys, oproj = oracle.visibility(cam, packed, None, 0, 0, 32, indices=ocut)
        assert np.array_equal(keys, okeys)
        assert projected.tobytes() == oproj.tobytes()
        assert np.array_equal(order, oracle.stable_argsort(okeys))
    r.close()
