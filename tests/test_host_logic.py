"""Host-side logic of the product against the reference's own C++ (CPU only): record packing,
LOD selection metadata, tree depth, world pricing, the adaptive LOD threshold, camera and
covariance helpers, and the project-owned numerics the kernels share with the oracle."""
from __future__ import annotations

import math
import re
from pathlib import Path

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam
from splatkit_b200 import synthetic

from scenes import hierarchy_cloud, layout_tree, uniform_nodes, tree_from_reference

ROOT = Path(__file__).resolve().parent.parent


def test_library_exports_every_declared_symbol():
    header = "".join(p.read_text() for p in sorted((ROOT / "include").glob("*.h")))
    declared = set(re.findall(r"\b(sk_[a-z0-9_]+)\s*\(", header))
    lib = sk.library()
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing
    assert declared == set(sk.exported_symbols())


@pytest.mark.parametrize("degree", [0, 1, 2, 3])
def test_packing_matches_reference(reference, degree):
    cloud = synthetic.random_cloud(20000, seed=7, sh_degree=3)
    cloud.alphas[::97] = np.linspace(1.5, 900, len(cloud.alphas[::97]))  # LOD opacities > 1
    cloud.colors[::101] = -0.5
    cloud.covariances[::89] *= 1e5  # saturating halves
    ours = sk.pack_splats(cloud)
    theirs = reference.pack_splats(cloud)
    assert ours.tobytes() == theirs.tobytes()
    stride = reference.sh_stride(degree)
    assert sk.sh_device_stride(degree) == (stride + 3) // 4 * 4
    if degree:
        sh_ours = sk.pack_sh(cloud, degree)
        sh_theirs = reference.pack_sh(cloud, degree)
        assert np.array_equal(sh_ours[:, :stride], sh_theirs)
        assert not sh_ours[:, stride:].any()


def test_half_conversion_matches_reference(oracle, reference):
    rng = np.random.default_rng(3)
    values = np.concatenate([rng.integers(0, 2**32, 50000, dtype=np.uint64).astype(np.uint32)
                            .view(np.float32),
                             np.array([0.0, -0.0, 65504, 65519.99, 65520, 1e9, -1e9, 2**-25,
                                       2**-24, 3 * 2**-26, np.inf, -np.inf], np.float32)])
    for v in values:
        if np.isnan(v):
            continue
        assert oracle.float_to_half(float(v)) == reference.to_half(float(v))


def test_own_log_within_one_ulp(oracle):
    rng = np.random.default_rng(4)
    xs = np.concatenate([rng.uniform(1, 130000, 5000), np.exp(rng.uniform(-60, 60, 5000))])
    for x in xs.astype(np.float32):
        got = oracle.ln(float(x))
        want = math.log(float(x))
        assert abs(got - want) <= np.spacing(np.float32(abs(want))) * 1.0 + 1e-45


def test_selection_data_matches_reference(reference):
    tree = reference.build_lod_tree(hierarchy_cloud(), octree_depth=6, selection=True)
    ours = tree_from_reference({**tree, "clusters": np.zeros(0, sk.LOD_CLUSTER_DTYPE),
                                "leaves": np.zeros(0, np.uint32)})
    clusters, leaves = sk.build_lod_selection(ours)
    assert clusters.tobytes() == tree["clusters"].tobytes()
    assert np.array_equal(leaves, tree["leaves"])


def test_selection_data_with_harmonics_matches_reference(reference):
    cloud = synthetic.random_cloud(6000, seed=11, sh_degree=3, half_extent=3.0)
    tree = reference.build_lod_tree(cloud, selection=True)
    ours = tree_from_reference({**tree, "clusters": np.zeros(0, sk.LOD_CLUSTER_DTYPE),
                                "leaves": np.zeros(0, np.uint32)})
    clusters, leaves = sk.build_lod_selection(ours)
    assert clusters.tobytes() == tree["clusters"].tobytes()
    assert np.array_equal(leaves, tree["leaves"])


def test_lod_depth_matches_reference(reference):
    tree = reference.build_lod_tree(hierarchy_cloud(), octree_depth=6)
    assert sk.lod_depth(tree["layout"], tree["leaf_count"]) == tree["depth"]
    lay = layout_tree(5, lambda i: (1, 2) if i == 0 else ((3, 2) if i == 2 else (0, 0)))
    ref = reference.make_tree(uniform_nodes(5), lay, 3)
    assert sk.lod_depth(lay, 3) == ref["depth"] == 2
    bad = lay.copy()
    bad[0]["child_start"] = 2
    assert sk.lod_depth(bad, 3) == -1
    assert sk.lod_depth(lay, 4) == -1


def test_world_bytes_match_reference(reference):
    for args in [(1000, 0, 1000, 0, 0), (1_000_000, 3, 1_000_000, 0, 0),
                 (7_200_000, 0, 4_000_000, 300_000, 6_000_000), (21_700_000, 3, 6_000_000, 0, 0)]:
        assert sk.world_bytes(*args) == reference.gpu_world_bytes(*args)


def test_lod_threshold_matches_reference(reference):
    rng = np.random.default_rng(5)
    for policy in (0.1, 1.0, 16.0, 100.0):
        ref = reference.lod_threshold(policy)
        state = np.array([policy, policy], np.float32)
        for _ in range(300):
            selected = int(rng.integers(0, 5000))
            limited = int(rng.integers(0, 3)) * int(rng.integers(0, 2))
            limit = int(rng.integers(1, 5000))
            assert sk.lod_threshold_update(state, selected, limited, limit) == \
                ref.update(selected, limited, limit)


def test_camera_matrices_match_reference(reference):
    for fovy, aspect, near, far in [(1.0, 1.0, 0.1, 100.0), (math.radians(60), 16 / 9, 0.05, 200.0),
                                    (math.radians(65), 1206 / 2622, 0.05, 200.0)]:
        assert np.allclose(skcam.perspective(fovy, aspect, near, far),
                           reference.perspective(fovy, aspect, near, far), rtol=2e-7, atol=0)
    for eye, target in [((0, 0, 10), (0, 0, 0)), ((15, 0, 3), (0, 0, 0)), ((-90, 1.7, 0), (10, 1.7, 0)),
                        ((0, 5, 0), (0, 0, 0))]:
        assert np.allclose(skcam.look_at_view(eye, target), reference.look_at_view(eye, target),
                           rtol=1e-6, atol=1e-6)


def test_covariance_matches_reference(reference):
    cloud_q = synthetic.shoemake_quaternions(np.random.default_rng(6).random((200, 3)))
    scales = np.exp(np.random.default_rng(7).normal(-3, 0.5, (200, 3))).astype(np.float32)
    ours = synthetic.covariance_from_quaternion_scale(cloud_q, scales)
    for i in range(200):
        assert ours[i].tobytes() == reference.covariance(cloud_q[i], scales[i]).tobytes()


def test_policy_validation_matches_reference(reference):
    cases = [(1.0, 0, 1 / 255, 1.0, 16, (0.05, 0.05, 0.08), True),
             (0.0, 0, 1 / 255, 1.0, 16, (0.05, 0.05, 0.08), False),
             (1.0, 0, 2.0, 1.0, 32, (0, 0, 0), False),
             (1.0, 0, 0.5, -1.0, 32, (0, 0, 0), False),
             (1.0, 0, 0.5, 1.0, 24, (0, 0, 0), False),
             (1.0, 0, 0.5, 1.0, 32, (0, 1.5, 0), False)]
    for *args, expected in cases:
        assert reference.valid_render_policy(*args) == expected


def test_frame_entry_points_reject_a_missing_context():
    # argument checks come before any device work, so they hold without a GPU
    import ctypes
    lib = sk.library()
    t = ctypes.c_uint64()
    buf = np.zeros(16, np.uint8)
    assert lib.sk_set_timing(None, 1) == sk.SK_E_INVALID
    assert lib.sk_set_binning(None, 0) == sk.SK_E_INVALID
    assert lib.sk_capture_next_frame(None, buf.ctypes.data, buf.nbytes, sk.FORMAT_RGBA8,
                                     ctypes.byref(t)) == sk.SK_E_INVALID
    assert lib.sk_wait_capture(None, 1) == sk.SK_E_INVALID
    assert lib.sk_draw(None, None) == sk.SK_E_INVALID


def test_device_tree_build_rejects_bad_clouds_before_device_work():
    import ctypes
    lib = sk.library()
    handle = ctypes.c_void_p()
    assert lib.sk_build_lod_tree_device(None, None, None, 0, 0, 1, ctypes.byref(handle)) == sk.SK_E_INVALID
    empty = sk.Cloud(np.zeros((0, 3), np.float32), np.zeros((0, 6), np.float32),
                     np.zeros((0, 3), np.float32), np.zeros(0, np.float32))
    v = empty.view()
    assert lib.sk_build_lod_tree_device(ctypes.byref(v), None, None, 0, 0, 1, ctypes.byref(handle)) == sk.SK_E_INVALID
    assert not handle.value
    # a count above 2^31 - 1 (2n - 1 nodes would not fit 32 bits) is refused before any array is read
    one = sk.Cloud(np.zeros((1, 3), np.float32), np.zeros((1, 6), np.float32),
                   np.zeros((1, 3), np.float32), np.zeros(1, np.float32))
    v = one.view()
    v.count = 0x80000000
    assert lib.sk_build_lod_tree_device(ctypes.byref(v), None, None, 0, 0, 1, ctypes.byref(handle)) == sk.SK_E_LIMIT
    assert not handle.value
