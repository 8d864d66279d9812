""".lodsplat files: the product reader against the reference's own writer and decoder (CPU), and
an uploaded file drawing the same frame as the same tree uploaded from memory (GPU)."""
from __future__ import annotations

import struct

import numpy as np
import pytest

import splatkit_b200 as sk
from splatkit_b200 import synthetic


def cluster_cloud(n=6000, seed=3, sh_degree=2):
    return synthetic.random_cloud(n, seed=seed, sh_degree=sh_degree, half_extent=5.0)


def assert_same_tree(ours: sk.LodTree, ref: dict):
    np.testing.assert_array_equal(ours.nodes.positions, ref["positions"])
    np.testing.assert_array_equal(ours.nodes.covariances, ref["covariances"])
    np.testing.assert_array_equal(ours.nodes.colors, ref["colors"])
    np.testing.assert_array_equal(ours.nodes.alphas, ref["alphas"])
    if ref["sh"] is None:
        assert ours.nodes.sh is None
    else:
        np.testing.assert_array_equal(ours.nodes.sh, ref["sh"])
    assert ours.layout.tobytes() == np.ascontiguousarray(ref["layout"]).tobytes()
    assert ours.leaf_count == ref["leaf_count"]
    if ref["clusters"] is None or len(ref["clusters"]) == 0:
        assert ours.clusters is None
    else:
        assert ours.clusters.tobytes() == np.ascontiguousarray(ref["clusters"]).tobytes()
        np.testing.assert_array_equal(ours.leaves, ref["leaves"])


@pytest.mark.parametrize("selection", [True, False])
def test_reader_matches_the_reference_decoder(reference, tmp_path, selection):
    path = tmp_path / "world.lodsplat"
    built = reference.write_lodsplat(cluster_cloud(), path, selection=selection)
    data = path.read_bytes()
    header = sk.lodsplat_header(data)
    assert header["version"] == (2 if selection else 1)
    assert header["node_count"] == len(built["layout"]) and header["depth"] == built["depth"]
    for max_sh in (3, 1, 0):
        assert_same_tree(sk.lodsplat_decode(data, max_sh), reference.decode_lodsplat(data, max_sh))


def test_reader_rejects_what_the_reference_rejects(reference, tmp_path):
    path = tmp_path / "world.lodsplat"
    reference.write_lodsplat(cluster_cloud(2400, seed=5), path)
    good = path.read_bytes()
    n = struct.unpack_from("<I", good, 12)[0]
    stride = 64 + 3 * 8 * 4
    bad = {
        "truncated": good[:-1],
        "magic": b"X" + good[1:],
        "version": good[:8] + struct.pack("<I", 3) + good[12:],
        "depth": good[:24] + struct.pack("<I", struct.unpack_from("<I", good, 24)[0] + 1) + good[28:],
        "alpha": good[:64 + 5 * stride + 60] + struct.pack("<f", float("nan")) + good[64 + 5 * stride + 64:],
        "child": good[:64 + 16] + struct.pack("<I", n + 7) + good[64 + 20:],
    }
    for name, data in bad.items():
        assert reference.decode_lodsplat(data) is None, name
        with pytest.raises(sk.SplatError):
            sk.lodsplat_decode(data)


@pytest.mark.gpu
def test_uploaded_file_draws_the_tree_it_holds(reference, tmp_path, cuda_device):
    from splatkit_b200 import camera as skcam

    path = tmp_path / "world.lodsplat"
    reference.write_lodsplat(cluster_cloud(9000, seed=7, sh_degree=3), path)
    tree = sk.lodsplat_decode(path.read_bytes())
    view, eye = skcam.orbit_view(4, radius=30.0)
    proj = skcam.perspective(1.0, 4 / 3, 0.05, 500.0)
    frame = sk.Frame(view, proj, eye, [], 3)
    out = []
    for upload in ("file", "bytes", "tree"):
        r = sk.Renderer(320, 240, image_format=sk.FORMAT_RGBA8)
        r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
        if upload == "file":
            r.upload_lodsplat(path, 3, 200_000)
        elif upload == "bytes":
            r.upload_lodsplat(path.read_bytes(), 3, 200_000)
        else:
            r.upload_lod_world(tree, 3, 200_000)
        r.draw(frame)
        cut, _ = r.read_cut()
        out.append((cut, r.read_order(), r.read_image(sk.FORMAT_RGBA8)))
        r.close()
    for cut, order, image in out[1:]:
        np.testing.assert_array_equal(cut, out[0][0])
        np.testing.assert_array_equal(order, out[0][1])
        np.testing.assert_array_equal(image, out[0][2])
    assert len(out[0][0]) > 0
