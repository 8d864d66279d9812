"""Scenes of the reference's own known-answer tests, rebuilt from the values in its test files
(packages/splatkit-ios/tests/rendering/metal/...), plus helpers that pack a cloud the way the
reference's GpuLayout does so the oracle sees the same bytes as the GPU."""
from __future__ import annotations

import math

import numpy as np

import splatkit_b200 as sk
from splatkit_b200 import camera as skcam

INF = float("inf")


def identity():
    m = np.zeros(16, np.float32)
    m[0] = m[5] = m[10] = m[15] = 1
    return m


def half_bits(x: float) -> int:
    return int(np.array([x], np.float16).view(np.uint16)[0])


def unit_cov_splats(positions, rgba8=0xFFFFFFFF, variance=1.0, lod_alpha=0):
    """GpuSplat records with an isotropic covariance (MetalVisibilityPassTest.mm:93-109)."""
    n = len(positions)
    s = np.zeros(n, sk.SPLAT_DTYPE)
    s["position"] = np.asarray(positions, np.float32)
    s["rgba8"] = rgba8
    v = half_bits(variance)
    s["cov"][:, 0] = v
    s["cov"][:, 1] = v << 16
    s["cov"][:, 2] = v << 16
    s["lodAlpha"] = lod_alpha
    return s


def test_camera(proj=None, view=None, cam_pos=(0, 0, 0)):
    """The visibility tests' camera (MetalVisibilityPassTest.mm:110-121): focal 500 px over a
    1000 px square. These tests set focal/tanHalfFov directly; a 1000 px screen with
    proj = perspective(1, 1, 0.1, 100) gives focal 500 * P00, so callers pass proj[0] = 1."""
    view = identity() if view is None else view
    proj = skcam.perspective(1.0, 1.0, 0.1, 100.0) if proj is None else proj
    return view, proj, np.asarray(cam_pos, np.float32)


def three_splats():
    """MetalFrameComputeTest.mm:54-62."""
    return sk.Cloud(positions=[[0, 0, -2], [0.6, 0.2, -2.5], [-0.5, -0.3, -1.8]],
                    covariances=[[0.02, 0, 0, 0.02, 0, 0.02], [0.01, 0, 0, 0.03, 0, 0.01],
                                 [0.03, 0, 0, 0.01, 0, 0.01]],
                    colors=[[1, 0, 0], [0, 1, 0], [0, 0.4, 1]], alphas=[1, 0.9, 0.8])


def hierarchy_cloud():
    """MetalLodSelectionTest.mm:22-38: 515 splats on a 17x17 grid in two layers."""
    pos, cov, col, alp = [], [], [], []
    for i in range(515):
        x = (i % 17) / 8.0 - 1
        y = ((i // 17) % 17) / 8.0 - 1
        z = -2.0 - (i // 289) * 0.25
        pos.append([x, y, z])
        cov.append([0.001, 0, 0, 0.001, 0, 0.001])
        col.append([1, 0, 0])
        alp.append(0.5)
    return sk.Cloud(pos, cov, col, alp, bounds_min=np.array([-1, -1, -3], np.float32),
                    bounds_max=np.array([1, 1, -2], np.float32))


def lod_camera(distance=0.0):
    """MetalLodSelectionTest.mm:39-51 (set as a 1000 px square with P00 = 1: focal 500)."""
    view = identity()
    view[14] = -distance
    proj = skcam.perspective(1.0, 1.0, 0.1, 1000000.0)
    return view, proj, np.array([0, 0, distance], np.float32)


def tree_from_reference(d) -> sk.LodTree:
    nodes = sk.Cloud(d["positions"], d["covariances"], d["colors"], d["alphas"], d["sh_degree"],
                     d["sh"])
    return sk.LodTree(nodes, d["layout"], d["leaf_count"],
                      d["clusters"] if len(d["clusters"]) else None,
                      d["leaves"] if len(d["leaves"]) else None)


def layout_tree(n_nodes, child_of):
    """A LodNode layout from a function i -> (child_start, child_count)."""
    lay = np.zeros(n_nodes, sk.LOD_NODE_DTYPE)
    for i in range(n_nodes):
        cs, cc = child_of(i)
        lay[i]["position"] = (0, 0, -2)
        lay[i]["size"] = 0.02
        lay[i]["child_start"] = cs
        lay[i]["child_count"] = cc
    return lay


def uniform_nodes(n, position=(0, 0, -2), variance=0.0001, color=0.5, alpha=0.1):
    return sk.Cloud(np.tile(np.asarray(position, np.float32), (n, 1)),
                    np.tile(np.array([variance, 0, 0, variance, 0, variance], np.float32), (n, 1)),
                    np.full((n, 3), color, np.float32), np.full(n, alpha, np.float32))


def leaves_under(layout, node, out):
    cc = int(layout[node]["child_count"])
    if cc == 0:
        out.append(node)
    cs = int(layout[node]["child_start"])
    for k in range(cc):
        leaves_under(layout, cs + k, out)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return INF if mse == 0 else 10 * math.log10(1.0 / mse)
