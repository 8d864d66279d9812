"""Seeded synthetic splat scenes with the shapes and value distributions of the benchmark
workloads (no dataset is involved). Draw order and distributions are part of each function's
contract so any consumer can regenerate the same bytes.

Covariances are built as the reference does (splat-core/src/math/Covariance.cpp:7-17 with
Mat4::rotation of a unit quaternion, Mat4.h:47-63): M = R diag(s), Sigma = M M^T, every product
and sum in float32 in that order.
"""
from __future__ import annotations

import numpy as np

from . import Cloud, sh_coefficients

f32 = np.float32


def covariance_from_quaternion_scale(q: np.ndarray, s: np.ndarray) -> np.ndarray:
    """q: (n, 4) unit quaternions (x, y, z, w); s: (n, 3) scales -> (n, 6) xx, xy, xz, yy, yz, zz."""
    q = q.astype(np.float32)
    s = s.astype(np.float32)
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    one, two = f32(1), f32(2)
    r = np.empty((len(q), 3, 3), np.float32)
    r[:, 0, 0] = one - two * (y * y + z * z)
    r[:, 0, 1] = two * (x * y - w * z)
    r[:, 0, 2] = two * (x * z + w * y)
    r[:, 1, 0] = two * (x * y + w * z)
    r[:, 1, 1] = one - two * (x * x + z * z)
    r[:, 1, 2] = two * (y * z - w * x)
    r[:, 2, 0] = two * (x * z - w * y)
    r[:, 2, 1] = two * (y * z + w * x)
    r[:, 2, 2] = one - two * (x * x + y * y)
    m = r * s[:, None, :]

    def dot(a, b):
        return m[:, a, 0] * m[:, b, 0] + m[:, a, 1] * m[:, b, 1] + m[:, a, 2] * m[:, b, 2]

    return np.stack([dot(0, 0), dot(0, 1), dot(0, 2), dot(1, 1), dot(1, 2), dot(2, 2)], axis=1)


def shoemake_quaternions(u: np.ndarray) -> np.ndarray:
    """Uniform unit quaternions (x, y, z, w) from u ~ U[0,1)^3 (Shoemake, Graphics Gems III)."""
    u = u.astype(np.float64)
    a, b = np.sqrt(1 - u[:, 0]), np.sqrt(u[:, 0])
    t1, t2 = 2 * np.pi * u[:, 1], 2 * np.pi * u[:, 2]
    q = np.stack([a * np.sin(t1), a * np.cos(t1), b * np.sin(t2), b * np.cos(t2)], axis=1)
    return q.astype(np.float32)


def random_cloud(n: int, seed: int = 0, sh_degree: int = 0, half_extent: float = 10.0,
                 log_scale_mean: float = -3.0, log_scale_std: float = 0.5,
                 sh_std: float = 0.1) -> Cloud:
    """The benchmark cloud: positions U[-h, h]^3, log-scales N(mean, std) per axis, uniform
    rotations, opacity sigmoid(N(0, 1)), colour (the SH DC term) U[0, 1], higher SH bands
    N(0, sh_std), channel fastest. numpy PCG64(seed), drawn in exactly this order: positions
    (n, 3), log-scales (n, 3), rotation uniforms (n, 3), opacity normals (n), colours (n, 3),
    then harmonics (n, 3 * ((d + 1)^2 - 1))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    positions = rng.uniform(-half_extent, half_extent, (n, 3)).astype(np.float32)
    scales = np.exp(rng.normal(log_scale_mean, log_scale_std, (n, 3))).astype(np.float32)
    q = shoemake_quaternions(rng.random((n, 3)))
    alphas = (1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.0, n)))).astype(np.float32)
    colors = rng.random((n, 3)).astype(np.float32)
    sh = None
    if sh_degree > 0:
        sh = rng.normal(0.0, sh_std, (n, 3 * sh_coefficients(sh_degree))).astype(np.float32)
    cov = covariance_from_quaternion_scale(q, scales)
    lo = positions.min(axis=0) if n else np.zeros(3, np.float32)
    hi = positions.max(axis=0) if n else np.zeros(3, np.float32)
    return Cloud(positions, cov, colors, alphas, sh_degree, sh, lo, hi)


def clustered_cloud(clusters: int = 2000, per_cluster: int = 3000, seed: int = 0,
                    half_extent: float = 100.0, rms: float = 2.0) -> Cloud:
    """The LOD workload: cluster centres U[-h, h]^3; per cluster a random rotation times
    diag(exp(N(0, 0.3))) scaled so the offsets' RMS radius is `rms` m, applied to N(0, 1)
    draws; other attributes as random_cloud with SH degree 0. PCG64(seed) order: centres,
    per-cluster rotation uniforms (clusters, 3), per-cluster log axis scales (clusters, 3),
    member normals (clusters * per_cluster, 3), then the random_cloud attributes except
    positions (log-scales, rotation uniforms, opacity, colours)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.uniform(-half_extent, half_extent, (clusters, 3))
    rot = shoemake_quaternions(rng.random((clusters, 3))).astype(np.float64)
    axes = np.exp(rng.normal(0.0, 0.3, (clusters, 3)))
    axes *= rms / np.sqrt((axes ** 2).sum(axis=1, keepdims=True))  # E|A z|^2 = sum(a^2) = rms^2
    x, y, z, w = rot[:, 0], rot[:, 1], rot[:, 2], rot[:, 3]
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    A = R * axes[:, None, :]
    n = clusters * per_cluster
    draws = rng.normal(0.0, 1.0, (n, 3)).reshape(clusters, per_cluster, 3)
    positions = (centres[:, None, :] + np.einsum("cij,cpj->cpi", A, draws)).reshape(n, 3)
    positions = positions.astype(np.float32)
    scales = np.exp(rng.normal(-3.0, 0.5, (n, 3))).astype(np.float32)
    q = shoemake_quaternions(rng.random((n, 3)))
    alphas = (1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.0, n)))).astype(np.float32)
    colors = rng.random((n, 3)).astype(np.float32)
    cov = covariance_from_quaternion_scale(q, scales)
    return Cloud(positions, cov, colors, alphas, 0, None, positions.min(axis=0),
                 positions.max(axis=0))
