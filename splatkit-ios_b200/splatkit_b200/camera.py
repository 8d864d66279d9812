"""Camera matrices in the reference's conventions (float32, column major m[col * 4 + row]):
right handed, -Z forward, +Y up, clip depth in [0, 1].

  perspective   splat-core/include/splat/math/Mat4.h:75-86 (Mat4::perspective)
  look_at_view  splatkit-engine/src/camera/WalkCamera.cpp:24-37,218-227,535-537
                (setLookAt, then viewMatrix = (T(position) R)^-1 for a rigid transform)
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def perspective(fovy_radians: float, aspect: float, near: float, far: float) -> np.ndarray:
    ys = f32(1.0) / f32(math.tan(float(f32(fovy_radians) * f32(0.5))))
    xs = ys / f32(aspect)
    zs = f32(far) / (f32(near) - f32(far))
    m = np.zeros(16, np.float32)
    m[0] = xs
    m[5] = ys
    m[10] = zs
    m[14] = f32(near) * zs
    m[11] = f32(-1.0)
    return m


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]], np.float32)


def _normalize(v):
    length = f32(math.sqrt(float(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])))
    return (v / length).astype(np.float32) if length > 0 else np.zeros(3, np.float32)


def look_at_view(position, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    p = np.asarray(position, np.float32)
    t = np.asarray(target, np.float32)
    forward = _normalize((t - p).astype(np.float32))
    right = _cross(forward, np.asarray(up, np.float32))
    if math.sqrt(float(np.dot(right, right))) < 1e-6:
        right = _cross(forward, np.array([0, 0, 1], np.float32))
    right = _normalize(right)
    top = _cross(right, forward)
    # rotation columns: right, top, -forward; view = R^T, -R^T p
    r = np.stack([right, top, -forward], axis=1).astype(np.float32)  # r[row, col]
    m = np.zeros(16, np.float32)
    for row in range(3):
        for col in range(3):
            m[col * 4 + row] = r[col, row]
    for row in range(3):
        m[12 + row] = -(m[row] * p[0] + m[4 + row] * p[1] + m[8 + row] * p[2])
    m[15] = 1.0
    return m


def orbit_view(frame: int, radius: float = 15.0, degrees_per_frame: float = 3.0, height: float = 0.0,
               target=(0.0, 0.0, 0.0)):
    """Camera `frame` of an orbit around `target` in the y = height plane."""
    angle = math.radians(degrees_per_frame * frame)
    eye = np.array([radius * math.sin(angle), height, radius * math.cos(angle)], np.float32)
    return look_at_view(eye, target), eye
