"""splatkit_b200: Python mirror of the B200 splat renderer's C ABI (include/splatkit_b200.h).

The verbs follow the reference's renderer surface, ``splatkit::SplatRenderer``
(packages/splatkit-engine/include/splatkit/rendering/SplatRenderer.h:36-160): upload a
world (flat or LOD), apply a render policy, draw a frame, read back the image and the frame
statistics. Every call goes through ``libsplatkit_b200.so``; there is no other path. If the
library or a CUDA device is missing, constructing a :class:`Renderer` raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import camera  # noqa: F401  (re-exported helpers)

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = _HERE.parent / "libsplatkit_b200.so"

# status codes (include/splatkit_b200.h)
SK_OK = 0
SK_E_INVALID = 1
SK_E_OOM = 2
SK_E_ADMISSION = 3
SK_E_DEVICE = 4
SK_E_TIMEOUT = 5
SK_E_UNSUPPORTED = 6
SK_E_NO_WORLD = 7
SK_E_LIMIT = 8
STATUS_NAMES = {0: "ok", 1: "invalid", 2: "out of memory", 3: "admission", 4: "device",
                5: "timeout", 6: "unsupported", 7: "no world", 8: "beyond a fixed limit"}

FORMAT_RGBA8 = 0
FORMAT_RGBA32F = 1
FORMAT_BGRA8 = 2

PROJECTED_DTYPE = np.dtype([("center", "<f4", (2,)), ("axis1", "<u4"), ("axis2", "<u4"),
                            ("color0", "<u4"), ("color1", "<u4"), ("radius", "<f4"),
                            ("index", "<u4")])
LOD_NODE_DTYPE = np.dtype([("position", "<f4", (3,)), ("size", "<f4"),
                           ("child_start", "<u4"), ("child_count", "<u4")])
LOD_CLUSTER_DTYPE = np.dtype([("center", "<f4", (3,)), ("radius", "<f4"), ("extent", "<f4", (3,)),
                              ("error", "<f4"), ("color_variance", "<f4"), ("opacity", "<f4"),
                              ("node", "<u4"), ("child_start", "<u4"), ("child_count", "<u4"),
                              ("leaf_start", "<u4"), ("leaf_count", "<u4"),
                              ("subtree_leaves", "<u4")])
assert PROJECTED_DTYPE.itemsize == 32 and LOD_NODE_DTYPE.itemsize == 24
assert LOD_CLUSTER_DTYPE.itemsize == 64


class SplatError(RuntimeError):
    """A non-OK status from the C ABI; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


# ---- ctypes mirror of the ABI structs -----------------------------------------------------
_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)


class _Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("image_format", ctypes.c_int32), ("time_stages", ctypes.c_uint32)]


class _Cloud(ctypes.Structure):
    _fields_ = [("positions", _f32p), ("covariances", _f32p), ("colors", _f32p),
                ("alphas", _f32p), ("sh", _f32p), ("count", ctypes.c_uint32),
                ("sh_degree", ctypes.c_int32)]


class _LodView(ctypes.Structure):
    _fields_ = [("nodes", _Cloud), ("layout", ctypes.c_void_p), ("node_count", ctypes.c_uint32),
                ("leaf_count", ctypes.c_uint32), ("clusters", ctypes.c_void_p),
                ("cluster_count", ctypes.c_uint32), ("leaves", _u32p),
                ("leaf_ref_count", ctypes.c_uint32)]


class _Range(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_uint32), ("count", ctypes.c_uint32)]


class _Frame(ctypes.Structure):
    _fields_ = [("view", ctypes.c_float * 16), ("proj", ctypes.c_float * 16),
                ("camera_position", ctypes.c_float * 3), ("reveal_level", ctypes.c_float),
                ("ranges", ctypes.POINTER(_Range)), ("range_count", ctypes.c_uint32),
                ("sh_degree", ctypes.c_int32), ("reveal_band", ctypes.c_float),
                ("reveal_tint_amount", ctypes.c_float), ("reveal_brightness_boost", ctypes.c_float),
                ("reveal_tint", ctypes.c_float * 3)]


class _PartStyle(ctypes.Structure):
    _fields_ = [("tint", ctypes.c_float * 3), ("tint_amount", ctypes.c_float),
                ("brightness", ctypes.c_float), ("opacity", ctypes.c_float),
                ("reserved", ctypes.c_float * 2)]


class _BatchConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("lanes", ctypes.c_uint32),
                ("max_views", ctypes.c_uint32), ("use_graphs", ctypes.c_uint32)]


class _BatchView(ctypes.Structure):
    _fields_ = [("world", ctypes.c_void_p), ("frame", _Frame), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32)]


class _BatchStats(ctypes.Structure):
    _fields_ = [("views", ctypes.c_uint32), ("visible", ctypes.c_uint32),
                ("instances", ctypes.c_uint32), ("device_error", ctypes.c_uint32),
                ("gpu_ms", ctypes.c_double), ("fragments", ctypes.c_uint64)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("lanes", ctypes.c_uint32),
                ("max_batch_views", ctypes.c_uint32), ("max_batch_splats", ctypes.c_uint64),
                ("memory_budget", ctypes.c_uint64), ("max_queue_ms", ctypes.c_double)]


class _Request(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("frame", _Frame), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("image", ctypes.c_void_p)]


class _Completion(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("visible", ctypes.c_uint32),
                ("batch_views", ctypes.c_uint32), ("queue_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]


class _BatchTuning(ctypes.Structure):
    _fields_ = [("emission_balanced", ctypes.c_uint32), ("sort_tile_keys", ctypes.c_uint32),
                ("lanes", ctypes.c_uint32), ("sorted_lists", ctypes.c_uint32), ("gpu_ms", ctypes.c_double),
                ("views_per_s", ctypes.c_double)]


class _LodsplatHeader(ctypes.Structure):
    _fields_ = [("version", ctypes.c_uint32), ("node_count", ctypes.c_uint32),
                ("leaf_count", ctypes.c_uint32), ("sh_degree", ctypes.c_int32),
                ("depth", ctypes.c_uint32), ("cluster_count", ctypes.c_uint32),
                ("leaf_ref_count", ctypes.c_uint32), ("bounds_min", ctypes.c_float * 3),
                ("bounds_max", ctypes.c_float * 3)]


class _Policy(ctypes.Structure):
    _fields_ = [("lod_error_pixels", ctypes.c_float), ("lod_splat_limit", ctypes.c_uint32),
                ("alpha_threshold", ctypes.c_float), ("subpixel_threshold", ctypes.c_float),
                ("enable_frustum_culling", ctypes.c_uint32),
                ("enable_early_termination", ctypes.c_uint32),
                ("sort_depth_bits", ctypes.c_uint32), ("background", ctypes.c_double * 3)]


class _Caps(ctypes.Structure):
    _fields_ = [("max_lod_capacity_splats", ctypes.c_uint32),
                ("min_residency_capacity_splats", ctypes.c_uint32),
                ("max_residency_capacity_splats", ctypes.c_uint32),
                ("supports_subgroups", ctypes.c_uint32), ("max_texture_dimension", ctypes.c_uint32),
                ("sorts_on_gpu", ctypes.c_uint32), ("selects_lod_on_gpu", ctypes.c_uint32),
                ("total_memory", ctypes.c_uint64)]


class _Stats(ctypes.Structure):
    _fields_ = [("submitted_frames", ctypes.c_uint64), ("completed_frames", ctypes.c_uint64),
                ("gpu_ms", ctypes.c_double), ("select_ms", ctypes.c_double),
                ("cull_ms", ctypes.c_double), ("sort_ms", ctypes.c_double),
                ("bin_ms", ctypes.c_double), ("composite_ms", ctypes.c_double),
                ("draw_count", ctypes.c_uint32), ("selected_count", ctypes.c_uint32),
                ("lod_limited", ctypes.c_uint32), ("lod_evaluated", ctypes.c_uint32),
                ("instances", ctypes.c_uint32), ("device_error", ctypes.c_uint32),
                ("fragments", ctypes.c_uint64), ("lod_pixels", ctypes.c_float),
                ("instances_read", ctypes.c_uint32)]


# Every function the header declares, with its ctypes signature.
_SIGNATURES = {
    "sk_create": (ctypes.c_int32, [ctypes.POINTER(_Config), ctypes.POINTER(ctypes.c_void_p)]),
    "sk_destroy": (None, [ctypes.c_void_p]),
    "sk_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "sk_resize": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    "sk_device_capabilities": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Caps)]),
    "sk_apply_render_policy": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Policy)]),
    "sk_default_policy": (None, [ctypes.POINTER(_Policy)]),
    "sk_available_memory": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "sk_gpu_failed": (ctypes.c_int32, [ctypes.c_void_p]),
    "sk_upload_world": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Cloud), ctypes.c_int32]),
    "sk_upload_lod_world": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_LodView),
                                             ctypes.c_int32, ctypes.c_uint32]),
    "sk_create_slab": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32]),
    "sk_upload_tile": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(_Cloud)]),
    "sk_world_info": (ctypes.c_int32, [ctypes.c_void_p, _u32p, ctypes.POINTER(ctypes.c_int32)]),
    "sk_draw": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Frame)]),
    "sk_read_image": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                       ctypes.c_int32]),
    "sk_wait_idle": (ctypes.c_int32, [ctypes.c_void_p]),
    "sk_get_stats": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Stats)]),
    "sk_set_timing": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    "sk_set_binning": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    "sk_capture_next_frame": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                               ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    "sk_wait_capture": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64]),
    "sk_read_visible": (ctypes.c_int32, [ctypes.c_void_p, _u32p, ctypes.c_void_p, ctypes.c_uint32,
                                         _u32p]),
    "sk_read_order": (ctypes.c_int32, [ctypes.c_void_p, _u32p, ctypes.c_uint32, _u32p]),
    "sk_read_cut": (ctypes.c_int32, [ctypes.c_void_p, _u32p, ctypes.c_uint32, _u32p, _u32p]),
    "sk_read_tile_lists": (ctypes.c_int32, [ctypes.c_void_p, _u32p, _u32p, ctypes.c_uint32, _u32p]),
    "sk_sort_workspace_bytes": (ctypes.c_size_t, [ctypes.c_uint32]),
    "sk_sh_device_stride": (ctypes.c_uint32, [ctypes.c_int32]),
    "sk_pack_splats": (ctypes.c_int32, [ctypes.POINTER(_Cloud), ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_void_p]),
    "sk_pack_sh": (ctypes.c_int32, [ctypes.POINTER(_Cloud), ctypes.c_int32, ctypes.c_uint32,
                                    ctypes.c_uint32, _u32p, ctypes.c_uint32]),
    "sk_build_lod_selection": (ctypes.c_int32, [ctypes.POINTER(_LodView), ctypes.c_void_p,
                                                ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32,
                                                _u32p]),
    "sk_lod_depth": (ctypes.c_int64, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    "sk_world_bytes": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint64,
                                         ctypes.c_uint64, ctypes.c_uint64]),
    "sk_lod_threshold_update": (ctypes.c_float, [_f32p, ctypes.c_uint32, ctypes.c_uint32,
                                                 ctypes.c_uint32]),
    "sk_radix_argsort_device": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                 ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_size_t, ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    "sk_batch_create": (ctypes.c_int32, [ctypes.POINTER(_BatchConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "sk_batch_destroy": (None, [ctypes.c_void_p]),
    "sk_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "sk_batch_apply_render_policy": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Policy)]),
    "sk_batch_submit": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_BatchView), ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "sk_batch_poll": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]),
    "sk_batch_wait": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64]),
    "sk_batch_read_image": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                             ctypes.c_void_p, ctypes.c_size_t]),
    "sk_batch_view_visible": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                               ctypes.POINTER(ctypes.c_uint32)]),
    "sk_batch_get_stats": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(_BatchStats)]),
    "sk_batch_autotune": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_BatchView), ctypes.c_uint32,
                                           ctypes.POINTER(_BatchTuning)]),
    "sk_batch_set_tuning": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_BatchTuning)]),
    "sk_lodsplat_read_header": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(_LodsplatHeader)]),
    "sk_lodsplat_decode": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32] + [ctypes.c_void_p] * 8),
    "sk_upload_lodsplat": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32,
                                            ctypes.c_uint32]),
    "sk_upload_lodsplat_file": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_uint32]),
    "sk_write_lodsplat": (ctypes.c_int32, [ctypes.POINTER(_LodView), _f32p, _f32p, ctypes.c_char_p]),
    "sk_build_lod_tree_device": (ctypes.c_int32, [ctypes.POINTER(_Cloud), _f32p, _f32p, ctypes.c_uint32,
                                                  ctypes.c_uint32, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "sk_lod_tree_view": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_LodView), _f32p, _f32p]),
    "sk_lod_tree_free": (None, [ctypes.c_void_p]),
    "sk_upload_labels": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32]),
    "sk_set_part_styles": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_PartStyle), ctypes.c_void_p,
                                            ctypes.c_uint32]),
    "sk_server_create": (ctypes.c_int32, [ctypes.POINTER(_ServerConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "sk_server_destroy": (None, [ctypes.c_void_p]),
    "sk_server_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "sk_server_add_scene": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]),
    "sk_server_submit": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_uint64)]),
    "sk_server_take_completions": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Completion), ctypes.c_uint32,
                                                    ctypes.POINTER(ctypes.c_uint32)]),
    "sk_server_drain": (ctypes.c_int32, [ctypes.c_void_p]),
    "sk_server_replay": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_double),
                                          ctypes.c_uint32, ctypes.POINTER(_Completion)]),
    "sk_server_alloc_host": (ctypes.c_void_p, [ctypes.c_size_t]),
    "sk_server_free_host": (None, [ctypes.c_void_p]),
    "sk_radix_argsort_noalloc": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_uint32, ctypes.c_int32,
                                                  ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p]),
    # test hooks (include/splatkit_b200_testing.h)
    "sk_testing_fail_device_allocations": (None, [ctypes.c_uint32]),
    "sk_testing_fail_next_check": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32]),
    "sk_testing_withhold_sort_status": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
}

_lib: Optional[ctypes.CDLL] = None


def library() -> ctypes.CDLL:
    """Loads libsplatkit_b200.so (built in-tree by ``make -C splatkit-ios_b200``)."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise SplatError(SK_E_DEVICE, f"{LIBRARY_PATH} is not built")
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def exported_symbols() -> Sequence[str]:
    return tuple(_SIGNATURES)


def _ptr(a: Optional[np.ndarray], kind=_f32p):
    if a is None:
        return ctypes.cast(None, kind)
    return a.ctypes.data_as(kind)


# ---- world data ---------------------------------------------------------------------------
def sh_coefficients(degree: int) -> int:
    return 0 if degree <= 0 else (degree + 1) ** 2 - 1


@dataclass
class Cloud:
    """A SplatCloud (splat-core/include/splat/formats/SplatCloud.h:30-51), structure of arrays."""

    positions: np.ndarray  # (n, 3) float32
    covariances: np.ndarray  # (n, 6) float32: xx, xy, xz, yy, yz, zz
    colors: np.ndarray  # (n, 3) float32 in [0, 1]
    alphas: np.ndarray  # (n,) float32
    sh_degree: int = 0
    sh: Optional[np.ndarray] = None  # (n, 3 * coefficients) float32, channel fastest
    bounds_min: Optional[np.ndarray] = None
    bounds_max: Optional[np.ndarray] = None

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, np.float32).reshape(-1, 3)
        self.covariances = np.ascontiguousarray(self.covariances, np.float32).reshape(-1, 6)
        self.colors = np.ascontiguousarray(self.colors, np.float32).reshape(-1, 3)
        self.alphas = np.ascontiguousarray(self.alphas, np.float32).reshape(-1)
        if self.sh is not None:
            self.sh = np.ascontiguousarray(self.sh, np.float32).reshape(len(self.alphas), -1)

    @property
    def count(self) -> int:
        return int(self.alphas.shape[0])

    def view(self) -> _Cloud:
        return _Cloud(_ptr(self.positions), _ptr(self.covariances), _ptr(self.colors),
                      _ptr(self.alphas), _ptr(self.sh if self.sh_degree > 0 else None),
                      self.count, self.sh_degree)


@dataclass
class LodTree:
    """A LodTree (splat-core/include/splat/lod/LodTree.h:47-55): nodes in layout order."""

    nodes: Cloud
    layout: np.ndarray  # LOD_NODE_DTYPE
    leaf_count: int
    clusters: Optional[np.ndarray] = None  # LOD_CLUSTER_DTYPE
    leaves: Optional[np.ndarray] = None  # uint32 leaf references

    def view(self) -> _LodView:
        layout = np.ascontiguousarray(self.layout)
        self._keep = [layout]
        clusters = None if self.clusters is None else np.ascontiguousarray(self.clusters)
        leaves = None if self.leaves is None else np.ascontiguousarray(self.leaves, np.uint32)
        self._keep += [clusters, leaves]
        return _LodView(self.nodes.view(), layout.ctypes.data, len(layout), self.leaf_count,
                        None if clusters is None else clusters.ctypes.data,
                        0 if clusters is None else len(clusters),
                        _ptr(leaves, _u32p), 0 if leaves is None else len(leaves))


@dataclass
class Policy:
    """RenderPolicy (splatkit-engine/include/splatkit/rendering/RenderPolicy.h:17-40)."""

    lod_error_pixels: float = 1.0
    lod_splat_limit: int = 0
    alpha_threshold: float = 1.0 / 255.0
    subpixel_threshold: float = 1.0
    enable_frustum_culling: bool = True
    enable_early_termination: bool = True
    sort_depth_bits: int = 16
    background: tuple = (0.05, 0.05, 0.08)

    def native(self) -> _Policy:
        p = _Policy()
        p.lod_error_pixels = self.lod_error_pixels
        p.lod_splat_limit = self.lod_splat_limit
        p.alpha_threshold = self.alpha_threshold
        p.subpixel_threshold = self.subpixel_threshold
        p.enable_frustum_culling = int(self.enable_frustum_culling)
        p.enable_early_termination = int(self.enable_early_termination)
        p.sort_depth_bits = self.sort_depth_bits
        for i in range(3):
            p.background[i] = float(self.background[i])
        return p


@dataclass
class Frame:
    """SplatRenderer::Frame (SplatRenderer.h:111-131) for the GPU order source."""

    view: np.ndarray  # (16,) column major
    proj: np.ndarray  # (16,) column major
    camera_position: np.ndarray  # (3,)
    ranges: Sequence[tuple] = ()
    sh_degree: int = 0
    reveal_level: float = float("inf")
    reveal_band: float = 0.0  # RevealUniform (Reveal.h:25-35); 0: no glow
    reveal_tint_amount: float = 0.0
    reveal_brightness_boost: float = 0.0
    reveal_tint: Sequence[float] = (1.0, 1.0, 1.0)

    def native(self):
        f = _Frame()
        view = np.asarray(self.view, np.float32).reshape(16)
        proj = np.asarray(self.proj, np.float32).reshape(16)
        for i in range(16):
            f.view[i] = float(view[i])
            f.proj[i] = float(proj[i])
        pos = np.asarray(self.camera_position, np.float32).reshape(3)
        for i in range(3):
            f.camera_position[i] = float(pos[i])
        f.reveal_level = self.reveal_level
        f.reveal_band = self.reveal_band
        f.reveal_tint_amount = self.reveal_tint_amount
        f.reveal_brightness_boost = self.reveal_brightness_boost
        for i in range(3):
            f.reveal_tint[i] = float(self.reveal_tint[i])
        ranges = (_Range * max(1, len(self.ranges)))(*[_Range(int(o), int(c)) for o, c in self.ranges])
        f.ranges = ctypes.cast(ranges, ctypes.POINTER(_Range)) if len(self.ranges) else None
        f.range_count = len(self.ranges)
        f.sh_degree = self.sh_degree
        return f, ranges


# ---- the renderer -------------------------------------------------------------------------
class Renderer:
    """A headless splat renderer on one CUDA device (``CudaSplatRenderer``'s Python mirror)."""

    def __init__(self, width: int, height: int, device: int = 0, image_format: int = FORMAT_RGBA8,
                 time_stages: bool | str = True):
        # True: per-stage events; "frame": the frame's own pair only (stage kernels stay chained)
        self._lib = library()
        timing = 2 if time_stages == "frame" else (1 if time_stages else 0)
        cfg = _Config(device, width, height, image_format, timing)
        handle = ctypes.c_void_p()
        st = self._lib.sk_create(ctypes.byref(cfg), ctypes.byref(handle))
        if st != SK_OK:
            raise SplatError(st, "sk_create failed (is a CUDA device visible?)")
        self._h = handle
        self.width, self.height, self.image_format = width, height, image_format
        self._captures = {}

    # lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._lib.sk_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != SK_OK:
            msg = self._lib.sk_last_error(self._h)
            raise SplatError(st, f"{what}: {msg.decode() if msg else ''}")

    # SplatRenderer verbs
    def resize(self, width: int, height: int):
        self._check(self._lib.sk_resize(self._h, width, height), "resize")
        self.width, self.height = width, height

    def device_capabilities(self) -> dict:
        caps = _Caps()
        self._check(self._lib.sk_device_capabilities(self._h, ctypes.byref(caps)), "capabilities")
        return {name: getattr(caps, name) for name, _ in _Caps._fields_}

    def apply_render_policy(self, policy: Policy):
        p = policy.native()
        self._check(self._lib.sk_apply_render_policy(self._h, ctypes.byref(p)), "policy")

    def set_binning(self, mode: str):
        """"auto": cell lists written in place on targets of up to 4096 cells, else sorted;
        "sorted": always the stable (cell, splat) sort. Both give the same lists."""
        code = {"auto": 0, "sorted": 1}[mode]
        self._check(self._lib.sk_set_binning(self._h, code), "binning")

    def set_timing(self, time_stages: bool | str):
        """True: per-stage events; "frame": the frame's own pair only; False: none."""
        timing = 2 if time_stages == "frame" else (1 if time_stages else 0)
        self._check(self._lib.sk_set_timing(self._h, timing), "timing")

    def available_memory(self) -> int:
        v = ctypes.c_uint64()
        self._check(self._lib.sk_available_memory(self._h, ctypes.byref(v)), "memory")
        return v.value

    def gpu_failed(self) -> bool:
        return bool(self._lib.sk_gpu_failed(self._h))

    def upload_world(self, cloud: Cloud, max_sh_degree: int = 3):
        v = cloud.view()
        self._check(self._lib.sk_upload_world(self._h, ctypes.byref(v), max_sh_degree), "upload")

    def upload_lod_world(self, tree: LodTree, max_sh_degree: int, budget: int):
        v = tree.view()
        self._check(self._lib.sk_upload_lod_world(self._h, ctypes.byref(v), max_sh_degree, budget),
                    "LOD upload")

    def upload_lodsplat(self, source, max_sh_degree: int, budget: int):
        """A .lodsplat file (a path, read by mapping it) or its bytes, decoded and uploaded."""
        if isinstance(source, (bytes, bytearray, memoryview)):
            buf = np.frombuffer(source, np.uint8)
            self._check(self._lib.sk_upload_lodsplat(self._h, buf.ctypes.data, len(buf), max_sh_degree,
                                                     budget), "lodsplat upload")
        else:
            self._check(self._lib.sk_upload_lodsplat_file(self._h, os.fsencode(str(source)), max_sh_degree,
                                                          budget), "lodsplat upload")

    def upload_labels(self, labels: np.ndarray, offset: int = 0):
        """Part labels (uint16) of world records [offset, offset + len(labels))."""
        lab = np.ascontiguousarray(labels, np.uint16)
        self._check(self._lib.sk_upload_labels(self._h, offset, lab.ctypes.data, len(lab)), "labels")

    def set_part_styles(self, palette, states):
        """palette: up to 10 (tint rgb, tint_amount, brightness, opacity); states[label] -> entry."""
        pal = (_PartStyle * 10)()
        for i in range(10):
            pal[i].tint[0] = pal[i].tint[1] = pal[i].tint[2] = 1.0
            pal[i].tint_amount, pal[i].brightness, pal[i].opacity = 0.0, 1.0, 1.0
        for i, entry in enumerate(palette):
            tint, amount, brightness, opacity = entry
            for j in range(3):
                pal[i].tint[j] = float(tint[j])
            pal[i].tint_amount, pal[i].brightness, pal[i].opacity = amount, brightness, opacity
        st = np.ascontiguousarray(states, np.uint32)
        self._check(self._lib.sk_set_part_styles(self._h, pal, st.ctypes.data if len(st) else None,
                                                 len(st)), "part styles")

    def create_slab(self, capacity: int, sh_degree: int):
        self._check(self._lib.sk_create_slab(self._h, capacity, sh_degree), "slab")

    def upload_tile(self, offset: int, cloud: Cloud):
        v = cloud.view()
        self._check(self._lib.sk_upload_tile(self._h, offset, ctypes.byref(v)), "tile")

    def testing_fail_next_check(self, cuda_error: int):
        """Test hook: the next CUDA status this context checks reads as `cuda_error`."""
        self._check(self._lib.sk_testing_fail_next_check(self._h, cuda_error), "testing")

    def testing_withhold_sort_status(self, tile: int):
        """Test hook: in the next frame, depth-sort tile `tile` publishes no look-back status."""
        self._check(self._lib.sk_testing_withhold_sort_status(self._h, tile), "testing")

    def world(self):
        n = ctypes.c_uint32()
        d = ctypes.c_int32()
        st = self._lib.sk_world_info(self._h, ctypes.byref(n), ctypes.byref(d))
        if st == SK_E_NO_WORLD:
            return None
        self._check(st, "world")
        return n.value, d.value

    def draw(self, frame: Frame):
        f, keep = frame.native()
        self._check(self._lib.sk_draw(self._h, ctypes.byref(f)), "draw")
        del keep

    def wait_idle(self):
        self._check(self._lib.sk_wait_idle(self._h), "wait")

    def capture_next_frame(self, out: np.ndarray) -> int:
        """captureNextFrame: the next draw's image is copied into `out` (the context's pixel
        format; pinned memory lets the copy overlap later frames). Returns a ticket for
        wait_capture; `out` must stay alive and untouched until then."""
        fmt = self.image_format
        need = self.width * self.height * (16 if fmt == FORMAT_RGBA32F else 4)
        if not out.flags["C_CONTIGUOUS"] or out.nbytes < need:
            raise SplatError(SK_E_INVALID, "capture buffer too small or not contiguous")
        t = ctypes.c_uint64()
        self._check(self._lib.sk_capture_next_frame(self._h, out.ctypes.data, out.nbytes, fmt,
                                                    ctypes.byref(t)), "capture")
        self._captures[t.value] = out
        return t.value

    def wait_capture(self, ticket: int) -> np.ndarray:
        """Blocks until the captured frame's image is in its buffer; returns the buffer."""
        self._check(self._lib.sk_wait_capture(self._h, ticket), "capture wait")
        return self._captures.pop(ticket, None)

    def read_image(self, fmt: int = None, out: Optional[np.ndarray] = None) -> np.ndarray:
        fmt = self.image_format if fmt is None else fmt
        if out is None:
            if fmt == FORMAT_RGBA32F:
                out = np.empty((self.height, self.width, 4), np.float32)
            else:
                out = np.empty((self.height, self.width, 4), np.uint8)
        self._check(self._lib.sk_read_image(self._h, out.ctypes.data, out.nbytes, fmt), "read image")
        return out

    def stats(self) -> dict:
        s = _Stats()
        self._check(self._lib.sk_get_stats(self._h, ctypes.byref(s)), "stats")
        return {name: getattr(s, name) for name, _ in _Stats._fields_}

    def read_visible(self):
        n = ctypes.c_uint32()
        self._check(self._lib.sk_read_visible(self._h, None, None, 0, ctypes.byref(n)), "visible")
        keys = np.empty(n.value, np.uint32)
        proj = np.empty(n.value, PROJECTED_DTYPE)
        self._check(self._lib.sk_read_visible(self._h, _ptr(keys, _u32p), proj.ctypes.data,
                                              n.value, ctypes.byref(n)), "visible")
        return keys, proj

    def read_order(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(self._lib.sk_read_order(self._h, None, 0, ctypes.byref(n)), "order")
        order = np.empty(n.value, np.uint32)
        self._check(self._lib.sk_read_order(self._h, _ptr(order, _u32p), n.value,
                                            ctypes.byref(n)), "order")
        return order

    def read_tile_lists(self):
        """(ranges (cells, 2), values): each 32x32 binning cell's front-to-back projected indices
        (a composite tile of 16x16 pixels reads the list of the cell it lies in)."""
        cells = ((self.width + 31) // 32) * ((self.height + 31) // 32)
        ranges = np.zeros((cells, 2), np.uint32)
        n = ctypes.c_uint32()
        self._check(self._lib.sk_read_tile_lists(self._h, _ptr(ranges, _u32p), None, 0,
                                                 ctypes.byref(n)), "tile lists")
        values = np.empty(n.value, np.uint32)
        self._check(self._lib.sk_read_tile_lists(self._h, _ptr(ranges, _u32p), _ptr(values, _u32p),
                                                 n.value, ctypes.byref(n)), "tile lists")
        return ranges, values

    def read_cut(self):
        n = ctypes.c_uint32()
        stats = np.zeros(6, np.uint32)
        self._check(self._lib.sk_read_cut(self._h, None, 0, ctypes.byref(n), _ptr(stats, _u32p)),
                    "cut")
        cut = np.empty(n.value, np.uint32)
        self._check(self._lib.sk_read_cut(self._h, _ptr(cut, _u32p), n.value, ctypes.byref(n),
                                          _ptr(stats, _u32p)), "cut")
        return cut, stats


# ---- batched multi-view rendering ----------------------------------------------------------
class BatchView:
    """One view of a batch: the renderer whose resident world it draws, the frame, the size."""

    def __init__(self, renderer: "Renderer", frame: Frame, width: int, height: int):
        self.renderer, self.frame, self.width, self.height = renderer, frame, width, height


class Batch:
    """Many views drawn together (sk_batch_*): every stage runs once over the whole batch.

    ``submit`` returns a ticket at once; results stay readable until the lane that ran the
    ticket is reused, ``lanes`` submissions later."""

    def __init__(self, device: int = 0, lanes: int = 2, max_views: int = 64, use_graphs: bool = False):
        self._lib = library()
        cfg = _BatchConfig(device, lanes, max_views, 1 if use_graphs else 0)
        handle = ctypes.c_void_p()
        st = self._lib.sk_batch_create(ctypes.byref(cfg), ctypes.byref(handle))
        if st != SK_OK:
            raise SplatError(st, "sk_batch_create failed (is a CUDA device visible?)")
        self._h = handle
        self._sizes = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sk_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != SK_OK:
            msg = self._lib.sk_batch_last_error(self._h)
            raise SplatError(st, f"{what}: {msg.decode() if msg else ''}")

    def apply_render_policy(self, policy: Policy):
        p = policy.native()
        self._check(self._lib.sk_batch_apply_render_policy(self._h, ctypes.byref(p)), "policy")

    def submit(self, views: Sequence[BatchView]) -> int:
        arr = (_BatchView * len(views))()
        keep = []
        for i, v in enumerate(views):
            f, ranges = v.frame.native()
            keep.append(ranges)
            arr[i].world = v.renderer._h
            arr[i].frame = f
            arr[i].width, arr[i].height = v.width, v.height
        ticket = ctypes.c_uint64()
        self._check(self._lib.sk_batch_submit(self._h, arr, len(views), ctypes.byref(ticket)), "submit")
        self._sizes[ticket.value] = [(v.width, v.height) for v in views]
        if len(self._sizes) > 64:
            self._sizes.pop(next(iter(self._sizes)))
        return ticket.value

    @staticmethod
    def _views(views):
        arr = (_BatchView * len(views))()
        keep = []
        for i, v in enumerate(views):
            f, ranges = v.frame.native()
            keep.append(ranges)
            arr[i].world = v.renderer._h
            arr[i].frame = f
            arr[i].width, arr[i].height = v.width, v.height
        return arr, keep

    def autotune(self, views: Sequence[BatchView]) -> dict:
        """Times the sample under every launch shape and keeps the fastest (sk_batch_autotune)."""
        arr, keep = self._views(views)
        t = _BatchTuning()
        self._check(self._lib.sk_batch_autotune(self._h, arr, len(views), ctypes.byref(t)), "autotune")
        return {name: getattr(t, name) for name, _ in _BatchTuning._fields_}

    def set_tuning(self, emission_balanced: int, sort_tile_keys: int, lanes: int, sorted_lists: int = 0):
        t = _BatchTuning(emission_balanced, sort_tile_keys, lanes, sorted_lists, 0.0, 0.0)
        self._check(self._lib.sk_batch_set_tuning(self._h, ctypes.byref(t)), "set_tuning")

    def poll(self, ticket: int) -> bool:
        done = ctypes.c_int32()
        self._check(self._lib.sk_batch_poll(self._h, ticket, ctypes.byref(done)), "poll")
        return bool(done.value)

    def wait(self, ticket: int):
        self._check(self._lib.sk_batch_wait(self._h, ticket), "wait")

    def read_image(self, ticket: int, view: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        w, h = self._sizes[ticket][view]
        if out is None:
            out = np.empty((h, w, 4), np.uint8)
        self._check(self._lib.sk_batch_read_image(self._h, ticket, view, out.ctypes.data, out.nbytes),
                    "read_image")
        return out

    def view_visible(self, ticket: int, view: int) -> int:
        n = ctypes.c_uint32()
        self._check(self._lib.sk_batch_view_visible(self._h, ticket, view, ctypes.byref(n)), "visible")
        return n.value

    def stats(self, ticket: int) -> dict:
        st = _BatchStats()
        self._check(self._lib.sk_batch_get_stats(self._h, ticket, ctypes.byref(st)), "stats")
        return {name: getattr(st, name) for name, _ in _BatchStats._fields_}


# ---- serving ---------------------------------------------------------------------------------
class HostImage:
    """A pinned host image buffer (sk_server_alloc_host) viewed as an (h, w, 4) uint8 array."""

    def __init__(self, width: int, height: int):
        self._lib = library()
        self.nbytes = width * height * 4
        self.ptr = self._lib.sk_server_alloc_host(self.nbytes)
        if not self.ptr:
            raise SplatError(SK_E_OOM, "pinned host allocation failed")
        buf = (ctypes.c_uint8 * self.nbytes).from_address(self.ptr)
        self.array = np.frombuffer(buf, np.uint8).reshape(height, width, 4)

    def close(self):
        if getattr(self, "ptr", None):
            self.array = None
            self._lib.sk_server_free_host(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Request:
    """One render request: scene index, frame, size, and the host image it is written into."""

    def __init__(self, scene: int, frame: Frame, width: int, height: int,
                 image: Optional[HostImage] = None):
        self.scene, self.frame, self.width, self.height, self.image = scene, frame, width, height, image

    def native(self):
        f, ranges = self.frame.native()
        r = _Request()
        r.scene, r.frame, r.width, r.height = self.scene, f, self.width, self.height
        r.image = self.image.ptr if self.image is not None else None
        return r, ranges


COMPLETION_FIELDS = [name for name, _ in _Completion._fields_]


class Server:
    """Continuous-batching render server over resident scenes (sk_server_*)."""

    def __init__(self, device: int = 0, lanes: int = 2, max_batch_views: int = 64,
                 max_batch_splats: int = 64_000_000, memory_budget: int = 120 << 30,
                 max_queue_ms: float = 0.0):
        self._lib = library()
        cfg = _ServerConfig(device, lanes, max_batch_views, max_batch_splats, memory_budget, max_queue_ms)
        handle = ctypes.c_void_p()
        st = self._lib.sk_server_create(ctypes.byref(cfg), ctypes.byref(handle))
        if st != SK_OK:
            raise SplatError(st, "sk_server_create failed (is a CUDA device visible?)")
        self._h = handle
        self._scenes = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sk_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != SK_OK:
            msg = self._lib.sk_server_last_error(self._h)
            raise SplatError(st, f"{what}: {msg.decode() if msg else ''}")

    def add_scene(self, renderer: "Renderer") -> int:
        idx = ctypes.c_uint32()
        self._check(self._lib.sk_server_add_scene(self._h, renderer._h, ctypes.byref(idx)), "add_scene")
        self._scenes.append(renderer)
        return idx.value

    def submit(self, request: Request) -> int:
        r, keep = request.native()
        rid = ctypes.c_uint64()
        self._check(self._lib.sk_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)), "submit")
        return rid.value

    def drain(self):
        self._check(self._lib.sk_server_drain(self._h), "drain")

    def take_completions(self, capacity: int = 4096) -> list:
        out = (_Completion * capacity)()
        n = ctypes.c_uint32()
        self._check(self._lib.sk_server_take_completions(self._h, out, capacity, ctypes.byref(n)), "take")
        return [{k: getattr(out[i], k) for k in COMPLETION_FIELDS} for i in range(n.value)]

    def replay(self, requests: Sequence[Request], arrival_us: Sequence[float]) -> list:
        """Submits request i at arrival_us[i] after the call starts; returns the completions."""
        arr = (_Request * len(requests))()
        keep = []
        for i, req in enumerate(requests):
            r, ranges = req.native()
            keep.append(ranges)
            arr[i] = r
        times = (ctypes.c_double * len(requests))(*[float(t) for t in arrival_us])
        out = (_Completion * len(requests))()
        self._check(self._lib.sk_server_replay(self._h, arr, times, len(requests), out), "replay")
        return [{k: getattr(out[i], k) for k in COMPLETION_FIELDS} for i in range(len(requests))]


# ---- .lodsplat files -------------------------------------------------------------------------
def lodsplat_header(data: bytes) -> dict:
    """readLodSplatHeader: the header fields, or SplatError when the file is not valid."""
    buf = np.frombuffer(data, np.uint8)
    h = _LodsplatHeader()
    st = library().sk_lodsplat_read_header(buf.ctypes.data, len(buf), ctypes.byref(h))
    if st != SK_OK:
        raise SplatError(st, "not a valid LODSPLAT header")
    out = {name: getattr(h, name) for name, _ in _LodsplatHeader._fields_}
    out["bounds_min"], out["bounds_max"] = list(h.bounds_min), list(h.bounds_max)
    return out


def lodsplat_decode(data: bytes, max_sh_degree: int = 3) -> LodTree:
    """decodeLodSplat into a LodTree (selection data from a version-2 file)."""
    hd = lodsplat_header(data)
    n, degree = hd["node_count"], min(hd["sh_degree"], max(0, min(max_sh_degree, 3)))
    coeffs = 3 * ((degree + 1) ** 2 - 1)
    pos, cov = np.empty((n, 3), np.float32), np.empty((n, 6), np.float32)
    col, alp = np.empty((n, 3), np.float32), np.empty(n, np.float32)
    sh = np.empty((n, coeffs), np.float32) if coeffs else None
    layout = np.empty(n, LOD_NODE_DTYPE)
    clusters = np.empty(hd["cluster_count"], LOD_CLUSTER_DTYPE) if hd["cluster_count"] else None
    leaves = np.empty(hd["leaf_ref_count"], np.uint32) if hd["leaf_ref_count"] else None
    buf = np.frombuffer(data, np.uint8)
    ptrs = [a.ctypes.data if a is not None else None for a in (pos, cov, col, alp, sh, layout, clusters, leaves)]
    st = library().sk_lodsplat_decode(buf.ctypes.data, len(buf), max_sh_degree, *ptrs)
    if st != SK_OK:
        raise SplatError(st, "LODSPLAT rejected")
    cloud = Cloud(pos, cov, col, alp, sh_degree=degree, sh=sh,
                  bounds_min=np.array(hd["bounds_min"], np.float32),
                  bounds_max=np.array(hd["bounds_max"], np.float32))
    return LodTree(cloud, layout, hd["leaf_count"], clusters, leaves)


class _TreeMemory:
    """Owns one built tree (sk_lod_tree); the numpy views of its arrays keep it alive, and it is
    freed with the last of them."""

    def __init__(self, lib, handle: int):
        self._free = lib.sk_lod_tree_free
        self.handle = handle

    def __del__(self):
        if self.handle:
            self._free(self.handle)
            self.handle = None


class _TreeArray:
    """The array interface of one array of a built tree (no copy, read only: the memory belongs
    to the library), holding the tree."""

    def __init__(self, owner: _TreeMemory, ptr: int, dtype, shape):
        self._owner = owner
        dt = np.dtype(dtype)
        self.__array_interface__ = {"version": 3, "data": (ptr, True), "shape": tuple(shape),
                                    "typestr": dt.str, "descr": dt.descr}


def _tree_array(owner: _TreeMemory, ptr, dtype, shape) -> Optional[np.ndarray]:
    if not ptr or int(np.prod(shape)) == 0:
        return None
    return np.asarray(_TreeArray(owner, int(ptr), dtype, shape))


def build_lod_tree(cloud: Cloud, bounds_min=None, bounds_max=None, octree_depth: int = 0,
                   cluster_leaves: int = 0, selection: bool = True) -> LodTree:
    """buildLodTree on the current GPU (sk_build_lod_tree_device): bounds default to the cloud's,
    else the positions' own box. The reference builder's layout, attributes within a few ulp."""
    lib = library()
    entry = "sk_build_lod_tree_device"
    lo = bounds_min if bounds_min is not None else cloud.bounds_min
    hi = bounds_max if bounds_max is not None else cloud.bounds_max
    lo = None if lo is None else np.ascontiguousarray(lo, np.float32)
    hi = None if hi is None else np.ascontiguousarray(hi, np.float32)
    v = cloud.view()
    handle = ctypes.c_void_p()
    st = getattr(lib, entry)(ctypes.byref(v), _ptr(lo), _ptr(hi), octree_depth, cluster_leaves,
                             1 if selection else 0, ctypes.byref(handle))
    if st != SK_OK:
        raise SplatError(st, entry)
    owner = _TreeMemory(lib, handle.value)  # the arrays below are views of the tree's own memory
    t = _LodView()
    bmin, bmax = np.zeros(3, np.float32), np.zeros(3, np.float32)
    st = lib.sk_lod_tree_view(handle, ctypes.byref(t), _ptr(bmin), _ptr(bmax))
    if st != SK_OK:
        raise SplatError(st, "sk_lod_tree_view")
    n, d = t.node_count, t.nodes.sh_degree
    coeffs = 3 * ((d + 1) ** 2 - 1)
    addr = lambda p: ctypes.cast(p, ctypes.c_void_p).value
    nodes = Cloud(_tree_array(owner, addr(t.nodes.positions), np.float32, (n, 3)),
                  _tree_array(owner, addr(t.nodes.covariances), np.float32, (n, 6)),
                  _tree_array(owner, addr(t.nodes.colors), np.float32, (n, 3)),
                  _tree_array(owner, addr(t.nodes.alphas), np.float32, (n,)),
                  sh_degree=d,
                  sh=_tree_array(owner, addr(t.nodes.sh), np.float32, (n, coeffs)) if coeffs else None,
                  bounds_min=bmin, bounds_max=bmax)
    layout = _tree_array(owner, t.layout, LOD_NODE_DTYPE, (n,))
    clusters = _tree_array(owner, t.clusters, LOD_CLUSTER_DTYPE, (t.cluster_count,))
    leaves = _tree_array(owner, addr(t.leaves), np.uint32, (t.leaf_ref_count,))
    return LodTree(nodes, layout, t.leaf_count, clusters, leaves)


def write_lodsplat(tree: LodTree, path):
    """writeLodSplat: version 2 when the tree has selection data; refuses an existing path."""
    bmin = tree.nodes.bounds_min if tree.nodes.bounds_min is not None else np.zeros(3, np.float32)
    bmax = tree.nodes.bounds_max if tree.nodes.bounds_max is not None else np.zeros(3, np.float32)
    bmin, bmax = np.ascontiguousarray(bmin, np.float32), np.ascontiguousarray(bmax, np.float32)
    v = tree.view()
    st = library().sk_write_lodsplat(ctypes.byref(v), _ptr(bmin), _ptr(bmax), os.fsencode(str(path)))
    if st != SK_OK:
        raise SplatError(st, f"cannot write {path}")


def radix_argsort_device(keys_ptr: int, count_ptr: int, capacity: int, bits: int, order_ptr: int,
                         workspace_ptr: int, workspace_bytes: int, error_ptr: int, stream: int = 0):
    """The standalone sort operator over caller device memory (MetalRadixSort's contract)."""
    st = library().sk_radix_argsort_device(keys_ptr, count_ptr, capacity, bits, order_ptr,
                                           workspace_ptr, workspace_bytes, error_ptr, stream)
    if st != SK_OK:
        raise SplatError(st, "sk_radix_argsort_device")


NOALLOC_SORT_MAX_KEYS = 1 << 20  # SK_NOALLOC_SORT_MAX_KEYS


def radix_argsort_noalloc(keys_ptr: int, count_ptr: int, capacity: int, bits: int, order_ptr: int,
                          error_ptr: int, stream: int = 0):
    """The same sort with its workspace in the library's fixed device array: no allocation,
    capacity at most NOALLOC_SORT_MAX_KEYS (SK_E_LIMIT beyond), calls on one device ordered."""
    st = library().sk_radix_argsort_noalloc(keys_ptr, count_ptr, capacity, bits, order_ptr,
                                            error_ptr, stream)
    if st != SK_OK:
        raise SplatError(st, "sk_radix_argsort_noalloc")


def testing_fail_device_allocations(count: int):
    """Test hook: the next `count` device allocations of the library fail as out of memory."""
    library().sk_testing_fail_device_allocations(count)


def sort_workspace_bytes(capacity: int) -> int:
    return int(library().sk_sort_workspace_bytes(capacity))


# ---- host-side world preparation (no device needed) -----------------------------------------
SPLAT_DTYPE = np.dtype([("position", "<f4", (3,)), ("rgba8", "<u4"), ("cov", "<u4", (3,)),
                        ("lodAlpha", "<u4")])


def sh_device_stride(degree: int) -> int:
    return int(library().sk_sh_device_stride(degree))


def pack_splats(cloud: Cloud) -> np.ndarray:
    """The 32-byte GPU records of a cloud (GpuLayout.cpp:122-137)."""
    out = np.empty(cloud.count, SPLAT_DTYPE)
    v = cloud.view()
    st = library().sk_pack_splats(ctypes.byref(v), 0, cloud.count, out.ctypes.data)
    if st != SK_OK:
        raise SplatError(st, "sk_pack_splats")
    return out


def pack_sh(cloud: Cloud, degree: int, stride: Optional[int] = None) -> np.ndarray:
    """Harmonics halves, channel fastest, `stride` words per splat (GpuLayout.cpp:92-113)."""
    stride = sh_device_stride(degree) if stride is None else stride
    out = np.zeros((cloud.count, max(stride, 1)), np.uint32)
    v = cloud.view()
    st = library().sk_pack_sh(ctypes.byref(v), degree, 0, cloud.count, _ptr(out, _u32p), stride)
    if st != SK_OK:
        raise SplatError(st, "sk_pack_sh")
    return out[:, :stride]


def build_lod_selection(tree: LodTree):
    """The interior clusters and leaf references of a tree (LodSelection.cpp:47-133)."""
    v = tree.view()
    nc, nl = ctypes.c_uint32(), ctypes.c_uint32()
    lib = library()
    st = lib.sk_build_lod_selection(ctypes.byref(v), None, 0, ctypes.byref(nc), None, 0,
                                    ctypes.byref(nl))
    if st != SK_OK:
        raise SplatError(st, "sk_build_lod_selection")
    clusters = np.empty(nc.value, LOD_CLUSTER_DTYPE)
    leaves = np.empty(nl.value, np.uint32)
    st = lib.sk_build_lod_selection(ctypes.byref(v), clusters.ctypes.data, nc.value,
                                    ctypes.byref(nc), _ptr(leaves, _u32p), nl.value,
                                    ctypes.byref(nl))
    if st != SK_OK:
        raise SplatError(st, "sk_build_lod_selection")
    return clusters, leaves


def lod_depth(layout: np.ndarray, leaf_count: int) -> int:
    layout = np.ascontiguousarray(layout, LOD_NODE_DTYPE)
    return int(library().sk_lod_depth(layout.ctypes.data, len(layout), leaf_count))


def world_bytes(records: int, sh_degree: int, draw_capacity: int, clusters: int = 0,
                leaf_refs: int = 0) -> int:
    return int(library().sk_world_bytes(records, sh_degree, draw_capacity, clusters, leaf_refs))


def lod_threshold_update(state: np.ndarray, selected: int, limited: int, limit: int) -> float:
    """state: float32[2] = (policy pixels, current pixels), updated in place."""
    return float(library().sk_lod_threshold_update(_ptr(state), selected, limited, limit))
