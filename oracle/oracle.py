"""Test infrastructure only: numpy bindings of the CPU oracle.

  Oracle     liboracle.so   - the project's restatement of the reference's per-frame shader
                              math (oracle/splat_oracle.cpp; see splat_oracle.h for the
                              reference lines each function follows).
  Reference  _ref/libsk_ref.so - the reference's own C++ (splat-core, splatkit-engine) compiled
                              unmodified by oracle/Makefile, behind oracle/ref_shim.cpp.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module; the product
never does.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libsk_ref.so"

PROJECTED_DTYPE = np.dtype([("center", "<f4", (2,)), ("axis1", "<u4"), ("axis2", "<u4"),
                            ("color0", "<u4"), ("color1", "<u4"), ("radius", "<f4"),
                            ("index", "<u4")])
SPLAT_DTYPE = np.dtype([("position", "<f4", (3,)), ("rgba8", "<u4"), ("cov", "<u4", (3,)),
                        ("lodAlpha", "<u4")])
LOD_NODE_DTYPE = np.dtype([("position", "<f4", (3,)), ("size", "<f4"),
                           ("child_start", "<u4"), ("child_count", "<u4")])
LOD_CLUSTER_DTYPE = np.dtype([("center", "<f4", (3,)), ("radius", "<f4"), ("extent", "<f4", (3,)),
                              ("error", "<f4"), ("color_variance", "<f4"), ("opacity", "<f4"),
                              ("node", "<u4"), ("child_start", "<u4"), ("child_count", "<u4"),
                              ("leaf_start", "<u4"), ("leaf_count", "<u4"),
                              ("subtree_leaves", "<u4")])


class Camera(ctypes.Structure):
    """sko_camera: the 208-byte per-view uniform (metal/layout/SplatTypes.metalh:7-22)."""

    _fields_ = [("view", ctypes.c_float * 16), ("proj", ctypes.c_float * 16),
                ("focal", ctypes.c_float * 2), ("tanHalfFov", ctypes.c_float * 2),
                ("screenSize", ctypes.c_float * 2), ("outputLinear", ctypes.c_uint32),
                ("minPixelRadius", ctypes.c_float), ("cameraPosition", ctypes.c_float * 4),
                ("reveal", ctypes.c_float * 4), ("revealTint", ctypes.c_float * 4)]


assert ctypes.sizeof(Camera) == 208

_vp = ctypes.c_void_p


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


class Oracle:
    def __init__(self):
        if not ORACLE_LIB.exists():
            raise FileNotFoundError(f"{ORACLE_LIB} not built (make -C oracle)")
        lib = ctypes.CDLL(str(ORACLE_LIB))
        sig = {
            "sko_camera_make": (None, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_float, _vp]),
            "sko_ln": (ctypes.c_float, [ctypes.c_float]),
            "sko_float_to_half": (ctypes.c_uint16, [ctypes.c_float]),
            "sko_half_to_float": (ctypes.c_float, [ctypes.c_uint16]),
            "sko_visibility": (ctypes.c_uint32, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_int,
                                                 ctypes.c_int, _vp, ctypes.c_uint32, _vp,
                                                 ctypes.c_uint32, _vp, _vp, ctypes.c_int, _vp]),
            "sko_stable_argsort": (None, [_vp, ctypes.c_uint32, _vp]),
            "sko_radix_argsort": (None, [_vp, ctypes.c_uint32, ctypes.c_int, _vp, ctypes.c_int]),
            "sko_lod_select": (ctypes.c_uint32, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                                 ctypes.c_uint32, _vp, _vp]),
            "sko_composite": (None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     _vp, ctypes.c_int, ctypes.c_float, ctypes.c_int, _vp,
                                     ctypes.c_int]),
            "sko_composite_fragments": (ctypes.c_uint64, [_vp, _vp, ctypes.c_uint32,
                                                          ctypes.c_uint32, ctypes.c_uint32,
                                                          ctypes.c_float, ctypes.c_int]),
            "sko_mt19937": (None, [ctypes.c_uint32, ctypes.c_uint32, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib

    # numerics
    def ln(self, x: float) -> float:
        return self.lib.sko_ln(x)

    def float_to_half(self, x: float) -> int:
        return self.lib.sko_float_to_half(x)

    def camera(self, view, proj, position, width, height, min_pixel_radius=1.0) -> Camera:
        cam = Camera()
        v = np.ascontiguousarray(view, np.float32).reshape(16)
        p = np.ascontiguousarray(proj, np.float32).reshape(16)
        c = np.ascontiguousarray(position, np.float32).reshape(3)
        self.lib.sko_camera_make(_p(v), _p(p), _p(c), width, height, min_pixel_radius,
                                 ctypes.addressof(cam))
        return cam

    def visibility(self, cam: Camera, splats: np.ndarray, sh: Optional[np.ndarray], sh_stride: int,
                   sh_degree: int, key_bits: int, ranges: Sequence = (), indices=None,
                   threads: int = 1, parts=None):
        """parts: None, or (labels uint16[n], palette float32[10, 8], states uint32[k])."""
        splats = np.ascontiguousarray(splats)
        sh = None if sh is None or sh_degree == 0 else np.ascontiguousarray(sh, np.uint32)
        if indices is not None:
            idx = np.ascontiguousarray(indices, np.uint32)
            total = len(idx)
            rng_arr, rc = None, 0
        else:
            idx = None
            rng_arr = np.ascontiguousarray(np.array(ranges, np.uint32).reshape(-1, 2))
            rc = len(rng_arr)
            total = int(rng_arr[:, 1].sum()) if rc else 0
        keys = np.empty(max(total, 1), np.uint32)
        proj = np.empty(max(total, 1), PROJECTED_DTYPE)
        parts_struct, keep = None, None
        if parts is not None:
            labels = np.ascontiguousarray(parts[0], np.uint16)
            palette = np.ascontiguousarray(parts[1], np.float32).reshape(10, 8)
            states = np.ascontiguousarray(parts[2], np.uint32)
            keep = (labels, palette, states)
            parts_struct = (ctypes.c_void_p * 4)(labels.ctypes.data, palette.ctypes.data,
                                                 states.ctypes.data, len(states))
        n = self.lib.sko_visibility(ctypes.addressof(cam), _p(splats), _p(sh), sh_stride,
                                    sh_degree, key_bits, _p(rng_arr), rc, _p(idx),
                                    0 if idx is None else len(idx), _p(keys), _p(proj), threads,
                                    None if parts_struct is None else ctypes.addressof(parts_struct))
        del keep
        return keys[:n].copy(), proj[:n].copy()

    def stable_argsort(self, keys: np.ndarray) -> np.ndarray:
        keys = np.ascontiguousarray(keys, np.uint32)
        out = np.empty(len(keys), np.uint32)
        self.lib.sko_stable_argsort(_p(keys), len(keys), _p(out))
        return out

    def radix_argsort(self, keys: np.ndarray, bits: int, threads: int = 1) -> np.ndarray:
        keys = np.ascontiguousarray(keys, np.uint32)
        out = np.empty(len(keys), np.uint32)
        self.lib.sko_radix_argsort(_p(keys), len(keys), bits, _p(out), threads)
        return out

    def lod_select(self, cam: Camera, clusters: np.ndarray, leaves: np.ndarray, rounds: int,
                   capacity: int, pixel_limit: float, color_weight: float = 4.0, cull: bool = True):
        clusters = np.ascontiguousarray(clusters)
        leaves = np.ascontiguousarray(leaves, np.uint32)
        out = np.empty(max(capacity, 1), np.uint32)
        stats = np.zeros(6, np.uint32)
        n = self.lib.sko_lod_select(ctypes.addressof(cam), _p(clusters), len(clusters), _p(leaves),
                                    rounds, capacity, pixel_limit, color_weight, int(cull),
                                    _p(out), _p(stats))
        return out[:n].copy(), stats

    def composite(self, projected: np.ndarray, order: np.ndarray, width: int, height: int,
                  background=(0.05, 0.05, 0.08), opaque: bool = True, cutoff: float = 1e-4,
                  precision: int = 64, threads: int = 1) -> np.ndarray:
        projected = np.ascontiguousarray(projected)
        order = np.ascontiguousarray(order, np.uint32)
        bg = np.array(background, np.float32)
        out = np.empty((height, width, 4), np.float32)
        self.lib.sko_composite(_p(projected), _p(order), len(order), width, height, _p(bg),
                               int(opaque), cutoff, precision, _p(out), threads)
        return out

    def fragments(self, projected, order, width, height, cutoff=1e-4, threads=1) -> int:
        projected = np.ascontiguousarray(projected)
        order = np.ascontiguousarray(order, np.uint32)
        return int(self.lib.sko_composite_fragments(_p(projected), _p(order), len(order), width,
                                                    height, cutoff, threads))

    def mt19937(self, seed: int, n: int) -> np.ndarray:
        out = np.empty(n, np.uint32)
        self.lib.sko_mt19937(seed, n, _p(out))
        return out


class Reference:
    """The reference's own C++ through oracle/ref_shim.cpp."""

    def __init__(self):
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
        lib = ctypes.CDLL(str(REF_LIB))
        u32, f32, sz = ctypes.c_uint32, ctypes.c_float, ctypes.c_size_t
        sig = {
            "skref_to_half": (ctypes.c_uint16, [f32]),
            "skref_from_half": (f32, [ctypes.c_uint16]),
            "skref_perspective": (None, [f32, f32, f32, f32, _vp]),
            "skref_look_at_view": (None, [_vp, _vp, _vp, _vp]),
            "skref_covariance": (None, [_vp, _vp, _vp]),
            "skref_sh_stride": (sz, [ctypes.c_int]),
            "skref_gpu_world_bytes": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_int,
                                                        ctypes.c_uint64, ctypes.c_uint64,
                                                        ctypes.c_uint64]),
            "skref_pack_splats": (None, [_vp, _vp, _vp, _vp, sz, _vp]),
            "skref_pack_sh": (None, [_vp, sz, ctypes.c_int, ctypes.c_int, _vp]),
            "skref_build_lod_tree": (_vp, [_vp, _vp, _vp, _vp, _vp, sz, ctypes.c_int, _vp, _vp,
                                           u32, u32]),
            "skref_make_tree": (_vp, [_vp, _vp, _vp, _vp, _vp, sz, ctypes.c_int, _vp, sz]),
            "skref_tree_build_selection": (None, [_vp]),
            "skref_validate_lod_tree": (ctypes.c_int64, [_vp]),
            "skref_tree_node_count": (sz, [_vp]),
            "skref_tree_leaf_count": (sz, [_vp]),
            "skref_tree_sh_degree": (ctypes.c_int, [_vp]),
            "skref_tree_cluster_count": (sz, [_vp]),
            "skref_tree_leaf_ref_count": (sz, [_vp]),
            "skref_tree_sh_floats": (sz, [_vp]),
            "skref_tree_copy_nodes": (None, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "skref_tree_copy_layout": (None, [_vp, _vp]),
            "skref_tree_copy_clusters": (None, [_vp, _vp]),
            "skref_tree_copy_leaves": (None, [_vp, _vp]),
            "skref_free_tree": (None, [_vp]),
            "skref_write_lodsplat": (ctypes.c_int, [_vp, ctypes.c_char_p]),
            "skref_decode_lodsplat": (_vp, [_vp, sz, ctypes.c_int]),
            "skref_lod_threshold_new": (_vp, [f32]),
            "skref_lod_threshold_update": (f32, [_vp, u32, u32, u32]),
            "skref_lod_threshold_free": (None, [_vp]),
            "skref_valid_render_policy": (ctypes.c_int, [f32, u32, f32, f32, u32, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib

    def to_half(self, x: float) -> int:
        return self.lib.skref_to_half(x)

    def perspective(self, fovy, aspect, near, far) -> np.ndarray:
        out = np.empty(16, np.float32)
        self.lib.skref_perspective(fovy, aspect, near, far, _p(out))
        return out

    def look_at_view(self, position, target, up=(0, 1, 0)) -> np.ndarray:
        out = np.empty(16, np.float32)
        a = [np.ascontiguousarray(x, np.float32) for x in (position, target, up)]
        self.lib.skref_look_at_view(_p(a[0]), _p(a[1]), _p(a[2]), _p(out))
        return out

    def covariance(self, q, s) -> np.ndarray:
        out = np.empty(6, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        s = np.ascontiguousarray(s, np.float32)
        self.lib.skref_covariance(_p(q), _p(s), _p(out))
        return out

    def sh_stride(self, degree: int) -> int:
        return int(self.lib.skref_sh_stride(degree))

    def gpu_world_bytes(self, records, sh_degree, draw_capacity, clusters, leaf_refs) -> int:
        return int(self.lib.skref_gpu_world_bytes(records, sh_degree, draw_capacity, clusters,
                                                  leaf_refs))

    def pack_splats(self, cloud) -> np.ndarray:
        out = np.empty(cloud.count, SPLAT_DTYPE)
        self.lib.skref_pack_splats(_p(cloud.positions), _p(cloud.covariances), _p(cloud.colors),
                                   _p(cloud.alphas), cloud.count, _p(out))
        return out

    def pack_sh(self, cloud, degree: int) -> np.ndarray:
        stride = self.sh_stride(degree)
        out = np.zeros((cloud.count, max(stride, 1)), np.uint32)
        if degree > 0:
            sh = np.ascontiguousarray(cloud.sh, np.float32)
            self.lib.skref_pack_sh(_p(sh), cloud.count, cloud.sh_degree, degree, _p(out))
        return out[:, :stride] if stride else out[:, :0]

    # trees
    def _tree_arrays(self, handle) -> dict:
        lib = self.lib
        n = lib.skref_tree_node_count(handle)
        shf = lib.skref_tree_sh_floats(handle)
        pos = np.empty((n, 3), np.float32)
        cov = np.empty((n, 6), np.float32)
        col = np.empty((n, 3), np.float32)
        alp = np.empty(n, np.float32)
        sh = np.empty(max(shf, 1), np.float32)
        lib.skref_tree_copy_nodes(handle, _p(pos), _p(cov), _p(col), _p(alp), _p(sh))
        layout = np.empty(n, LOD_NODE_DTYPE)
        lib.skref_tree_copy_layout(handle, _p(layout))
        clusters = np.empty(lib.skref_tree_cluster_count(handle), LOD_CLUSTER_DTYPE)
        if len(clusters):
            lib.skref_tree_copy_clusters(handle, _p(clusters))
        leaves = np.empty(lib.skref_tree_leaf_ref_count(handle), np.uint32)
        if len(leaves):
            lib.skref_tree_copy_leaves(handle, _p(leaves))
        degree = lib.skref_tree_sh_degree(handle)
        return dict(positions=pos, covariances=cov, colors=col, alphas=alp,
                    sh=sh[:shf].reshape(n, -1) if shf else None, sh_degree=degree, layout=layout,
                    leaf_count=int(lib.skref_tree_leaf_count(handle)), clusters=clusters,
                    leaves=leaves, depth=int(lib.skref_validate_lod_tree(handle)))

    def build_lod_tree(self, cloud, octree_depth: int = 0, cluster_leaves: int = 0,
                       selection: bool = True) -> dict:
        lo = None if cloud.bounds_min is None else np.ascontiguousarray(cloud.bounds_min, np.float32)
        hi = None if cloud.bounds_max is None else np.ascontiguousarray(cloud.bounds_max, np.float32)
        sh = None if cloud.sh is None else np.ascontiguousarray(cloud.sh, np.float32)
        h = self.lib.skref_build_lod_tree(_p(cloud.positions), _p(cloud.covariances),
                                          _p(cloud.colors), _p(cloud.alphas), _p(sh), cloud.count,
                                          cloud.sh_degree, _p(lo), _p(hi), octree_depth,
                                          cluster_leaves)
        try:
            if selection:
                self.lib.skref_tree_build_selection(h)
            return self._tree_arrays(h)
        finally:
            self.lib.skref_free_tree(h)

    def write_lodsplat(self, cloud, path: str, octree_depth: int = 0, cluster_leaves: int = 0,
                       selection: bool = True) -> dict:
        """Builds the tree with the reference builder, writes it as a .lodsplat (version 2 with
        selection data, else 1) and returns its arrays."""
        lo = None if cloud.bounds_min is None else np.ascontiguousarray(cloud.bounds_min, np.float32)
        hi = None if cloud.bounds_max is None else np.ascontiguousarray(cloud.bounds_max, np.float32)
        sh = None if cloud.sh is None else np.ascontiguousarray(cloud.sh, np.float32)
        h = self.lib.skref_build_lod_tree(_p(cloud.positions), _p(cloud.covariances),
                                          _p(cloud.colors), _p(cloud.alphas), _p(sh), cloud.count,
                                          cloud.sh_degree, _p(lo), _p(hi), octree_depth,
                                          cluster_leaves)
        try:
            if selection:
                self.lib.skref_tree_build_selection(h)
            if self.lib.skref_write_lodsplat(h, str(path).encode()) != 0:
                raise RuntimeError("reference writeLodSplat failed")
            return self._tree_arrays(h)
        finally:
            self.lib.skref_free_tree(h)

    def decode_lodsplat(self, data: bytes, max_sh_degree: int = 3):
        """The reference decoder's arrays, or None when it rejects the file."""
        buf = np.frombuffer(data, np.uint8)
        h = self.lib.skref_decode_lodsplat(buf.ctypes.data, len(buf), max_sh_degree)
        if not h:
            return None
        try:
            return self._tree_arrays(h)
        finally:
            self.lib.skref_free_tree(h)

    def make_tree(self, nodes_cloud, layout: np.ndarray, leaf_count: int,
                  selection: bool = True) -> dict:
        layout = np.ascontiguousarray(layout, LOD_NODE_DTYPE)
        sh = None if nodes_cloud.sh is None else np.ascontiguousarray(nodes_cloud.sh, np.float32)
        h = self.lib.skref_make_tree(_p(nodes_cloud.positions), _p(nodes_cloud.covariances),
                                     _p(nodes_cloud.colors), _p(nodes_cloud.alphas), _p(sh),
                                     nodes_cloud.count, nodes_cloud.sh_degree, _p(layout),
                                     leaf_count)
        try:
            if selection:
                self.lib.skref_tree_build_selection(h)
            return self._tree_arrays(h)
        finally:
            self.lib.skref_free_tree(h)

    def lod_threshold(self, policy_pixels: float):
        lib = self.lib
        h = lib.skref_lod_threshold_new(policy_pixels)

        class _T:
            def update(self, selected, limited, limit):
                return lib.skref_lod_threshold_update(h, selected, limited, limit)

            def __del__(self):
                lib.skref_lod_threshold_free(h)

        return _T()

    def valid_render_policy(self, lod_error_pixels, lod_splat_limit, alpha_threshold,
                            subpixel_threshold, sort_depth, background) -> bool:
        bg = np.ascontiguousarray(background, np.float64)
        return bool(self.lib.skref_valid_render_policy(lod_error_pixels, lod_splat_limit,
                                                       alpha_threshold, subpixel_threshold,
                                                       sort_depth, _p(bg)))


def available() -> bool:
    return ORACLE_LIB.exists()


def reference_available() -> bool:
    return REF_LIB.exists()
