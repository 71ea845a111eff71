"""ctypes access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the checker and the CPU baseline; the product never imports it.
Parity is unpinned: the reference has no golden data and cannot be built here,
so the oracle is a line-by-line restatement of the reference worklets (see
beams_oracle.cpp for the cited lines and the VTK-m definitions it restates).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build_oracle

_lib = None


class OracleScene(C.Structure):
    _fields_ = [("field", C.c_void_p), ("dims", C.c_int * 3), ("origin", C.c_double * 3),
                ("spacing", C.c_double * 3), ("range", C.c_double * 2), ("tf", C.c_void_p), ("tf_n", C.c_int),
                ("light_kind", C.c_int), ("light", C.c_double * 3), ("light_color", C.c_float * 3),
                ("light_intensity", C.c_float), ("map_m", C.c_int * 3), ("use_map", C.c_int),
                ("sample_distance", C.c_float), ("alpha_cutoff", C.c_float), ("light_steps", C.c_float),
                ("slab_fp64", C.c_int), ("cam_pos", C.c_double * 3), ("cam_look", C.c_double * 3),
                ("cam_up", C.c_double * 3), ("fov_y_deg", C.c_double), ("width", C.c_int), ("height", C.c_int),
                ("precision", C.c_int), ("ray_max", C.c_void_p), ("coords", C.c_void_p * 3)]


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        L = C.CDLL(str(path))
        P, S = C.c_void_p, C.POINTER(OracleScene)
        u64p = C.POINTER(C.c_uint64)
        for name, args in {
            "oracle_light_march_f32": [S, P, C.c_int, u64p],
            "oracle_light_march_f64": [S, P, C.c_int, u64p],
            "oracle_light_march_ids_f32": [S, P, C.c_int64, P, C.c_int, u64p],
            "oracle_light_march_ids_f64": [S, P, C.c_int64, P, C.c_int, u64p],
            "oracle_light_march_points_f64": [S, P, C.c_int64, P, P, C.c_int],
            "oracle_light_march_points_f32": [S, P, C.c_int64, P, P, C.c_int],
            "oracle_view_march_f32": [S, P, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, u64p],
            "oracle_view_march_f64": [S, P, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, u64p],
            "oracle_view_march_cells_f32": [S, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, u64p],
            "oracle_view_march_cells_f64": [S, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, u64p],
            "oracle_view_march_lazy_f64": [S, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, u64p],
            "oracle_window_depth_to_distance": [S, P, C.c_double, C.c_double, P],
            "oracle_view_march_multi_f32": [S, P, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int,
                                            u64p],
            "oracle_ray_setup_f32": [S, C.c_int, C.c_int, P],
            "oracle_composite_f32": [P, C.c_int, C.c_int, P, P],
            "oracle_generate_noise": [P, C.c_int, C.c_int, C.c_int, P, C.c_int, C.c_float, C.c_float,
                                      C.c_float, C.c_int],
            "oracle_render_bricks_f32": [P, C.c_int, P, P, P, P, C.c_int, u64p],
            "oracle_generate_spheres": [P, C.c_int, C.c_int, C.c_int, P, P, P, C.c_int, C.c_float, C.c_int,
                                        C.c_float, C.c_float],
            "oracle_record_samples_f32": [S, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int64, P],
            "oracle_render_bricks_f64": [P, C.c_int, P, P, P, P, C.c_int, u64p],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """Oracle bound to one scene and one field array (z, y, x) float32."""

    def __init__(self, scene, field: np.ndarray | None = None, threads: int = 0, precision: bool = False):
        self.scene = scene
        self.field = np.ascontiguousarray(scene.field_numpy() if field is None else field, np.float32)
        self.tf = np.ascontiguousarray(scene.tf, np.float32)
        self.threads = threads
        s = scene
        self.cs = OracleScene(
            _p(self.field), (C.c_int * 3)(*s.dims), (C.c_double * 3)(*s.origin), (C.c_double * 3)(*s.spacing),
            (C.c_double * 2)(*s.value_range), _p(self.tf), self.tf.shape[0], s.light_kind,
            (C.c_double * 3)(*s.light), (C.c_float * 3)(*s.light_color), s.light_intensity,
            (C.c_int * 3)(*self._map_cells(s.map_m)), int(s.use_map), s.sample_distance, s.cutoff,
            s.light_steps, int(s.slab_fp64), (C.c_double * 3)(*s.cam_pos), (C.c_double * 3)(*s.cam_look),
            (C.c_double * 3)(*s.cam_up), s.fov_y_deg, s.width, s.height, int(precision))
        coords = getattr(scene, "coords", None)
        if coords is not None:
            self._coords = [np.ascontiguousarray(c, np.float32) for c in coords]
            for d in range(3):
                self.cs.coords[d] = self._coords[d].ctypes.data

    def set_ray_limits(self, limits):
        """Canvas depth clipping: (height, width) float32 per-pixel ray limits, or None."""
        self._ray_max = None if limits is None else np.ascontiguousarray(limits, np.float32)
        self.cs.ray_max = None if limits is None else self._ray_max.ctypes.data

    def window_depth_to_distance(self, depth, near, far):
        """Per-pixel ray limits (float64) of an OpenGL window-depth buffer under this camera."""
        d = np.ascontiguousarray(depth, np.float32)
        out = np.empty(d.shape, np.float64)
        if lib().oracle_window_depth_to_distance(C.byref(self.cs), _p(d), float(near), float(far), _p(out)):
            raise RuntimeError("oracle depth conversion rejected its input")
        return out

    @staticmethod
    def _map_cells(m):
        """Map cells per axis (x, y, z): one integer for a cubic map, or three."""
        return tuple(int(v) for v in m) if isinstance(m, (tuple, list)) else (int(m),) * 3

    @property
    def map_shape(self):
        mx, my, mz = self._map_cells(self.scene.map_m)
        return (mz + 1, my + 1, mx + 1)

    def light_march(self, fp64: bool = False):
        out = np.empty(self.map_shape, np.float64 if fp64 else np.float32)
        ns = C.c_uint64()
        fn = lib().oracle_light_march_f64 if fp64 else lib().oracle_light_march_f32
        if fn(C.byref(self.cs), _p(out), self.threads, C.byref(ns)):
            raise RuntimeError("oracle light march rejected the scene")
        return out, ns.value

    def light_march_ids(self, ids: np.ndarray, fp64: bool = False):
        ids = np.ascontiguousarray(ids, np.int64)
        out = np.empty(ids.shape[0], np.float64 if fp64 else np.float32)
        ns = C.c_uint64()
        fn = lib().oracle_light_march_ids_f64 if fp64 else lib().oracle_light_march_ids_f32
        if fn(C.byref(self.cs), _p(ids), ids.shape[0], _p(out), self.threads, C.byref(ns)):
            raise RuntimeError("oracle light march rejected the scene")
        return out, ns.value

    def point_opacity(self, pts: np.ndarray, light_pos: np.ndarray | None = None, fp64: bool = True):
        """Light-march opacity from the light (or light_pos per point) to each point."""
        dt = np.float64 if fp64 else np.float32
        pts = np.ascontiguousarray(pts, dt).reshape(-1, 3)
        out = np.empty(pts.shape[0], dt)
        lp = None if light_pos is None else np.ascontiguousarray(light_pos, dt).reshape(-1, 3)
        fn = lib().oracle_light_march_points_f64 if fp64 else lib().oracle_light_march_points_f32
        if fn(C.byref(self.cs), _p(pts), pts.shape[0], None if lp is None else _p(lp), _p(out), self.threads):
            raise RuntimeError("oracle point march rejected the scene")
        return out

    def view_march(self, map_values=None, window=None, fp64: bool = False):
        s = self.scene
        x0, y0, w, h = window if window is not None else (0, 0, s.width, s.height)
        dt = np.float64 if fp64 else np.float32
        out = np.zeros((h, w, 4), dt)
        if s.use_map and map_values is None:
            map_values, _ = self.light_march(fp64)
        mp = None if map_values is None else np.ascontiguousarray(map_values, dt)
        lit = C.c_uint64()
        fn = lib().oracle_view_march_f64 if fp64 else lib().oracle_view_march_f32
        if fn(C.byref(self.cs), None if mp is None else _p(mp), x0, y0, w, h, _p(out), self.threads,
              C.byref(lit)):
            raise RuntimeError("oracle view march rejected the scene")
        return out, lit.value

    def view_march_cells(self, window=None, fp64: bool = False):
        """Unlit march of a cell-centred field (SamplerCellAssoc): build the Oracle
        with field = the (nz-1, ny-1, nx-1) cell values and the scene's point dims."""
        s = self.scene
        x0, y0, w, h = window if window is not None else (0, 0, s.width, s.height)
        if self.field.size != (s.dims[0] - 1) * (s.dims[1] - 1) * (s.dims[2] - 1):
            raise ValueError("view_march_cells needs the (dims - 1)^3 cell values as the field")
        dt = np.float64 if fp64 else np.float32
        out = np.zeros((h, w, 4), dt)
        lit = C.c_uint64()
        fn = lib().oracle_view_march_cells_f64 if fp64 else lib().oracle_view_march_cells_f32
        if fn(C.byref(self.cs), x0, y0, w, h, _p(out), self.threads, C.byref(lit)):
            raise RuntimeError("oracle cell-field march rejected the scene")
        return out, lit.value

    def view_march_multi(self, maps, light_colors, window=None):
        """Multi-light extension: maps is (n_lights, map vertices) exact-form
        opacity, light_colors (n_lights, 3) colour * intensity in float32."""
        s = self.scene
        x0, y0, w, h = window if window is not None else (0, 0, s.width, s.height)
        mp = np.ascontiguousarray(maps, np.float32)
        lc = np.ascontiguousarray(light_colors, np.float32).reshape(-1, 3)
        if mp.shape[0] != lc.shape[0]:
            raise ValueError("one map per light colour")
        out = np.zeros((h, w, 4), np.float32)
        lit = C.c_uint64()
        if lib().oracle_view_march_multi_f32(C.byref(self.cs), _p(mp), lc.shape[0], _p(lc), x0, y0, w, h, _p(out),
                                             self.threads, C.byref(lit)):
            raise RuntimeError("oracle multi-light view march rejected the scene")
        return out, lit.value

    def view_march_lazy_f64(self, window, stride: int = 1):
        x0, y0, w, h = window
        ow, oh = -(-w // stride), -(-h // stride)
        out = np.zeros((oh, ow, 4), np.float64)
        lit = C.c_uint64()
        if lib().oracle_view_march_lazy_f64(C.byref(self.cs), x0, y0, w, h, stride, _p(out), self.threads,
                                            C.byref(lit)):
            raise RuntimeError("oracle lazy view march rejected the scene")
        return out, lit.value

    def record_samples(self, window=None, cap=1 << 24):
        """Lit samples per pixel in march order: (records (n,7), counts (h,w))."""
        s = self.scene
        x0, y0, w, h = window if window is not None else (0, 0, s.width, s.height)
        rec = np.zeros((cap, 7), np.float32)
        counts = np.zeros((h, w), np.int32)
        rc = lib().oracle_record_samples_f32(C.byref(self.cs), x0, y0, w, h, _p(rec), cap, _p(counts))
        if rc == 1:
            raise RuntimeError("oracle sample recorder rejected the scene")
        if rc == 2:
            raise RuntimeError("sample cap reached")
        return rec[:counts.sum()], counts

    def ray_setup(self, x: int, y: int):
        out = np.zeros(8, np.float32)
        lib().oracle_ray_setup_f32(C.byref(self.cs), x, y, _p(out))
        return out


def render_bricks(bricks, fp64: bool = False, threads: int = 0, ray_limits=None):
    """Multi-block render of a list of brick scenes (scenes.split_bricks), with
    optional per-pixel ray limits (canvas depth clipping) shared by all bricks.
    Returns (rgba, brick_images, local_maps, final_maps, lit)."""
    orcs = [Oracle(b, threads=threads) for b in bricks]
    for o in orcs:
        o.set_ray_limits(ray_limits)
    arr = (OracleScene * len(bricks))(*[o.cs for o in orcs])
    dt = np.float64 if fp64 else np.float32
    W, H = bricks[0].width, bricks[0].height
    nverts = [int(np.prod(o.map_shape)) for o in orcs]
    local = np.zeros(sum(nverts), dt)
    final = np.zeros(sum(nverts), dt)
    imgs = np.zeros((len(bricks), H, W, 4), dt)
    rgba = np.zeros((H, W, 4), dt)
    lit = C.c_uint64()
    fn = lib().oracle_render_bricks_f64 if fp64 else lib().oracle_render_bricks_f32
    if fn(C.cast(arr, C.c_void_p), len(bricks), _p(local), _p(final), _p(imgs), _p(rgba), threads, C.byref(lit)):
        raise RuntimeError("oracle brick render rejected the scenes")
    split = np.cumsum(nverts)[:-1]
    return rgba, imgs, np.split(local, split), np.split(final, split), lit.value


def composite(images: np.ndarray, order) -> np.ndarray:
    """Sort-last over of premultiplied RGBA images (MapperLightedVolume.cxx:284-297)."""
    imgs = np.ascontiguousarray(images, np.float32)
    n = imgs.shape[0]
    npix = imgs[0].size // 4
    order = np.ascontiguousarray(order, np.int32)
    out = np.zeros(imgs.shape[1:], np.float32)
    if lib().oracle_composite_f32(_p(imgs), n, npix, _p(order), _p(out)):
        raise RuntimeError("oracle composite rejected the input")
    return out


def noise_field(dims, perm, octaves=4, base_freq=4.0, lacunarity=2.0, gain=0.5, threads=0) -> np.ndarray:
    """Gradient-noise field on the CPU (z, y, x), the same float32 operations as the
    library's device generator."""
    nx, ny, nz = dims
    out = np.empty((nz, ny, nx), np.float32)
    perm = np.ascontiguousarray(perm, np.uint8)
    if lib().oracle_generate_noise(_p(out), nx, ny, nz, _p(perm), octaves, base_freq, lacunarity, gain, threads):
        raise RuntimeError("oracle noise generator rejected the arguments")
    return out


def spheres_field(dims, origin, spacing, ellipsoids, default=0.1, floor=None):
    """sources::Spheres field (float32, (z, y, x)); floor = (height, value) or None."""
    nx, ny, nz = dims
    out = np.zeros((nz, ny, nx), np.float32)
    e = np.ascontiguousarray(ellipsoids, np.float32).reshape(-1, 8)
    org = np.asarray(origin, np.float32)
    sp = np.asarray(spacing, np.float32)
    fy, fv = (0.0, 0.0) if floor is None else floor
    floor_y = float(np.float32(org[1]) + np.float32(fy))
    if lib().oracle_generate_spheres(_p(out), nx, ny, nz, _p(org), _p(sp), _p(e), e.shape[0], float(default),
                                     int(floor is not None), floor_y, float(fv)):
        raise RuntimeError("oracle spheres generator rejected the arguments")
    return out


def quantize(field: np.ndarray, dtype: str) -> np.ndarray:
    """float32 values of a field rounded to bfloat16 or float16 (round to nearest even)."""
    f = np.ascontiguousarray(field, np.float32)
    if dtype == "f16":
        return f.astype(np.float16).astype(np.float32)
    if dtype == "bf16":
        u = f.view(np.uint32).astype(np.uint64)
        lsb = (u >> 16) & 1
        r = ((u + 0x7FFF + lsb) >> 16) << 16
        return r.astype(np.uint32).view(np.float32)
    raise ValueError(dtype)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(1.0 / mse)


def blend_background(img, bg):
    """Porter-Duff "over" of a premultiplied float32 RGBA image over the colour bg
    (a = bg.a (1 - C.a), C.rgb += bg.rgb a, C.a += a; pixels with C.a >= 1 kept),
    in float32 with one rounding per operation."""
    out = np.array(img, np.float32, copy=True)
    b = np.asarray(bg, np.float32)
    m = out[..., 3] < np.float32(1)
    a = b[3] * (np.float32(1) - out[..., 3])
    for k in range(3):
        out[..., k] = np.where(m, out[..., k] + b[k] * a, out[..., k])
    out[..., 3] = np.where(m, a + out[..., 3], out[..., 3])
    return out
