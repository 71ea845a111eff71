"""ctypes binding of libbeams_b200.so and a mirror of the reference's mapper API.

``Renderer`` is a thin 1:1 wrapper of the C ABI (include/beams_b200.h).
``MapperLightedVolume`` mirrors beams::rendering::MapperLightedVolume
(beams/rendering/MapperLightedVolume.h:16-62): the same setter names, the same
argument meaning, the same error behaviour (the reference throws
vtkm::cont::ErrorBadValue; this raises BeamsError with the library's message).

There is no fallback: importing this module fails loudly when the CUDA library
has not been built, and every render runs the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libbeams_b200.so"

BEAMS_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "CUDA", 4: "OOM", 5: "TIMEOUT",
                6: "CONFIG", 7: "INTERNAL", 8: "STATE"}
F32, BF16, F16 = 0, 1, 2
ASSOC_POINTS, ASSOC_CELLS = 0, 1
FORM_EXACT, FORM_PRECISION, FORM_MLP = 0, 1, 2
DEPTH_RAY_DISTANCE, DEPTH_WINDOW = 0, 1
OUT_HOST, OUT_DEVICE, OUT_HOST_ASYNC = 0, 1, 2


class MlpOptions(C.Structure):
    _fields_ = [("samples_log2", C.c_int), ("n_lights", C.c_int), ("epochs", C.c_int), ("batch", C.c_int),
                ("lr", C.c_float), ("seed", C.c_uint), ("fallback_tol", C.c_float), ("probe_fraction", C.c_float),
                ("knot", C.c_int), ("scene_light", C.c_int), ("focus", C.c_float)]


class MlpReport(C.Structure):
    _fields_ = [("datagen_ms", C.c_float), ("train_ms", C.c_float), ("holdout_rmse", C.c_float),
                ("initial_rmse", C.c_float), ("unlit_rmse", C.c_float), ("mean_rmse", C.c_float),
                ("steps", C.c_int), ("samples", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def mlp_options(samples_log2=24, n_lights=32, epochs=4, batch=16384, lr=2e-3, seed=1, fallback_tol=0.01,
                probe_fraction=0.01, knot=4, scene_light=0, focus=0.875):
    return MlpOptions(samples_log2, n_lights, epochs, batch, lr, seed, fallback_tol, probe_fraction, knot,
                      scene_light, focus)


class Tuning(C.Structure):
    _fields_ = [("light_brick", C.c_int), ("no_empty_skip", C.c_int), ("no_view_skip", C.c_int),
                ("reserved", C.c_int)]


class BeamsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Volume(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int), ("dims", C.c_int * 3),
                ("origin", C.c_double * 3), ("spacing", C.c_double * 3), ("range", C.c_double * 2),
                ("assoc", C.c_int), ("on_device", C.c_int)]


# beams_profile_fn: (user, frame name, depth, ms)
PROFILE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_char_p, C.c_int, C.c_double)


class Camera(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("look_at", C.c_double * 3), ("up", C.c_double * 3),
                ("fov_y_deg", C.c_double), ("width", C.c_int), ("height", C.c_int)]


class Request(C.Structure):
    _fields_ = [("volume", C.c_int), ("camera", Camera), ("light_kind", C.c_int), ("light", C.c_double * 3),
                ("light_color", C.c_float * 3), ("light_intensity", C.c_float), ("map_cells", C.c_int),
                ("sample_distance", C.c_float), ("termination_alpha", C.c_float), ("rgba_out", C.c_void_p),
                ("out_on_device", C.c_int)]


class BatchOptions(C.Structure):
    _fields_ = [("tile_w", C.c_int), ("tile_h", C.c_int), ("light_brick", C.c_int), ("use_graph", C.c_int),
                ("no_skip", C.c_int), ("split", C.c_int), ("reserved", C.c_int)]


class ConfigLight(C.Structure):
    _fields_ = [("kind", C.c_int), ("position", C.c_double * 3), ("color", C.c_float * 3),
                ("intensity", C.c_float)]


class SceneDesc(C.Structure):
    """beams_scene_desc: a parsed stage TOML (see beams_parse_config_toml)."""
    _fields_ = [("provider_name", C.c_char * 64), ("provider_type", C.c_char * 32), ("cell_dims", C.c_int * 3),
                ("seed", C.c_uint), ("octaves", C.c_int), ("base_freq", C.c_float),
                ("width", C.c_int), ("height", C.c_int), ("sample_distance", C.c_float),
                ("termination_alpha", C.c_float), ("form", C.c_int), ("field_dtype", C.c_int),
                ("composite_background", C.c_int), ("background", C.c_float * 4),
                ("shadow_enabled", C.c_int), ("shadow_size", C.c_int * 3), ("shadow_size_ratio", C.c_float),
                ("light_steps", C.c_float), ("camera_explicit", C.c_int), ("azimuth", C.c_float),
                ("elevation", C.c_float), ("fov_y_deg", C.c_float), ("position", C.c_double * 3),
                ("look_at", C.c_double * 3), ("up", C.c_double * 3), ("n_lights", C.c_int),
                ("lights", ConfigLight * 8), ("tf_preset", C.c_char * 32), ("tf_points", C.c_int),
                ("tf_x", C.c_double * 64), ("tf_alpha", C.c_float * 64), ("tf_range", C.c_float * 2),
                ("tf_size", C.c_int), ("mlp_knot", C.c_int), ("mlp_probe_fraction", C.c_float),
                ("mlp_fallback_tol", C.c_float), ("mlp_samples_log2", C.c_int), ("mlp_lights", C.c_int),
                ("file_name", C.c_char * 256)]


def parse_config(text: str) -> SceneDesc:
    """Parses stage TOML text; raises BeamsError with "line N: ..." on errors."""
    d, err = SceneDesc(), C.create_string_buffer(512)
    st = lib().beams_parse_config_toml(text.encode(), C.byref(d), err, 512)
    if st != BEAMS_OK:
        raise BeamsError(st, err.value.decode())
    return d


def load_config(path) -> SceneDesc:
    d, err = SceneDesc(), C.create_string_buffer(512)
    st = lib().beams_load_config_toml(str(path).encode(), C.byref(d), err, 512)
    if st != BEAMS_OK:
        raise BeamsError(st, err.value.decode())
    return d


def scene_color_table(d: SceneDesc) -> np.ndarray:
    out = np.zeros((d.tf_size, 4), np.float32)
    st = lib().beams_scene_color_table(C.byref(d), _ptr(out), d.tf_size)
    if st != BEAMS_OK:
        raise BeamsError(st, "scene_color_table")
    return out


class Timings(C.Structure):
    _fields_ = [("map_build_ms", C.c_float), ("view_march_ms", C.c_float), ("composite_ms", C.c_float),
                ("total_ms", C.c_float), ("light_samples", C.c_ulonglong), ("lit_samples", C.c_ulonglong),
                ("rays_hit", C.c_ulonglong), ("mlp_samples", C.c_ulonglong), ("map_vertices", C.c_int),
                ("fallback_tiles", C.c_int), ("kernel_launches", C.c_int), ("mlp_rows", C.c_ulonglong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VtkField(C.Structure):
    _fields_ = [("dims", C.c_int * 3), ("assoc", C.c_int), ("origin", C.c_double * 3), ("spacing", C.c_double * 3),
                ("coords", C.POINTER(C.c_float) * 3), ("data", C.POINTER(C.c_float)), ("range", C.c_double * 2),
                ("name", C.c_char * 64)]


_lib = None


def lib():
    """Loads the CUDA library (raises when it is missing: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH} is missing: run pilot_b200/build.py (there is no CPU fallback)")
    L = C.CDLL(str(_LIB_PATH))
    P = C.c_void_p
    sig = {
        "beams_abi_version": ([], C.c_int),
        "beams_last_error": ([P], C.c_char_p),
        "beams_create": ([C.POINTER(P), C.c_int, P], C.c_int),
        "beams_destroy": ([P], C.c_int),
        "beams_set_volume": ([P, C.POINTER(Volume)], C.c_int),
        "beams_set_color_map": ([P, P, C.c_int], C.c_int),
        "beams_set_shadow_map_size": ([P, C.c_int, C.c_int, C.c_int], C.c_int),
        "beams_set_use_shadow_map": ([P, C.c_int], C.c_int),
        "beams_clear_lights": ([P], C.c_int),
        "beams_add_point_light": ([P, P, P, C.c_float], C.c_int),
        "beams_add_directional_light": ([P, P, P, C.c_float], C.c_int),
        "beams_set_sample_distance": ([P, C.c_float], C.c_int),
        "beams_set_termination_alpha": ([P, C.c_float], C.c_int),
        "beams_set_density_scale": ([P, C.c_float], C.c_int),
        "beams_get_density_scale": ([P, P], C.c_int),
        "beams_set_light_steps": ([P, C.c_float], C.c_int),
        "beams_set_slab_fp64": ([P, C.c_int], C.c_int),
        "beams_set_reuse_shadow_map": ([P, C.c_int], C.c_int),
        "beams_set_lazy_shadow_map": ([P, C.c_int], C.c_int),
        "beams_set_background": ([P, C.c_int, P], C.c_int),
        "beams_set_form": ([P, C.c_int, P], C.c_int),
        "beams_render": ([P, C.POINTER(Camera), P, C.c_int, C.POINTER(Timings)], C.c_int),
        "beams_get_shadow_map": ([P, P, C.c_size_t, C.c_int], C.c_int),
        "beams_build_shadow_map": ([P, C.POINTER(Timings)], C.c_int),
        "beams_generate_blobs": ([P, P, P, C.c_int, C.c_int, P], C.c_int),
        "beams_selftest_division": ([C.c_float, C.c_float, C.c_int, C.c_int, C.POINTER(C.c_ulonglong),
                                     C.POINTER(C.c_ulonglong)], C.c_int),
        "beams_set_bricks": ([P, P, C.c_int], C.c_int),
        "beams_mlp_train": ([P, C.POINTER(MlpOptions), C.POINTER(MlpReport)], C.c_int),
        "beams_mlp_param_count": ([], C.c_int),
        "beams_mlp_get_params": ([P, P, C.c_int], C.c_int),
        "beams_mlp_set_params": ([P, P, C.c_int], C.c_int),
        "beams_mlp_loss_grad": ([P, P, P, C.c_int, C.POINTER(C.c_float), P, P], C.c_int),
        "beams_mlp_encode": ([P, P, P, C.c_int, P], C.c_int),
        "beams_mlp_probe_errors": ([P, P, C.c_int], C.c_int),
        "beams_mlp_forward_tc": ([P, P, C.c_int, P], C.c_int),
        "beams_mlp_set_tensor_cores": ([P, C.c_int], C.c_int),
        "beams_mlp_set_probe_first": ([P, C.c_int], C.c_int),
        "beams_set_profiler": ([P, P, P], C.c_int),
        "beams_mlp_forward_tc_device": ([P, P, C.c_int, P], C.c_int),
        "beams_set_tuning": ([P, C.POINTER(Tuning)], C.c_int),
        "beams_set_multi_light": ([P, C.c_int], C.c_int),
        "beams_set_depth_buffer": ([P, P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int], C.c_int),
        "beams_get_ray_limits": ([P, C.POINTER(Camera), P, C.c_int], C.c_int),
        "beams_synchronize": ([P], C.c_int),
        "beams_batch_tuning_save": ([P, C.c_char_p], C.c_int),
        "beams_batch_tuning_load": ([P, C.c_char_p], C.c_int),
        "beams_batch_tuning_clear": ([P], C.c_int),
        "beams_set_volume_coordinates": ([P, P, P, P], C.c_int),
        "beams_vtk_read": ([C.c_char_p, C.POINTER(VtkField)], C.c_int),
        "beams_vtk_free": ([C.POINTER(VtkField)], None),
        "beams_test_fail_allocation": ([C.c_int], C.c_int),
        "beams_get_tuning": ([P, C.POINTER(Tuning)], C.c_int),
        "beams_batch_set_volumes": ([P, P, C.c_int], C.c_int),
        "beams_set_batch_options": ([P, C.POINTER(BatchOptions)], C.c_int),
        "beams_render_batch": ([P, P, C.c_int, C.POINTER(Timings)], C.c_int),
        "beams_batch_autotune": ([P, P, C.c_int, C.POINTER(BatchOptions), C.POINTER(C.c_float)], C.c_int),
        "beams_parse_config_toml": ([P, P, P, C.c_int], C.c_int),
        "beams_load_config_toml": ([P, P, P, C.c_int], C.c_int),
        "beams_apply_scene": ([P, P, C.POINTER(Camera)], C.c_int),
        "beams_orbit_light": ([P, P, C.c_int], C.c_int),
        "beams_scene_color_table": ([P, P, C.c_int], C.c_int),
        "beams_generate_spheres": ([P, P, P, P, P, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float, P], C.c_int),
        "beams_autotune": ([P, C.POINTER(Camera), C.POINTER(Tuning), C.POINTER(C.c_float), C.POINTER(C.c_float)],
                           C.c_int),
        "beams_mlp_save": ([P, C.c_char_p], C.c_int),
        "beams_mlp_load": ([P, C.c_char_p], C.c_int),
        "beams_get_brick_map": ([P, C.c_int, C.c_int, P, C.c_size_t, C.c_int], C.c_int),
        "beams_generate_noise": ([P, P, P, C.c_int, C.c_float, C.c_float, C.c_float, P], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def exported_symbols():
    """Names the header declares; used by the load test."""
    hdr = Path(__file__).resolve().parent.parent / "include" / "beams_b200.h"
    import re
    text = hdr.read_text()
    return sorted(set(re.findall(r"^\s*(?:beams_status|const char\*|int)\s+(beams_\w+)\s*\(", text, re.M)))


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


class Renderer:
    """1:1 wrapper of the beams_* C ABI."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._L = lib()
        h = C.c_void_p()
        self._check(self._L.beams_create(C.byref(h), int(device), C.c_void_p(stream) if stream else None), None)
        self._h = h
        self._keep = []

    def _check(self, st, h="self"):
        if st != BEAMS_OK:
            hh = self._h if h == "self" else h
            msg = self._L.beams_last_error(hh)
            raise BeamsError(st, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            self._L.beams_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- setters --------------------------------------------------------------
    def set_volume(self, data, dims=None, origin=(0, 0, 0), spacing=None, value_range=None,
                   dtype=F32, assoc=ASSOC_POINTS):
        """data: numpy array (z, y, x) on the host, or a torch CUDA tensor."""
        on_device = 0
        if isinstance(data, np.ndarray):
            arr = np.ascontiguousarray(data)
            if dims is None:
                nz, ny, nx = arr.shape
                dims = (nx, ny, nz) if assoc == ASSOC_POINTS else (nx + 1, ny + 1, nz + 1)
            if dtype == F32:
                arr = arr.astype(np.float32, copy=False)
            self._keep_host = arr
            ptr = arr.ctypes.data_as(C.c_void_p)
        else:  # torch tensor (float32, bfloat16 or float16)
            import torch
            on_device = 1 if data.is_cuda else 0
            dtype = {torch.float32: F32, torch.bfloat16: BF16, torch.float16: F16}[data.dtype]
            if dims is None:
                nz, ny, nx = data.shape
                dims = (nx, ny, nz) if assoc == ASSOC_POINTS else (nx + 1, ny + 1, nz + 1)
            ptr = C.c_void_p(data.data_ptr())
            self._keep_dev = data
        if spacing is None:
            spacing = tuple(1.0 / (d - 1) for d in dims)
        if value_range is None:
            value_range = (0.0, 1.0)
        v = Volume(ptr, dtype, (C.c_int * 3)(*dims), _d3(origin), _d3(spacing),
                   (C.c_double * 2)(*value_range), assoc, on_device)
        self._check(self._L.beams_set_volume(self._h, C.byref(v)))

    # -- configuration ----------------------------------------------------------
    def apply_scene(self, desc: SceneDesc) -> Camera:
        """Generates the described dataset on the device and configures the renderer; returns the camera."""
        cam = Camera()
        self._check(self._L.beams_apply_scene(self._h, C.byref(desc), C.byref(cam)))
        self._scene_desc = desc
        return cam

    def orbit_light(self, desc: SceneDesc, frame: int):
        self._check(self._L.beams_orbit_light(self._h, C.byref(desc), int(frame)))

    # -- batched form -----------------------------------------------------------
    def batch_set_volumes(self, volumes):
        """volumes: list of (array (z,y,x) float32 numpy or torch CUDA tensor, origin, spacing, value_range)."""
        vols = (Volume * len(volumes))()
        self._keep_batch = []
        for i, (data, origin, spacing, vrange) in enumerate(volumes):
            if isinstance(data, np.ndarray):
                arr = np.ascontiguousarray(data, np.float32)
                self._keep_batch.append(arr)
                ptr, on_dev = arr.ctypes.data_as(C.c_void_p), 0
                nz, ny, nx = arr.shape
            else:
                self._keep_batch.append(data)
                ptr, on_dev = C.c_void_p(data.data_ptr()), 1
                nz, ny, nx = data.shape
            vols[i] = Volume(ptr, F32, (C.c_int * 3)(nx, ny, nz), _d3(origin), _d3(spacing),
                             (C.c_double * 2)(*vrange), ASSOC_POINTS, on_dev)
        self._check(self._L.beams_batch_set_volumes(self._h, vols, len(volumes)))

    def set_batch_options(self, tile_w=32, tile_h=32, light_brick=8, use_graph=True, skip=True, split=False,
                          _withhold=False):
        """split: every map build, then every view march, as two launches (no waits between them)."""
        o = BatchOptions(int(tile_w), int(tile_h), int(light_brick), int(bool(use_graph)), int(not skip),
                         int(bool(split)), 0x7E57 if _withhold else 0)
        self._check(self._L.beams_set_batch_options(self._h, C.byref(o)))

    @staticmethod
    def request(volume, camera, light, light_kind=0, light_color=(1, 1, 1), light_intensity=1.0, map_cells=16,
                sample_distance=-1.0, termination_alpha=1.0, out=None):
        """One batch request; out: numpy (H,W,4) float32 or torch CUDA tensor (allocated if None)."""
        if out is None:
            out = np.zeros((camera.height, camera.width, 4), np.float32)
        on_dev = 0 if isinstance(out, np.ndarray) else int(out.is_cuda)
        rq = Request(int(volume), camera, int(light_kind), _d3(light), _f3(light_color), float(light_intensity),
                     int(map_cells), float(sample_distance), float(termination_alpha), _ptr(out), on_dev)
        return rq, out

    def batch_autotune(self, reqs):
        arr = (Request * len(reqs))(*[r for r, _ in reqs])
        o, ms = BatchOptions(), C.c_float()
        self._check(self._L.beams_batch_autotune(self._h, arr, len(reqs), C.byref(o), C.byref(ms)))
        return {"tile_w": o.tile_w, "tile_h": o.tile_h, "light_brick": o.light_brick, "skip": not o.no_skip,
                "split": bool(o.split), "batch_ms": ms.value}

    def batch_tuning_save(self, path):
        self._check(self._L.beams_batch_tuning_save(self._h, str(path).encode()))

    def batch_tuning_load(self, path):
        self._check(self._L.beams_batch_tuning_load(self._h, str(path).encode()))

    def batch_tuning_clear(self):
        self._check(self._L.beams_batch_tuning_clear(self._h))

    def render_batch(self, reqs, timings=True):
        """reqs: list of (Request, out) from Renderer.request; returns the outputs and timings."""
        arr = (Request * len(reqs))(*[r for r, _ in reqs])
        t = Timings() if timings else None
        self._check(self._L.beams_render_batch(self._h, arr, len(reqs), C.byref(t) if t is not None else None))
        return [o for _, o in reqs], (t.as_dict() if t is not None else None)

    def set_bricks(self, bricks):
        """bricks: list of (array (z,y,x) float32 numpy or torch CUDA tensor, origin, spacing, value_range)."""
        vols = (Volume * len(bricks))()
        self._keep_bricks = []
        for i, (data, origin, spacing, vrange) in enumerate(bricks):
            if isinstance(data, np.ndarray):
                arr = np.ascontiguousarray(data, np.float32)
                self._keep_bricks.append(arr)
                ptr, on_dev = arr.ctypes.data_as(C.c_void_p), 0
                nz, ny, nx = arr.shape
            else:
                self._keep_bricks.append(data)
                ptr, on_dev = C.c_void_p(data.data_ptr()), int(data.is_cuda)
                nz, ny, nx = data.shape
            vols[i] = Volume(ptr, F32, (C.c_int * 3)(nx, ny, nz), _d3(origin), _d3(spacing),
                             (C.c_double * 2)(*vrange), ASSOC_POINTS, on_dev)
        self._check(self._L.beams_set_bricks(self._h, C.cast(vols, C.c_void_p), len(bricks)))

    def get_brick_map(self, brick: int, stage: int, count: int):
        m = np.empty(count, np.float32)
        self._check(self._L.beams_get_brick_map(self._h, brick, stage, _ptr(m), m.size, 0))
        return m

    # -- learned form ---------------------------------------------------------
    def mlp_train(self, opts: MlpOptions | None = None):
        rep = MlpReport()
        self._check(self._L.beams_mlp_train(self._h, C.byref(opts) if opts is not None else None, C.byref(rep)))
        return rep.as_dict()

    def mlp_params(self):
        n = self._L.beams_mlp_param_count()
        out = np.empty(n, np.float32)
        self._check(self._L.beams_mlp_get_params(self._h, _ptr(out), n))
        return out

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._L.beams_mlp_set_params(self._h, _ptr(p), p.size))

    def mlp_loss_grad(self, features, target):
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        n = t.size
        g = np.empty(self._L.beams_mlp_param_count(), np.float32)
        T = np.empty(n, np.float32)
        loss = C.c_float()
        self._check(self._L.beams_mlp_loss_grad(self._h, _ptr(f), _ptr(t), n, C.byref(loss), _ptr(g), _ptr(T)))
        return loss.value, g, T

    def mlp_encode(self, pos, lfeat):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        lf = np.ascontiguousarray(lfeat, np.float32).reshape(-1, 3)
        out = np.empty((pos.shape[0], 112), np.float32)
        self._check(self._L.beams_mlp_encode(self._h, _ptr(pos), _ptr(lf), pos.shape[0], _ptr(out)))
        return out

    def mlp_forward_tc(self, features):
        """The tcgen05 forward pass on (n, 112) features; returns T (n,)."""
        X = np.ascontiguousarray(features, np.float32).reshape(-1, 112)
        T = np.empty(X.shape[0], np.float32)
        self._check(self._L.beams_mlp_forward_tc(self._h, _ptr(X), X.shape[0], _ptr(T)))
        return T

    def mlp_forward_tc_device(self, features_bf16, T):
        """tcgen05 forward on torch CUDA tensors: features (n, 112) bfloat16, T (n,) float32."""
        self._check(self._L.beams_mlp_forward_tc_device(self._h, _ptr(features_bf16), int(T.numel()), _ptr(T)))

    def set_profiler(self, fn):
        """fn(frame: str, depth: int, ms: float) after every render (the reference's
        SetProfiler frames: Render > Phase 1 / Phase 4 / Phase 5); None removes it."""
        if fn is None:
            self._profile_cb = None
            self._check(self._L.beams_set_profiler(self._h, None, None))
            return
        cb = PROFILE_FN(lambda _user, frame, depth, ms: fn(frame.decode(), depth, ms))
        self._profile_cb = cb  # kept alive while set
        self._check(self._L.beams_set_profiler(self._h, C.cast(cb, C.c_void_p), None))

    def mlp_set_tensor_cores(self, enable: bool):
        self._check(self._L.beams_mlp_set_tensor_cores(self._h, int(bool(enable))))

    def mlp_set_probe_first(self, mode: int):
        """Learned-frame order: 1 probe pixels first, 0 network first, -1 chosen per frame."""
        self._check(self._L.beams_mlp_set_probe_first(self._h, int(mode)))

    def mlp_probe_errors(self, n):
        out = np.empty(n, np.float32)
        self._check(self._L.beams_mlp_probe_errors(self._h, _ptr(out), int(n)))
        return out

    def mlp_save(self, path):
        self._check(self._L.beams_mlp_save(self._h, str(path).encode()))

    def mlp_load(self, path):
        self._check(self._L.beams_mlp_load(self._h, str(path).encode()))

    def set_color_map(self, rgba):
        t = np.ascontiguousarray(rgba, dtype=np.float32).reshape(-1, 4)
        self._check(self._L.beams_set_color_map(self._h, _ptr(t), t.shape[0]))

    def set_shadow_map_size(self, mx, my=None, mz=None):
        my = mx if my is None else my
        mz = mx if mz is None else mz
        self._check(self._L.beams_set_shadow_map_size(self._h, int(mx), int(my), int(mz)))

    def set_use_shadow_map(self, on: bool):
        self._check(self._L.beams_set_use_shadow_map(self._h, int(bool(on))))

    def clear_lights(self):
        self._check(self._L.beams_clear_lights(self._h))

    def add_point_light(self, pos, color=(1, 1, 1), intensity=1.0):
        self._check(self._L.beams_add_point_light(self._h, _d3(pos), _f3(color), float(intensity)))

    def add_directional_light(self, direction, color=(1, 1, 1), intensity=1.0):
        self._check(self._L.beams_add_directional_light(self._h, _d3(direction), _f3(color), float(intensity)))

    def set_sample_distance(self, d):
        self._check(self._L.beams_set_sample_distance(self._h, float(d)))

    def set_density_scale(self, scale):
        """MapperLightedVolume::SetDensityScale: stored, no effect on the image (as in the reference)."""
        self._check(self._L.beams_set_density_scale(self._h, float(scale)))

    def get_density_scale(self):
        v = C.c_float()
        self._check(self._L.beams_get_density_scale(self._h, C.byref(v)))
        return v.value

    def set_termination_alpha(self, a):
        self._check(self._L.beams_set_termination_alpha(self._h, float(a)))

    def set_light_steps(self, s):
        self._check(self._L.beams_set_light_steps(self._h, float(s)))

    def set_slab_fp64(self, on: bool):
        self._check(self._L.beams_set_slab_fp64(self._h, int(bool(on))))

    def set_reuse_shadow_map(self, on: bool):
        self._check(self._L.beams_set_reuse_shadow_map(self._h, int(bool(on))))

    def set_lazy_shadow_map(self, on: bool, keep_marks: bool = False):
        """Build only the map vertices the frame's view rays read (exact form);
        keep_marks keeps the marked cells while the view's inputs are unchanged."""
        self._check(self._L.beams_set_lazy_shadow_map(self._h, (2 if keep_marks else 1) if on else 0))

    def set_background(self, on: bool, rgba=(1, 1, 1, 1)):
        c = (C.c_float * 4)(*rgba)
        self._check(self._L.beams_set_background(self._h, int(bool(on)), c))

    def set_volume_coordinates(self, x=None, y=None, z=None):
        """Explicit rectilinear coordinates of the current volume (float32,
        strictly increasing, dims[d] values per axis); no arguments: uniform again."""
        if x is None and y is None and z is None:
            self._check(self._L.beams_set_volume_coordinates(self._h, None, None, None))
            return
        self._coords = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
        self._check(self._L.beams_set_volume_coordinates(self._h, *[_ptr(a) for a in self._coords]))

    def set_depth_buffer(self, depth, kind=0, near=0.0, far=0.0):
        """Canvas depth clipping: depth (H, W) float32 numpy or torch CUDA tensor,
        kind DEPTH_RAY_DISTANCE or DEPTH_WINDOW (with near/far); None clears."""
        if depth is None:
            self._check(self._L.beams_set_depth_buffer(self._h, None, 0, 0, 0, 0.0, 0.0, 0))
            return
        if isinstance(depth, np.ndarray):
            depth = np.ascontiguousarray(depth, np.float32)
            on_dev = 0
        else:
            on_dev = int(depth.is_cuda)
        h, w = depth.shape
        self._check(self._L.beams_set_depth_buffer(self._h, _ptr(depth), int(w), int(h), int(kind), float(near),
                                                   float(far), on_dev))

    def get_ray_limits(self, cam):
        out = np.empty((cam.height, cam.width), np.float32)
        self._check(self._L.beams_get_ray_limits(self._h, C.byref(cam), _ptr(out), 0))
        return out

    def set_multi_light(self, enable: bool):
        self._check(self._L.beams_set_multi_light(self._h, int(bool(enable))))

    def set_tuning(self, light_brick: int = 8, empty_skip: bool = True, view_skip: bool = True):
        t = Tuning(int(light_brick), 0 if empty_skip else 1, 0 if view_skip else 1)
        self._check(self._L.beams_set_tuning(self._h, C.byref(t)))

    def get_tuning(self):
        t = Tuning()
        self._check(self._L.beams_get_tuning(self._h, C.byref(t)))
        return {"light_brick": t.light_brick, "empty_skip": not t.no_empty_skip, "view_skip": not t.no_view_skip}

    def autotune(self, cam=None):
        """Picks the fastest tuning for the current scene (the view march too when a
        camera is given); returns it with the map-build and view-march times."""
        t, ms, vms = Tuning(), C.c_float(), C.c_float()
        self._check(self._L.beams_autotune(self._h, C.byref(cam) if cam is not None else None, C.byref(t),
                                           C.byref(ms), C.byref(vms)))
        return {"light_brick": t.light_brick, "empty_skip": not t.no_empty_skip, "view_skip": not t.no_view_skip,
                "map_ms": ms.value, "view_ms": vms.value}

    def set_form(self, form: int, field_dtype=BF16):
        """FORM_EXACT; FORM_PRECISION with the 16-bit field dtype (BF16 or F16);
        FORM_MLP with an MlpOptions (its knot, probe_fraction and fallback_tol
        are read; None takes the defaults)."""
        opts = None
        if form == FORM_PRECISION:
            self._prec_opts = (C.c_int * 1)(int(field_dtype))
            opts = C.cast(self._prec_opts, C.c_void_p)
        elif form == FORM_MLP and isinstance(field_dtype, MlpOptions):
            self._mlp_render_opts = field_dtype
            opts = C.cast(C.pointer(self._mlp_render_opts), C.c_void_p)
        self._check(self._L.beams_set_form(self._h, int(form), opts))

    # -- render ---------------------------------------------------------------
    @staticmethod
    def camera(position, look_at, up, fov_y_deg, width, height) -> Camera:
        return Camera(_d3(position), _d3(look_at), _d3(up), float(fov_y_deg), int(width), int(height))

    def render(self, cam: Camera, out=None, timings=True, host_async=False):
        """Renders into out (numpy (H,W,4) float32 host array or torch tensor, CUDA
        or host). host_async with a pinned host tensor queues the copy and returns
        at once (OUT_HOST_ASYNC): call synchronize() before reading out."""
        if out is None:
            out = np.zeros((cam.height, cam.width, 4), np.float32)
        on_dev = OUT_HOST if isinstance(out, np.ndarray) else (OUT_DEVICE if out.is_cuda else OUT_HOST)
        if host_async:
            if on_dev != OUT_HOST or isinstance(out, np.ndarray) or not out.is_pinned():
                raise ValueError("host_async needs a pinned host torch tensor")
            on_dev = OUT_HOST_ASYNC
        t = Timings() if timings else None
        self._check(self._L.beams_render(self._h, C.byref(cam), _ptr(out), on_dev,
                                         C.byref(t) if t is not None else None))
        return out, (t.as_dict() if t is not None else None)

    def synchronize(self):
        self._check(self._L.beams_synchronize(self._h))

    def build_shadow_map(self, timings=True):
        """Phase 1 only. With timings=False nothing synchronises."""
        t = Timings() if timings else None
        self._check(self._L.beams_build_shadow_map(self._h, C.byref(t) if t is not None else None))
        return t.as_dict() if t is not None else None

    def get_shadow_map(self, count):
        m = np.empty(count, np.float32)
        self._check(self._L.beams_get_shadow_map(self._h, _ptr(m), m.size, 0))
        return m


def vtk_read(path):
    """Reads a legacy VTK structured volume (beams_vtk_read): a dict with dims
    (point dims, x y z), assoc, origin, spacing, coords (three arrays for a
    rectilinear grid, else None), data (float32, shape z, y, x of points or
    cells), range and name."""
    L = lib()
    f = VtkField()
    st = L.beams_vtk_read(str(path).encode(), C.byref(f))
    if st != BEAMS_OK:
        raise BeamsError(st, L.beams_last_error(None).decode())
    try:
        nx, ny, nz = f.dims
        shape = (nz, ny, nx) if f.assoc == ASSOC_POINTS else (nz - 1, ny - 1, nx - 1)
        n = int(np.prod(shape))
        data = np.ctypeslib.as_array(f.data, shape=(n,)).copy().reshape(shape)
        coords = None
        if f.coords[0]:
            coords = [np.ctypeslib.as_array(f.coords[d], shape=(f.dims[d],)).copy() for d in range(3)]
        return {"dims": tuple(f.dims), "assoc": f.assoc, "origin": tuple(f.origin), "spacing": tuple(f.spacing),
                "coords": coords, "data": data, "range": tuple(f.range), "name": f.name.decode()}
    finally:
        L.beams_vtk_free(C.byref(f))


def selftest_division(origin: float, spacing: float, ncells: int, samples: int):
    """(checked, mismatches) of the kernels' division against IEEE division."""
    L = lib()
    chk, bad = C.c_ulonglong(), C.c_ulonglong()
    st = L.beams_selftest_division(origin, spacing, ncells, samples, C.byref(chk), C.byref(bad))
    if st != BEAMS_OK:
        raise BeamsError(st, L.beams_last_error(None).decode())
    return chk.value, bad.value


class MapperLightedVolume:
    """Mirror of beams::rendering::MapperLightedVolume over the C ABI.

    Reference: beams/rendering/MapperLightedVolume.h:16-62, .cxx:47-324.
    RenderCells takes the field, its bounds and range, a camera and returns the
    premultiplied RGBA canvas (the reference writes a CanvasRayTracer).
    """

    def __init__(self, device: int = 0):
        self._r = Renderer(device)
        self._width = self._height = None
        self._sample_distance = -1.0  # DEFAULT_SAMPLE_DISTANCE (MapperLightedVolume.cxx:19)
        self._color_map = None

    def SetCanvas(self, width: int, height: int):
        self._width, self._height = int(width), int(height)

    def SetShadowMapSize(self, size):
        sx, sy, sz = (size, size, size) if np.isscalar(size) else size
        self._r.set_shadow_map_size(sx, sy, sz)

    def SetUseShadowMap(self, use: bool):
        self._r.set_use_shadow_map(use)

    def AddLight(self, position, color=(1, 1, 1), intensity=1.0):
        self._r.add_point_light(position, color, intensity)

    def ClearLights(self):
        self._r.clear_lights()

    def SetSampleDistance(self, d: float):
        # Stored; validated when rendering, like the reference (LightedVolumeRenderer.cxx:1374-1379).
        self._sample_distance = float(d)

    def SetCompositeBackground(self, on: bool, rgba=(1, 1, 1, 1)):
        self._r.set_background(on, rgba)

    def SetDensityScale(self, s: float):
        self._r.set_density_scale(s)  # stored, never read (as in the reference)

    def SetActiveColorTable(self, rgba_table):
        self._color_map = np.asarray(rgba_table, np.float32).reshape(-1, 4)

    def RenderCells(self, field, origin, spacing, scalar_range, camera: dict, assoc=ASSOC_POINTS):
        if self._width is None:
            raise BeamsError(1, "Ray Tracer: no canvas set")
        if self._color_map is None:
            raise BeamsError(8, "no active color table")
        if self._sample_distance != -1.0:
            self._r.set_sample_distance(self._sample_distance)
        self._r.set_volume(field, origin=origin, spacing=spacing, value_range=scalar_range, assoc=assoc)
        self._r.set_color_map(self._color_map)
        cam = Renderer.camera(camera["position"], camera["look_at"], camera.get("up", (0, 1, 0)),
                              camera.get("fov_y_deg", 30.0), self._width, self._height)
        img, t = self._r.render(cam)
        self.last_timings = t
        return img

    @property
    def renderer(self) -> Renderer:
        return self._r
