"""Seeded synthetic scenes for the Beams renderer (tests and benchmarks).

The reference's data files are not shipped and the benchmark workloads use
synthetic fields, so every scene here is generated from a seed:

* ``config0``: 128^3 float32 sum of 8 Gaussian blobs (centres U[0.2,0.8]^3,
  sigma U[0.05,0.15], amplitude U[0.5,1]) normalised to [0,1]; 512x512 image,
  camera on the unit sphere around the centre (seeded direction), fov 30 deg;
  one directional light (seeded); map M = 128; step 0.5 voxel; alpha cut 0.99.
* ``config1``: 512^3 float32 4-octave gradient noise (lacunarity 2, gain 0.5)
  remapped to [0,1]; 1024x1024 image; point light at 2x the domain diagonal
  along a seeded direction; map M = 256; step 0.5 voxel; alpha cut 0.99.
* ``config2``: 1024^3 sum of 64 blobs plus 10% gradient noise, normalised;
  2048x2048 image; M = 512; step 0.25 voxel (the precision form's workload).

The domain is the unit cube, spacing 1/(N-1). The transfer function is a
256-entry table: alpha piecewise-linear through (0.2, 0), (0.4, 0.05),
(0.6, 0.2), (0.8, 0.6), clamped outside; RGB a linear blue-to-orange ramp.
"""
from __future__ import annotations

from dataclasses import dataclass, field as dc_field

import numpy as np

TF_POINTS = ((0.2, 0.0), (0.4, 0.05), (0.6, 0.2), (0.8, 0.6))
RGB_LO = np.array([0.23, 0.30, 0.75], np.float64)
RGB_HI = np.array([0.95, 0.55, 0.10], np.float64)


def tf_table(n: int = 256, points=TF_POINTS) -> np.ndarray:
    v = np.arange(n, dtype=np.float64) / (n - 1)
    xs = np.array([p[0] for p in points])
    ys = np.array([p[1] for p in points])
    a = np.interp(v, xs, ys)  # clamps to the end values outside [0.2, 0.8]
    rgb = RGB_LO[None, :] * (1 - v[:, None]) + RGB_HI[None, :] * v[:, None]
    return np.concatenate([rgb, a[:, None]], axis=1).astype(np.float32)


def random_unit(rng: np.random.Generator) -> np.ndarray:
    while True:
        v = rng.normal(size=3)
        n = np.linalg.norm(v)
        if n > 1e-6:
            return v / n


def blob_params(rng: np.random.Generator, nblobs: int = 8) -> np.ndarray:
    c = rng.uniform(0.2, 0.8, size=(nblobs, 3))
    s = rng.uniform(0.05, 0.15, size=(nblobs, 1))
    a = rng.uniform(0.5, 1.0, size=(nblobs, 1))
    return np.concatenate([c, s, a], axis=1).astype(np.float32)


def _normalise(v: np.ndarray) -> np.ndarray:
    lo, hi = float(v.min()), float(v.max())
    if hi > lo:
        v = (v - np.float32(lo)) * np.float32(1.0 / (hi - lo))
    return np.clip(v, 0, 1).astype(np.float32)


def blobs_numpy(n, params: np.ndarray, normalise: bool = True) -> np.ndarray:
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    z = (np.arange(nz, dtype=np.float32) / np.float32(nz - 1))[:, None, None]
    y = (np.arange(ny, dtype=np.float32) / np.float32(ny - 1))[None, :, None]
    x = (np.arange(nx, dtype=np.float32) / np.float32(nx - 1))[None, None, :]
    v = np.zeros((nz, ny, nx), np.float32)
    for cx, cy, cz, s, a in params:
        r2 = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2
        v += np.float32(a) * np.exp(-r2 / np.float32(2 * s * s)).astype(np.float32)
    return _normalise(v) if normalise else v


def _fade(t):
    return t * t * t * (t * (t * 6 - 15) + 10)


def _grad(h, x, y, z):
    h = h & 15
    u = np.where(h < 8, x, y)
    v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
    return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)


def perlin_numpy(x, y, z, perm: np.ndarray):
    """Gradient noise after Perlin's "Improving Noise" (2002)."""
    P = perm.astype(np.int64)
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    X, Y, Z = fx.astype(np.int64) & 255, fy.astype(np.int64) & 255, fz.astype(np.int64) & 255
    x, y, z = x - fx, y - fy, z - fz
    u, v, w = _fade(x), _fade(y), _fade(z)
    A = P[X] + Y
    AA, AB = P[A & 255] + Z, P[(A + 1) & 255] + Z
    B = P[(X + 1) & 255] + Y
    BA, BB = P[B & 255] + Z, P[(B + 1) & 255] + Z

    def L(t, a, b):
        return a + t * (b - a)

    return L(w,
             L(v, L(u, _grad(P[AA & 255], x, y, z), _grad(P[BA & 255], x - 1, y, z)),
               L(u, _grad(P[AB & 255], x, y - 1, z), _grad(P[BB & 255], x - 1, y - 1, z))),
             L(v, L(u, _grad(P[(AA + 1) & 255], x, y, z - 1), _grad(P[(BA + 1) & 255], x - 1, y, z - 1)),
               L(u, _grad(P[(AB + 1) & 255], x, y - 1, z - 1), _grad(P[(BB + 1) & 255], x - 1, y - 1, z - 1))))


def noise_numpy(n, perm, octaves=4, base_freq=4.0, lacunarity=2.0, gain=0.5) -> np.ndarray:
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    z = (np.arange(nz, dtype=np.float32) / np.float32(nz - 1))[:, None, None]
    y = (np.arange(ny, dtype=np.float32) / np.float32(ny - 1))[None, :, None]
    x = (np.arange(nx, dtype=np.float32) / np.float32(nx - 1))[None, None, :]
    x, y, z = np.broadcast_arrays(x, y, z)
    v = np.zeros((nz, ny, nx), np.float32)
    f, a = np.float32(base_freq), np.float32(1.0)
    for _ in range(octaves):
        v += (a * perlin_numpy(x * f, y * f, z * f, perm)).astype(np.float32)
        f *= np.float32(lacunarity)
        a *= np.float32(gain)
    return _normalise(v)


@dataclass
class Scene:
    name: str
    dims: tuple
    kind: str                      # "blobs" | "noise" | "array"
    params: np.ndarray | None      # blob params or permutation
    tf: np.ndarray
    light_kind: int                # 0 point, 1 directional
    light: tuple
    light_color: tuple = (1.0, 1.0, 1.0)
    light_intensity: float = 1.0
    map_m: int = 16
    sample_distance: float = -1.0
    cutoff: float = 1.0
    light_steps: float = 128.0
    cam_pos: tuple = (0.5, 0.5, 2.0)
    cam_look: tuple = (0.5, 0.5, 0.5)
    cam_up: tuple = (0.0, 1.0, 0.0)
    fov_y_deg: float = 30.0
    width: int = 64
    height: int = 64
    origin: tuple = (0.0, 0.0, 0.0)
    value_range: tuple = (0.0, 1.0)
    use_map: bool = True
    slab_fp64: bool = True
    array: np.ndarray | None = dc_field(default=None, repr=False)
    octaves: int = 4
    base_freq: float = 4.0

    brick_spacing: tuple | None = None
    noise_amp: float = 0.1

    @property
    def spacing(self):
        if self.brick_spacing is not None:
            return self.brick_spacing
        return tuple(1.0 / (d - 1) for d in self.dims)

    def field_numpy(self) -> np.ndarray:
        if self.array is not None:
            return self.array
        if self.kind == "blobs":
            self.array = blobs_numpy(self.dims, self.params)
        elif self.kind == "noise":
            self.array = noise_numpy(self.dims, self.params, self.octaves, self.base_freq)
        elif self.kind == "blobnoise":
            b = blobs_numpy(self.dims, self.params[0])
            nz = noise_numpy(self.dims, self.params[1], self.octaves, self.base_freq)
            self.array = _normalise(b + np.float32(self.noise_amp) * nz)
        else:
            raise ValueError(self.kind)
        return self.array

    def field_device(self, lib_handle=None):
        """Generates the field on the current CUDA device (torch tensor)."""
        import ctypes as C

        import torch

        from . import beams as B
        L = lib_handle or B.lib()
        nx, ny, nz = self.dims
        t = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
        n = (C.c_int * 3)(nx, ny, nz)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        if self.kind == "blobs":
            p = np.ascontiguousarray(self.params, np.float32)
            st = L.beams_generate_blobs(C.c_void_p(t.data_ptr()), n, p.ctypes.data_as(C.c_void_p),
                                        p.shape[0], 1, stream)
        elif self.kind == "noise":
            p = np.ascontiguousarray(self.params, np.uint8)
            st = L.beams_generate_noise(C.c_void_p(t.data_ptr()), n, p.ctypes.data_as(C.c_void_p),
                                        self.octaves, self.base_freq, 2.0, 0.5, stream)
        elif self.kind == "blobnoise":
            p = np.ascontiguousarray(self.params[0], np.float32)
            st = L.beams_generate_blobs(C.c_void_p(t.data_ptr()), n, p.ctypes.data_as(C.c_void_p),
                                        p.shape[0], 1, stream)
            if st == 0:
                nz = torch.empty_like(t)
                q = np.ascontiguousarray(self.params[1], np.uint8)
                st = L.beams_generate_noise(C.c_void_p(nz.data_ptr()), n, q.ctypes.data_as(C.c_void_p),
                                            self.octaves, self.base_freq, 2.0, 0.5, stream)
                if st == 0:
                    t.add_(nz, alpha=self.noise_amp)
                    del nz
                    lo, hi = t.min(), t.max()
                    t.sub_(lo).mul_(1.0 / (hi - lo)).clamp_(0, 1)
        else:
            return torch.from_numpy(self.field_numpy()).cuda()
        if st != 0:
            raise B.BeamsError(st, L.beams_last_error(None).decode())
        return t

    def configure(self, r) -> None:
        """Applies every setting except the volume to a Renderer."""
        r.set_color_map(self.tf)
        if isinstance(self.map_m, (tuple, list)):
            r.set_shadow_map_size(*self.map_m)
        else:
            r.set_shadow_map_size(self.map_m)
        r.set_use_shadow_map(self.use_map)
        r.clear_lights()
        if self.light_kind == 0:
            r.add_point_light(self.light, self.light_color, self.light_intensity)
        else:
            r.add_directional_light(self.light, self.light_color, self.light_intensity)
        if self.sample_distance > 0:
            r.set_sample_distance(self.sample_distance)
        r.set_termination_alpha(self.cutoff)
        r.set_light_steps(self.light_steps)
        r.set_slab_fp64(self.slab_fp64)

    def camera(self):
        from .beams import Renderer
        return Renderer.camera(self.cam_pos, self.cam_look, self.cam_up, self.fov_y_deg, self.width, self.height)


def _unit_sphere_camera(rng):
    d = random_unit(rng)
    pos = tuple(float(x) for x in (np.array([0.5, 0.5, 0.5]) + d))
    up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.9 else (1.0, 0.0, 0.0)
    return pos, up


def config0(seed: int = 0, n: int = 128, image: int = 512, m: int = 128, cutoff: float = 0.99) -> Scene:
    rng = np.random.default_rng(seed)
    params = blob_params(rng, 8)
    pos, up = _unit_sphere_camera(rng)
    ldir = tuple(float(x) for x in random_unit(rng))
    return Scene(name=f"blobs{n}_img{image}_M{m}", dims=(n, n, n), kind="blobs", params=params, tf=tf_table(),
                 light_kind=1, light=ldir, map_m=m, sample_distance=0.5 / (n - 1), cutoff=cutoff,
                 cam_pos=pos, cam_up=up, width=image, height=image)


def config1(seed: int = 1, n: int = 512, image: int = 1024, m: int = 256, cutoff: float = 0.99) -> Scene:
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256).astype(np.uint8)
    pos, up = _unit_sphere_camera(rng)
    ldir = random_unit(rng)
    diag = np.sqrt(3.0)
    lpos = tuple(float(x) for x in (np.array([0.5, 0.5, 0.5]) + 2.0 * diag * ldir))
    return Scene(name=f"noise{n}_img{image}_M{m}", dims=(n, n, n), kind="noise", params=perm, tf=tf_table(),
                 light_kind=0, light=lpos, map_m=m, sample_distance=0.5 / (n - 1), cutoff=cutoff,
                 cam_pos=pos, cam_up=up, width=image, height=image)


def config2(seed: int = 2, n: int = 1024, image: int = 2048, m: int = 512, cutoff: float = 0.99) -> Scene:
    """The precision form's workload: 64 Gaussian blobs plus 10% gradient noise,
    normalised to [0,1]; 2048^2 image; M = 512 map; view step 0.25 voxel; point
    light at 2x the diagonal."""
    rng = np.random.default_rng(seed)
    params = blob_params(rng, 64)
    perm = rng.permutation(256).astype(np.uint8)
    pos, up = _unit_sphere_camera(rng)
    ldir = random_unit(rng)
    lpos = tuple(float(x) for x in (np.array([0.5, 0.5, 0.5]) + 2.0 * np.sqrt(3.0) * ldir))
    return Scene(name=f"blobnoise{n}_img{image}_M{m}", dims=(n, n, n), kind="blobnoise", params=(params, perm),
                 tf=tf_table(), light_kind=0, light=lpos, map_m=m, sample_distance=0.25 / (n - 1), cutoff=cutoff,
                 cam_pos=pos, cam_up=up, width=image, height=image, base_freq=8.0)


def small(seed: int = 0, n: int = 24, image: int = 48, m: int = 12, kind: str = "blobs", light_kind: int = 0,
          cutoff: float = 1.0) -> Scene:
    """A small seeded scene that the CPU oracle finishes in well under a second."""
    rng = np.random.default_rng(seed)
    if kind == "blobs":
        params = blob_params(rng, 8)
    else:
        params = rng.permutation(256).astype(np.uint8)
    pos, up = _unit_sphere_camera(rng)
    ldir = random_unit(rng)
    light = tuple(float(x) for x in ldir) if light_kind == 1 else \
        tuple(float(x) for x in (np.array([0.5, 0.5, 0.5]) + 2.0 * np.sqrt(3.0) * ldir))
    return Scene(name=f"small_{kind}{n}", dims=(n, n, n), kind=kind, params=params, tf=tf_table(),
                 light_kind=light_kind, light=light, map_m=m, sample_distance=0.5 / (n - 1), cutoff=cutoff,
                 cam_pos=pos, cam_up=up, width=image, height=image, base_freq=2.0)


def split_bricks(s: Scene, splits=(2, 2, 2)) -> list:
    """Splits a scene's field into bricks, one dataset per brick as the reference's
    ranks hold them: the cells of each axis are cut into `splits` contiguous runs
    and neighbouring bricks share the point plane between them. Each brick keeps
    the scene's camera, light, TF, map size and sample distance."""
    from dataclasses import replace
    field = s.field_numpy()
    nx, ny, nz = s.dims
    h = s.spacing
    cuts = []
    for n, k in zip((nx, ny, nz), splits):
        cells = n - 1
        edges = [round(i * cells / k) for i in range(k + 1)]
        cuts.append([(edges[i], edges[i + 1]) for i in range(k)])  # cell ranges [a, b)
    bricks = []
    for (z0, z1) in cuts[2]:
        for (y0, y1) in cuts[1]:
            for (x0, x1) in cuts[0]:
                sub = np.ascontiguousarray(field[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1])
                org = (s.origin[0] + x0 * h[0], s.origin[1] + y0 * h[1], s.origin[2] + z0 * h[2])
                b = replace(s, name=f"{s.name}_brick{len(bricks)}", dims=(x1 - x0 + 1, y1 - y0 + 1, z1 - z0 + 1),
                            kind="array", params=None, array=sub, origin=org)
                b.brick_spacing = h
                bricks.append(b)
    return bricks
