"""Scenes from a stage TOML: the reference's sphere dataset generated on the
device (bit-exact against the oracle's restatement), the applied scene rendered
bit-exactly against the oracle, the light orbit, and the beams_run driver."""
import json
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle.oracle import Oracle, noise_field, spheres_field
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent

CONFIG = '''
[dataset_providers.spheres]
type = "subdivided_spheres"
cell_dims = [40, 36, 44]

[render]
width = 64
height = 56
termination_alpha = 1.0

[shadow_map]
size_ratio = 0.25
num_steps = 128

[camera]
azimuth = 35.0
elevation = 25.0
'''


def test_spheres_field_matches_oracle(cuda_device):
    dims = (37, 29, 33)
    org, sp = (0.1, -0.2, 0.05), (1 / 36, 1 / 28, 1 / 32)
    ell = np.array([[0.5, 0.3, 0.5, 0.3, 0.2, 0.25, 0.2, 1.0],
                    [0.6, 0.1, 0.4, 0.15, 0.15, 0.15, 0.9, 0.4],
                    [0.3, 0.0, 0.6, 0.2, 0.35, 0.1, 0.5, 0.5]], np.float32)
    t = torch.empty((dims[2], dims[1], dims[0]), device="cuda")
    import ctypes as C
    L = B.lib()
    st = L.beams_generate_spheres(C.c_void_p(t.data_ptr()), (C.c_int * 3)(*dims), (C.c_double * 3)(*org),
                                  (C.c_double * 3)(*sp), ell.ctypes.data_as(C.c_void_p), 3, 0.1, 1, -0.01, 0.7,
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    ref = spheres_field(dims, org, sp, ell, default=0.1, floor=(-0.01, 0.7))
    assert np.array_equal(t.cpu().numpy(), ref)


def test_device_noise_equals_oracle_noise_config1(cuda_device):
    """The benchmark's 512^3 gradient-noise field (the config-1 seed): the device
    generator (beams_generate_noise, what the GPU arm renders) and the oracle's
    CPU generator (what the reference arm renders) give the same float32 field
    bit for bit, the [0, 1] normalisation included."""
    s = scenes.config1()
    fd = s.field_device()
    torch.cuda.synchronize()
    dev = fd.cpu().numpy()
    del fd
    ref = noise_field(s.dims, s.params, s.octaves, s.base_freq)
    assert dev.shape == ref.shape
    assert np.array_equal(dev, ref), f"{int(np.sum(dev != ref))} of {dev.size} values differ"
    assert dev.min() == 0.0 and dev.max() == 1.0


def _oracle_scene(d, cam, field, light, intensity):
    dims = tuple(c + 1 for c in d.cell_dims)
    m = int(d.cell_dims[0] * d.shadow_size_ratio)
    s = scenes.Scene(name="cfg", dims=dims, kind="array", params=None, tf=B.scene_color_table(d),
                     light_kind=0, light=light, light_color=(1.0, 1.0, 1.0), light_intensity=intensity,
                     map_m=m, sample_distance=-1.0, cutoff=d.termination_alpha, light_steps=d.light_steps,
                     cam_pos=tuple(cam.position), cam_look=tuple(cam.look_at), cam_up=tuple(cam.up),
                     fov_y_deg=cam.fov_y_deg, width=cam.width, height=cam.height, array=field)
    s.brick_spacing = tuple(1.0 / c for c in d.cell_dims)
    return s


def test_applied_scene_renders_like_the_oracle(cuda_device):
    d = B.parse_config(CONFIG)
    with B.Renderer(0) as r:
        cam = r.apply_scene(d)
        img, t = r.render(cam)
        dims = tuple(c + 1 for c in d.cell_dims)
        field = spheres_field(dims, (0, 0, 0), tuple(1.0 / c for c in d.cell_dims),
                              [0.5, 0.5, 0.5, 0.45, 0.45, 0.45, 1.0, 1.0], default=0.1)
        s = _oracle_scene(d, cam, field, (0.5, 5.0, 0.5), 2.0)
        m = [int(c * d.shadow_size_ratio) for c in d.cell_dims]
        assert t["map_vertices"] == (m[0] + 1) * (m[1] + 1) * (m[2] + 1)
        # the oracle scene uses one map size per axis: compare the map and image only when cubic
        r.set_shadow_map_size(m[0])
        img, t = r.render(cam)
        o = Oracle(s)
        om, _ = o.light_march()
        gm = r.get_shadow_map((m[0] + 1) ** 3)
        assert np.array_equal(gm, om.ravel())
        oimg, lit = o.view_march(om)
        assert np.array_equal(img, oimg) and t["lit_samples"] == lit
        assert img[..., 3].max() > 0.5  # the sphere is in view
        # the light orbit of the driver loop: frame 18 = 90 degrees
        r.orbit_light(d, 18)
        img2, _ = r.render(cam)
        s2 = _oracle_scene(d, cam, field, (0.5, 1.0, 0.5), 2.0)
        o2 = Oracle(s2)
        om2, _ = o2.light_march()
        oimg2, _ = o2.view_march(om2)
        assert np.array_equal(img2, oimg2) and not np.array_equal(img2, img)


def _read_png(path):
    b = Path(path).read_bytes()
    assert b[:8] == bytes([137, 80, 78, 71, 13, 10, 26, 10])
    pos, idat = 8, b""
    w = h = None
    while pos < len(b):
        n = int.from_bytes(b[pos:pos + 4], "big")
        typ = b[pos + 4:pos + 8]
        data = b[pos + 8:pos + 8 + n]
        if typ == b"IHDR":
            w, h = int.from_bytes(data[:4], "big"), int.from_bytes(data[4:8], "big")
        elif typ == b"IDAT":
            idat += data
        assert zlib.crc32(typ + data) == int.from_bytes(b[pos + 8 + n:pos + 12 + n], "big")
        pos += 12 + n
    raw = zlib.decompress(idat)
    assert len(raw) == h * (4 * w + 1)
    return w, h


def test_driver_runs_the_light_orbit(cuda_device, tmp_path):
    cfg = tmp_path / "stage.toml"
    cfg.write_text(CONFIG.replace("[render]", "[render]\ncomposite_background = true"))
    exe = ROOT / "pilot_b200" / "bin" / "beams_run"
    p = subprocess.run([str(exe), f"--base-dir={tmp_path}", "--frames=3", f"--out={tmp_path}"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = [json.loads(x) for x in p.stdout.strip().splitlines()]
    assert [x["frame"] for x in lines] == [0, 1, 2] and all(x["lit_samples"] > 0 for x in lines)
    for k in range(3):
        assert _read_png(tmp_path / f"spheres_0_{k:03d}.png") == (64, 56)
    # the lazy map with kept marks (the camera is fixed, the light orbits): the
    # same images byte for byte
    lazy_dir = tmp_path / "lazy"
    lazy_dir.mkdir()
    p = subprocess.run([str(exe), f"--base-dir={tmp_path}", "--frames=3", f"--out={lazy_dir}", "--lazy-shadow-map"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lazy_lines = [json.loads(x) for x in p.stdout.strip().splitlines()]
    assert [x["lit_samples"] for x in lazy_lines] == [x["lit_samples"] for x in lines]
    for k in range(3):
        name = f"spheres_0_{k:03d}.png"
        assert (lazy_dir / name).read_bytes() == (tmp_path / name).read_bytes(), name


def test_vtk_file_scene_renders_like_the_oracle(cuda_device, tmp_path):
    """A stage whose dataset is a legacy VTK file (a rectilinear grid here):
    beams_load_config_toml resolves the file next to the stage file,
    beams_apply_scene reads it and the render matches the oracle on the same
    coordinates and values bit for bit."""
    from test_vtk_cpu import write_vtk
    n = 33
    rng = np.random.default_rng(5)
    field = scenes.noise_numpy(n, rng.permutation(256).astype(np.uint8), base_freq=3.0).astype(np.float32)
    t = np.linspace(0.0, 1.0, n)
    coords = [np.float32(t ** 1.3), np.float32(t), np.float32(0.5 * (t + t ** 2))]
    write_vtk(tmp_path / "vol.vtk", field, True, kind="RECTILINEAR_GRID", coords=coords)
    (tmp_path / "stage.toml").write_text('''
[dataset_providers.volume]
type = "vtk_file"
file_name = "vol.vtk"

[render]
width = 48
height = 40
termination_alpha = 1.0

[shadow_map]
size_ratio = 0.5

[camera]
azimuth = 30.0
elevation = 20.0
''')
    d = B.load_config(tmp_path / "stage.toml")
    assert d.file_name.decode() == str(tmp_path / "vol.vtk")
    with B.Renderer(0) as r:
        cam = r.apply_scene(d)
        img, tt = r.render(cam)
        m = int((n - 1) * d.shadow_size_ratio)
        s = scenes.Scene(name="vtk", dims=(n, n, n), kind="array", params=None, tf=B.scene_color_table(d),
                         light_kind=0, light=(0.5, 5.0, 0.5), light_color=(1.0, 1.0, 1.0), light_intensity=2.0,
                         map_m=m, sample_distance=-1.0, cutoff=d.termination_alpha, light_steps=d.light_steps,
                         cam_pos=tuple(cam.position), cam_look=tuple(cam.look_at), cam_up=tuple(cam.up),
                         fov_y_deg=cam.fov_y_deg, width=cam.width, height=cam.height, array=field,
                         value_range=(float(field.min()), float(field.max())))
        s.coords = coords
        o = Oracle(s)
        om, _ = o.light_march()
        assert np.array_equal(r.get_shadow_map((m + 1) ** 3), om.ravel())
        oimg, lit = o.view_march(om)
        assert np.array_equal(img, oimg) and tt["lit_samples"] == lit
        assert img[..., 3].max() > 0.1
