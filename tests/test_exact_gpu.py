"""Parity of the exact form (K1 light march, K2 view march) against the CPU oracle.

Tolerances:
  * map (K1) vs oracle f32 mode: bit-exact (both compute the same IEEE float32
    operations in the same order; -fmad=false on the device);
  * image (K2) vs oracle f32 mode: max per-pixel |dRGBA| <= 2e-3 (the plain-path
    bar); the fraction of bit-identical pixels is reported and expected ~1;
  * every image also reports its error against the FP64 oracle (PSNR).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, psnr
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def gpu_render(s, field=None, renderer=None):
    r = renderer or B.Renderer(0)
    r.set_volume(s.field_numpy() if field is None else field, origin=s.origin, spacing=s.spacing,
                 value_range=s.value_range)
    s.configure(r)
    img, t = r.render(s.camera())
    m = r.get_shadow_map((s.map_m + 1) ** 3).reshape((s.map_m + 1,) * 3) if s.use_map else None
    return img, m, t, r


SMALL = [
    dict(seed=0, kind="blobs", light_kind=0),
    dict(seed=1, kind="blobs", light_kind=1),
    dict(seed=2, kind="noise", light_kind=0),
    dict(seed=3, kind="noise", light_kind=1),
]


@pytest.mark.parametrize("cfg", SMALL, ids=lambda c: f"{c['kind']}-L{c['light_kind']}-s{c['seed']}")
def test_small_scene_parity(cuda_device, cfg):
    s = scenes.small(cfg["seed"], n=40, image=96, m=20, kind=cfg["kind"], light_kind=cfg["light_kind"])
    img, m, t, _ = gpu_render(s)
    o = Oracle(s)
    om, ons = o.light_march()
    assert np.array_equal(m, om), f"map mismatch: max {np.max(np.abs(m - om))}"
    oimg, olit = o.view_march(om)
    err = np.abs(img - oimg)
    same = np.mean(np.all(img == oimg, axis=-1))
    assert err.max() <= TOL, f"max |d| {err.max()}"
    assert same > 0.999, f"only {same:.4f} of pixels bit-identical"
    assert t["lit_samples"] == olit
    assert 0 < t["light_samples"] <= ons  # the device stops a ray once o == 1 exactly
    i64, _ = o.view_march(o.light_march(fp64=True)[0], fp64=True)
    print(f"{s.name}: max|d| vs f32 oracle {err.max():.2e}, identical {same:.5f}, "
          f"PSNR vs f64 {psnr(img, i64):.1f} dB")


@pytest.mark.parametrize("n", [24, 129, 257, 513, 1025])
def test_markstein_division_matches_ieee(cuda_device, n):
    """The kernels' parametric-coordinate division equals IEEE division for every
    cell width of the counting coordinates (0, 1/(n-1)) and 2^16 numerators each."""
    checked, bad = B.selftest_division(0.0, 1.0 / (n - 1), n - 1, 1 << 16)
    assert checked == (n - 1) << 16 and bad == 0
    # map axes: spacing = extent / M
    for m in (16, 128, 256, 512):
        checked, bad = B.selftest_division(0.0, 1.0 / m, m, 1 << 14)
        assert bad == 0


def test_slab_fp32_reference_mode(cuda_device):
    s = scenes.small(4, n=32, image=80, m=16, kind="blobs")
    s.slab_fp64 = False
    img, m, _, _ = gpu_render(s)
    oimg, _ = Oracle(s).view_march(m)
    assert np.max(np.abs(img - oimg)) <= TOL
    assert np.mean(np.all(img == oimg, axis=-1)) > 0.999


def test_no_shadow_map(cuda_device):
    """Unlit point field (use_map off); cell fields are in test_cells_gpu.py."""
    s = scenes.small(5, n=32, image=64, m=8)
    s.use_map = False
    img, _, t, r = gpu_render(s)
    oimg, lit = Oracle(s).view_march(None)
    assert np.max(np.abs(img - oimg)) <= TOL and t["map_vertices"] == 0 and t["lit_samples"] == lit


def test_config0_parity(cuda_device):
    """The 128^3 blob workload (config 0) at full size: 512^2, M = 128, directional light."""
    s = scenes.config0()
    img, m, t, _ = gpu_render(s)
    o = Oracle(s)
    om, _ = o.light_march()
    assert np.array_equal(m, om)
    oimg, olit = o.view_march(om)
    err = np.abs(img - oimg)
    assert err.max() <= TOL
    assert abs(t["lit_samples"] - olit) <= 1e-4 * olit
    i64, _ = o.view_march(o.light_march(fp64=True)[0], fp64=True)
    p = psnr(img, i64)
    print(f"config0: max|d| f32 {err.max():.2e}; vs f64 max {np.abs(img - i64).max():.2e} PSNR {p:.1f} dB; "
          f"lit {t['lit_samples']} map {t['map_build_ms']:.2f} ms view {t['view_march_ms']:.2f} ms")
    assert p > 40


def test_config1_full_size_properties(cuda_device):
    """The 512^3 noise workload (config 1: 1024^2, M = 256): properties at full size
    plus oracle parity on a random vertex subset and an image crop."""
    import torch
    s = scenes.config1()
    fd = s.field_device()
    r = B.Renderer(0)
    r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    img, t = r.render(s.camera())
    img2, _ = r.render(s.camera())
    assert np.array_equal(img, img2), "render is not deterministic"
    a = img[..., 3]
    assert a.min() >= 0 and a.max() < s.cutoff + 0.6 + 1e-6
    assert np.all(img[..., :3] <= a[..., None] + 1e-6)  # premultiplied, rgb <= 1
    assert t["rays_hit"] == s.width * s.height and t["lit_samples"] > 0
    pd = s.map_m + 1
    m = r.get_shadow_map(pd ** 3)
    assert 0 <= m.min() and m.max() <= 1
    field = fd.cpu().numpy()
    del fd
    torch.cuda.empty_cache()
    o = Oracle(s, field=field)
    ids = np.random.default_rng(7).choice(pd ** 3, 4096, replace=False)
    om, _ = o.light_march_ids(ids)
    assert np.array_equal(m[ids], om), "map vertex subset differs from the oracle"
    win = (480, 480, 48, 48)
    oc, _ = o.view_march(m.reshape((pd,) * 3), window=win)
    crop = img[480:528, 480:528]
    assert np.max(np.abs(crop - oc)) <= TOL
    print(f"config1: lit {t['lit_samples']} light {t['light_samples']} map {t['map_build_ms']:.2f} ms "
          f"view {t['view_march_ms']:.2f} ms")


def test_reuse_map_and_device_io(cuda_device):
    import torch
    s = scenes.small(6, n=32, image=64, m=16)
    r = B.Renderer(0)
    fd = torch.from_numpy(s.field_numpy()).cuda()
    r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    r.set_reuse_shadow_map(True)
    out = torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda")
    _, t1 = r.render(s.camera(), out=out)
    _, t2 = r.render(s.camera(), out=out)
    assert t1["map_vertices"] == 17 ** 3 and t2["map_vertices"] == 0
    host, _ = gpu_render(s)[:2]
    assert np.array_equal(out.cpu().numpy(), host)
    r.add_point_light((9, 9, 9))  # only the first light shades: the key is unchanged
    _, t3 = r.render(s.camera(), out=out)
    assert t3["map_vertices"] == 0
    r.clear_lights()
    r.add_point_light((9, 9, 9))
    _, t4 = r.render(s.camera(), out=out)
    assert t4["map_vertices"] == 17 ** 3


def test_error_paths(cuda_device):
    r = B.Renderer(0)
    cam = B.Renderer.camera((0.5, 0.5, 2), (0.5, 0.5, 0.5), (0, 1, 0), 30, 8, 8)
    with pytest.raises(B.BeamsError) as e:
        r.render(cam)
    assert e.value.status == 8  # STATE: no volume
    with pytest.raises(B.BeamsError) as e:
        r.set_sample_distance(0.0)
    assert e.value.status == 1 and "positive" in str(e.value)
    with pytest.raises(B.BeamsError):
        r.set_color_map(np.full((4, 4), np.nan, np.float32))
    with pytest.raises(B.BeamsError):
        r.set_shadow_map_size(0)
    s = scenes.small(0, n=16, image=8, m=4)
    r.set_volume(s.field_numpy(), spacing=s.spacing)
    r.set_color_map(s.tf)
    with pytest.raises(B.BeamsError) as e:
        r.render(cam)  # shadow map on, no light
    assert e.value.status == 8
    r.add_point_light((3, 3, 3))
    bad = B.Renderer.camera((0.5, 0.5, 2), (0.5, 0.5, 0.5), (0, 1, 0), 200, 8, 8)
    with pytest.raises(B.BeamsError):
        r.render(bad)
    img, _ = r.render(cam)
    assert np.isfinite(img).all()


def test_mapper_mirror(cuda_device):
    s = scenes.small(8, n=24, image=32, m=8)
    mapper = B.MapperLightedVolume(0)
    mapper.SetCanvas(s.width, s.height)
    mapper.SetShadowMapSize(s.map_m)
    mapper.SetUseShadowMap(True)
    mapper.AddLight(s.light)
    mapper.SetActiveColorTable(s.tf)
    mapper.SetSampleDistance(s.sample_distance)
    img = mapper.RenderCells(s.field_numpy(), s.origin, s.spacing, s.value_range,
                             dict(position=s.cam_pos, look_at=s.cam_look, up=s.cam_up, fov_y_deg=s.fov_y_deg))
    assert s.cutoff == 1.0  # the mapper keeps the reference's alpha >= 1 break
    ref, _ = Oracle(s).view_march(None)
    assert np.max(np.abs(img - ref)) <= TOL


@pytest.mark.parametrize("kind", ["blobs", "noise"])
def test_vertex_order_and_empty_skip_change_nothing(cuda_device, kind):
    """The map build's vertex order (rows or bricks) and its skipping of empty
    macro-cells are launch choices: map, image and sample counts stay identical."""
    s = scenes.small(71, n=40, image=48, m=20, kind=kind, light_kind=0)
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    ref = None
    for lb in (0, 8, 16, 32, 64):
        for skip in (False, True):
            r.set_tuning(light_brick=lb, empty_skip=skip, view_skip=skip)
            assert r.get_tuning() == {"light_brick": lb, "empty_skip": skip, "view_skip": skip}
            img, t = r.render(s.camera())
            m = r.get_shadow_map((s.map_m + 1) ** 3)
            cur = (m, img, t["light_samples"], t["lit_samples"])
            if ref is None:
                ref = cur
                om, _ = Oracle(s).light_march()
                assert np.array_equal(m, om.ravel())
            assert np.array_equal(cur[0], ref[0]) and np.array_equal(cur[1], ref[1]), (lb, skip)
            assert cur[2:] == ref[2:], (lb, skip, cur[2:], ref[2:])
    with pytest.raises(B.BeamsError):
        r.set_tuning(light_brick=12)
    best = r.autotune(s.camera())
    assert best["light_brick"] in (0, 8, 16, 32, 64) and best["map_ms"] > 0 and best["view_ms"] > 0
    img, _ = r.render(s.camera())
    assert np.array_equal(img, ref[1])


def test_async_host_output_and_double_buffered_renderers(cuda_device):
    """BEAMS_OUT_HOST_ASYNC: the image lands in pinned host memory after
    beams_synchronize; two renderers on two streams, uploading the field from
    pinned memory in turn, give the synchronous image every step."""
    import torch
    s = scenes.small(8, n=40, image=64, m=16)
    ref, _, _, _ = gpu_render(s)
    field = torch.from_numpy(s.field_numpy()).pin_memory()
    rs = []
    for _ in range(2):
        r = B.Renderer(0, stream=torch.cuda.Stream().cuda_stream)
        r.set_volume(field.numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        rs.append(r)
    outs = [torch.full((s.height, s.width, 4), -1.0).pin_memory() for _ in rs]
    for i in range(6):
        q = rs[i % 2]
        if i >= 2:
            q.synchronize()
            assert np.array_equal(outs[i % 2].numpy(), ref)
        q.set_volume(field, dims=s.dims, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        q.render(s.camera(), out=outs[i % 2], timings=False, host_async=True)
    for q in rs:
        q.synchronize()
    for o in outs:
        assert np.array_equal(o.numpy(), ref)
    with pytest.raises(ValueError):
        rs[0].render(s.camera(), out=np.zeros((s.height, s.width, 4), np.float32), host_async=True)


@pytest.mark.parametrize("offset,scale", [((1000.0, -500.0, 250.0), 1.0), ((3.0, 2.0, -1.0), 40.0),
                                          ((-20000.0, 0.0, 7.0), 0.5)])
def test_far_and_scaled_volumes_bit_exact(cuda_device, offset, scale):
    """Volumes far from the origin or at other scales: the float32 rounding of
    the sample positions grows with the coordinates, so this exercises the
    light march's bound on the steps that cannot fail its distance test (the
    map must still equal the oracle's bit for bit)."""
    s = scenes.small(12, n=32, image=48, m=12, kind="noise")
    off = np.asarray(offset)
    sp = scale / (s.dims[0] - 1)
    s.origin = tuple(float(v) for v in off)
    s.brick_spacing = (sp, sp, sp)
    s.light = tuple(float(v) for v in off + scale * (np.asarray(s.light)))
    s.cam_pos = tuple(float(v) for v in off + scale * np.asarray(s.cam_pos))
    s.cam_look = tuple(float(v) for v in off + scale * np.asarray(s.cam_look))
    s.sample_distance = 0.5 * sp
    img, m, t, _ = gpu_render(s)
    o = Oracle(s)
    om, _ = o.light_march()
    assert np.array_equal(m, om), f"map mismatch: max {np.max(np.abs(m - om))}"
    oimg, olit = o.view_march(om)
    assert np.max(np.abs(img - oimg)) <= TOL
    assert t["lit_samples"] == olit


@pytest.mark.parametrize("light_kind", [0, 1])
def test_non_cubic_volume_odd_image(cuda_device, light_kind):
    """Different point counts per axis (so different spacings and brick counts
    per axis of the light-aligned order) and an image whose sides are not
    multiples of the 8x4 warp tile."""
    import dataclasses
    s = scenes.small(14, n=24, image=32, m=11, kind="noise", light_kind=light_kind)
    s = dataclasses.replace(s, dims=(33, 21, 40), width=37, height=29, array=None)
    img, m, t, _ = gpu_render(s)
    o = Oracle(s)
    om, _ = o.light_march()
    assert np.array_equal(m, om), f"map mismatch: max {np.max(np.abs(m - om))}"
    oimg, olit = o.view_march(om)
    assert img.shape == (29, 37, 4)
    assert np.max(np.abs(img - oimg)) <= TOL
    assert np.mean(np.all(img == oimg, axis=-1)) > 0.999
    assert t["lit_samples"] == olit


def test_non_cubic_map(cuda_device):
    """A map with a different cell count per axis (beams_set_shadow_map_size(mx,
    my, mz)) over a non-cubic volume: vertex bricks, pencils and map tables all
    differ per axis."""
    import dataclasses
    s = scenes.small(15, n=24, image=40, m=8, kind="blobs")
    s = dataclasses.replace(s, dims=(30, 26, 35), map_m=(11, 7, 14), array=None)
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    img, t = r.render(s.camera())
    m = r.get_shadow_map(12 * 8 * 15).reshape(15, 8, 12)
    o = Oracle(s)
    om, _ = o.light_march()
    assert om.shape == (15, 8, 12)
    assert np.array_equal(m, om), f"map mismatch: max {np.max(np.abs(m - om))}"
    oimg, olit = o.view_march(om)
    assert np.max(np.abs(img - oimg)) <= TOL
    assert np.mean(np.all(img == oimg, axis=-1)) > 0.999
    assert t["lit_samples"] == olit


def test_density_scale_is_stored_and_changes_nothing(cuda_device):
    """SetDensityScale (MapperLightedVolume.cxx:86-89) stores a value nothing reads."""
    s = scenes.small(6, n=24, image=40, m=8)
    img, _, _, r = gpu_render(s)
    r.set_density_scale(3.5)
    assert r.get_density_scale() == 3.5
    img2, _ = r.render(s.camera())
    assert np.array_equal(img, img2)
    r.close()
