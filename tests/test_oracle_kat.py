"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests or golden data, so these closed forms pin the
reference behaviours the oracle restates:
  * light march advances before it samples, composites o += (1-o)a with
    a = TF alpha / max alpha (TransmittanceMap.h:299-331);
  * view march premultiplies c.a by (1 - C.a) and accumulates C.a += c.a
    (LightedVolumeRenderer.cxx:464-481), so a constant field gives
    C.a = 1 - (1-a)^k after k samples;
  * the slab test returns the analytic entry/exit (LightedVolumeRenderer.cxx:644-718);
  * the TF index truncates (LightedVolumeRenderer.cxx:453-454);
  * the cell-field march (LightedVolumeRenderer.cxx:501-642) composites one
    clamped TF entry per cell, breaks right after the composite that reaches
    the cut-off and clamps the result to 1.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, composite, psnr
from pilot_b200 import scenes


def const_scene(value=0.45, n=16, m=8, light=(0.013, 0.021, 1.0), image=16, cutoff=1e9, use_map=True):
    s = scenes.small(0, n=n, image=image, m=m, light_kind=1, cutoff=1.0)
    s.light = light
    s.cutoff = cutoff
    s.use_map = use_map
    s.array = np.full((n, n, n), value, np.float32)
    return s


def tf_alpha(s, value):
    idx = int(np.float32(value) * np.float32(s.tf.shape[0] - 1))
    return float(s.tf[idx, 3]), float(s.tf[:, 3].max())


def test_light_march_constant_field_closed_form():
    s = const_scene()
    o = Oracle(s)
    m, ns = o.light_march(fp64=True)
    a, amax = tf_alpha(s, 0.45)
    an = a / amax
    assert ns > 0
    # every vertex value is 1 - (1 - a/maxa)^k for an integer k >= 0
    k = np.log1p(-m) / np.log1p(-an)
    assert np.allclose(k, np.round(k), atol=1e-6), "map values are not whole powers of (1 - a)"
    # nearly +z light: k grows with z (samples from the entry face to the vertex)
    kz = np.round(k).mean(axis=(1, 2))
    assert np.all(np.diff(kz) >= 0) and kz[-1] > kz[0]
    # advance-then-sample: a vertex at depth z gets floor(z/step)+1 samples while the
    # next position is still inside (z axis, light along +z)
    ext = np.sqrt(3.0)
    step = ext / 128
    z = np.arange(s.map_m + 1) / s.map_m
    expect = np.minimum(np.floor(z / step) + 1, np.floor(1.0 / step))
    interior = np.round(k)[:, s.map_m // 2, s.map_m // 2]
    assert np.max(np.abs(interior - expect)) <= 1


def test_view_march_constant_field_alpha_is_whole_power():
    s = const_scene(use_map=False, image=12)
    o = Oracle(s)
    img, lit = o.view_march(None, fp64=True)
    a, _ = tf_alpha(s, 0.45)
    alpha = img[..., 3]
    assert lit > 0 and np.all(alpha > 0)
    k = np.log1p(-alpha) / np.log1p(-a)
    assert np.allclose(k, np.round(k), atol=1e-6)
    # premultiplied colour: rgb = tf_rgb * alpha with no shadowing
    idx = int(np.float32(0.45) * np.float32(255))
    assert np.allclose(img[..., :3], s.tf[idx, :3][None, None, :] * alpha[..., None], atol=1e-9)


def test_empty_transfer_function_renders_nothing():
    s = scenes.small(1, n=16, image=16, m=6)
    s.tf = s.tf.copy()
    s.tf[:, 3] = 0
    o = Oracle(s)
    m, _ = o.light_march()
    img, _ = o.view_march(m)
    assert np.all(m == 0)
    assert np.all(img == 0)


def test_slab_analytic_entry_exit():
    s = scenes.small(0, n=16, image=9, m=4)
    s.cam_pos, s.cam_look, s.cam_up = (0.5, 0.5, 2.0), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0)
    for fp64 in (True, False):
        s.slab_fp64 = fp64
        o = Oracle(s)
        r = o.ray_setup(4, 4)  # centre pixel of a 9x9 image looks straight down -z
        assert np.allclose(r[3:6], [0, 0, -1], atol=1e-7)
        assert abs(r[6] - 1.0) < 1e-6 and abs(r[7] - 2.0) < 1e-6
    # a ray that misses the box is flagged with t_enter = -1
    s.cam_look = (5.0, 5.0, 2.0 - 1e-3)
    s.cam_up = (0.0, 0.0, 1.0)
    o = Oracle(s)
    assert o.ray_setup(4, 4)[6] == -1.0


def test_single_opaque_block_casts_shadow_column():
    n, m = 24, 12
    f = np.zeros((n, n, n), np.float32)
    f[8:16, 8:16, 8:16] = 1.0  # opaque cube in the middle
    s = scenes.small(0, n=n, image=16, m=m, light_kind=1)
    s.light = (0.0, 0.0, 1.0)  # light travels along +z
    s.array = f
    o = Oracle(s)
    mp, _ = o.light_march(fp64=True)
    c = m // 2
    assert mp[m, c, c] > 0.99          # behind the block (far z face) is dark
    assert mp[0, c, c] == 0.0          # the entry face sees the light
    assert mp[m, 0, 0] < 1e-6          # outside the shadow column
    assert mp[m, c, 1] < mp[m, c, c]


def test_truncating_tf_index():
    # 0.7 * 255 = 178.5 -> index 178 (truncation, not rounding)
    s = const_scene(value=0.7, use_map=False, image=4)
    tf = np.zeros_like(s.tf)
    tf[178] = (1, 0, 0, 0.5)
    tf[179] = (0, 1, 0, 0.5)
    s.tf = tf
    img, _ = Oracle(s).view_march(None, fp64=True)
    assert np.all(img[..., 0] > 0) and np.all(img[..., 1] == 0)


def test_fp32_mode_tracks_fp64():
    s = scenes.small(2, n=24, image=40, m=12)
    o = Oracle(s)
    m32, _ = o.light_march()
    m64, _ = o.light_march(fp64=True)
    assert np.max(np.abs(m32 - m64)) < 1e-3
    i32, l32 = o.view_march(m32)
    i64, l64 = o.view_march(m64, fp64=True)
    assert psnr(i32, i64) > 60
    assert abs(l32 - l64) <= 0.01 * l64


def test_directional_light_matches_far_point_light():
    s = scenes.small(3, n=20, image=8, m=8, light_kind=1)
    d = np.array(s.light) / np.linalg.norm(s.light)
    mdir, _ = Oracle(s).light_march(fp64=True)
    far = np.array([0.5, 0.5, 0.5]) - d * 1e4 * np.sqrt(3)
    s.light_kind, s.light = 0, tuple(far)
    mpt, _ = Oracle(s).light_march(fp64=True)
    # sample positions differ (per-vertex origin vs one far origin): compare loosely
    assert np.mean(np.abs(mdir - mpt)) < 0.02


def test_composite_over_order():
    a = np.array([[[0.5, 0, 0, 0.5]]], np.float32)
    b = np.array([[[0, 0.8, 0, 0.8]]], np.float32)
    out = composite(np.stack([a, b]), [0, 1])
    assert np.allclose(out[0, 0], [0.5, 0.4, 0, 0.9])
    out2 = composite(np.stack([a, b]), [1, 0])
    assert np.allclose(out2[0, 0], [0.1, 0.8, 0, 0.9])


def test_oracle_rejects_bad_scene():
    s = scenes.small(0, n=16, image=8, m=4)
    s.light_steps = 0
    with pytest.raises(RuntimeError):
        Oracle(s).light_march()


def _light_color(s):
    return np.float32(s.light_color) * np.float32(s.light_intensity)


def test_multi_light_with_dark_second_light_equals_single_light():
    """Multi-light extension: a second light of colour 0 adds exact zeros, so the
    image equals the first-light-only image bit for bit."""
    s = scenes.small(6, n=24, image=32, m=12)
    o = Oracle(s)
    m0, _ = o.light_march()
    single, lit1 = o.view_march(m0)
    lc = np.stack([_light_color(s), np.zeros(3, np.float32)])
    multi, lit2 = o.view_march_multi(np.stack([m0, np.ones_like(m0)]), lc)
    assert np.array_equal(single, multi) and lit1 == lit2


def test_multi_light_two_half_lights_equal_one_full_light():
    """Halving a light's intensity scales every term by 2^-1 exactly, so two
    identical half-intensity lights sum to the full-intensity shading bit for bit."""
    s = scenes.small(7, n=24, image=32, m=12, light_kind=1)
    o = Oracle(s)
    m0, _ = o.light_march()
    single, _ = o.view_march(m0)
    half = _light_color(s) * np.float32(0.5)
    multi, _ = o.view_march_multi(np.stack([m0, m0]), np.stack([half, half]))
    assert np.array_equal(single, multi)


def test_multi_light_oracle_rejects_mismatched_inputs():
    s = scenes.small(0, n=16, image=8, m=4)
    m0, _ = Oracle(s).light_march()
    with pytest.raises(ValueError):
        Oracle(s).view_march_multi(np.stack([m0, m0]), np.ones((3, 3), np.float32))


def _camera_ray_lengths(s):
    """|forward + sx right + sy up| per pixel centre, from the camera alone (float64)."""
    p, l, u = (np.asarray(v, np.float64) for v in (s.cam_pos, s.cam_look, s.cam_up))
    f = (l - p) / np.linalg.norm(l - p)
    r = np.cross(f, u)
    r /= np.linalg.norm(r)
    up = np.cross(r, f)
    th = np.tan(np.radians(s.fov_y_deg) / 2)
    aspect = s.width / s.height
    sx = ((np.arange(s.width) + 0.5) * (2 * th * aspect / s.width) - th * aspect)[None, :]
    sy = ((np.arange(s.height) + 0.5) * (2 * th / s.height) - th)[:, None]
    v = f[None, None, :] + sx[..., None] * r[None, None, :] + sy[..., None] * up[None, None, :]
    return np.linalg.norm(v, axis=-1)


def test_window_depth_of_a_view_plane_unprojects_to_its_distance():
    """A plane at view depth t0 has window depth ((f+n) - 2fn/t0)/(f-n) mapped to
    [0, 1]; unprojected, each pixel's limit is t0 times its ray's length."""
    s = scenes.small(0, n=16, image=24, m=4)
    n, f, t0 = 0.1, 10.0, 1.3
    z = ((f + n) - 2 * f * n / t0) / (f - n)
    depth = np.full((s.height, s.width), (z + 1) / 2, np.float32)
    got = Oracle(s).window_depth_to_distance(depth, n, f)
    want = t0 * _camera_ray_lengths(s)
    assert np.max(np.abs(got - want) / want) < 1e-5  # depth was rounded to float32
    # d = 1 is the far plane, d = 0 the near plane, NaN reads as 1
    depth[0, 0], depth[0, 1], depth[0, 2] = 1.0, 0.0, np.nan
    got = Oracle(s).window_depth_to_distance(depth, n, f)
    L = _camera_ray_lengths(s)[0]
    assert np.allclose(got[0, :3], [f * L[0], n * L[1], f * L[2]], rtol=1e-12)


def test_ray_limits_clip_the_view_march():
    s = scenes.small(2, n=24, image=32, m=8)
    o = Oracle(s)
    m, _ = o.light_march()
    full, lit_full = o.view_march(m)
    o.set_ray_limits(np.full((s.height, s.width), np.inf, np.float32))
    same, lit_same = o.view_march(m)
    assert np.array_equal(full, same) and lit_full == lit_same
    o.set_ray_limits(np.zeros((s.height, s.width), np.float32))  # every ray ends at the camera
    none, lit_none = o.view_march(m)
    assert not none.any() and lit_none == 0
    # a limit half-way through the volume composites a prefix of each ray's samples
    cam_to_centre = np.linalg.norm(np.asarray(s.cam_pos) - 0.5)
    o.set_ray_limits(np.full((s.height, s.width), cam_to_centre, np.float32))
    half, lit_half = o.view_march(m)
    assert 0 < lit_half < lit_full
    assert np.all(half[..., 3] <= full[..., 3] + 1e-6)


def test_background_blend_is_over():
    from oracle.oracle import blend_background
    img = np.array([[[0, 0, 0, 0], [0.2, 0.1, 0.0, 0.5], [0.3, 0.3, 0.3, 1.0]]], np.float32)
    out = blend_background(img, (1.0, 0.5, 0.25, 0.8))
    assert np.allclose(out[0, 0], [0.8, 0.4, 0.2, 0.8])
    assert np.allclose(out[0, 1], [0.2 + 0.4, 0.1 + 0.2, 0.1, 0.5 + 0.4])
    assert np.array_equal(out[0, 2], img[0, 2])


def test_explicit_uniform_coordinates_equal_generated_ones():
    """Explicit coordinates equal to the generated float32 origin + spacing * i
    give the same map and image as the generated (counting) coordinates."""
    s = scenes.small(9, n=24, image=32, m=10)
    base_m, _ = Oracle(s).light_march()
    base_i, base_lit = Oracle(s).view_march(base_m)
    h = np.float32(s.spacing[0])
    c = np.float32(s.origin[0]) + h * np.arange(s.dims[0], dtype=np.float32)
    s.coords = (c, c.copy(), c.copy())
    m, _ = Oracle(s).light_march()
    i, lit = Oracle(s).view_march(m)
    assert np.array_equal(m, base_m) and np.array_equal(i, base_i) and lit == base_lit


def test_stretched_coordinates_move_the_samples():
    s = scenes.small(9, n=24, image=32, m=10)
    base_m, _ = Oracle(s).light_march()
    t = np.linspace(0, 1, s.dims[0])
    s.coords = tuple(np.float32(t ** p) for p in (1.4, 1.0, 0.8))
    m, _ = Oracle(s).light_march()
    assert not np.array_equal(m, base_m)
    assert np.all((m >= 0) & (m <= 1))


def test_cell_field_constant_closed_form():
    """SamplerCellAssoc (LightedVolumeRenderer.cxx:501-642) on a constant cell
    field: every sample composites the same TF entry, so C.a = 1 - (1 - A)^k
    and rgb = tf_rgb * C.a after k samples, with k equal to the composites
    counted, and the clamped index takes the first / last entry for values
    below / above the range."""
    s = const_scene(use_map=False, image=12)
    n = s.dims[0]
    for value, idx in ((0.45, int(np.float32(0.45) * np.float32(255))), (-3.0, 0), (7.5, 255)):
        cells = np.full((n - 1, n - 1, n - 1), value, np.float32)
        o = Oracle(s, field=cells)
        img, lit = o.view_march_cells(fp64=True)
        A = float(s.tf[idx, 3])
        alpha = img[..., 3]
        if A == 0.0:
            assert np.all(img == 0) and lit > 0
            continue
        assert np.allclose(img[..., :3], s.tf[idx, :3][None, None, :] * alpha[..., None], atol=1e-9)
        if A > 0.5:  # (1 - A)^k underflows double precision's distance from 1 within a few dozen samples
            assert np.all(alpha[alpha > 0] > 1 - 1e-9)
            continue
        k = np.log1p(-alpha) / np.log1p(-A)
        assert np.allclose(k, np.round(k), atol=1e-6)
        assert int(np.round(k).sum()) == lit  # one composite per counted sample


def test_cell_field_break_before_update_and_final_clamp():
    """The cell march breaks on C.a >= cutoff right after compositing (no
    further sample), and clamps every channel to 1 at the end: an opaque entry
    (A = 1) stops each ray after exactly one composite."""
    s = const_scene(use_map=False, image=10, cutoff=1.0)
    s.tf = s.tf.copy()
    s.tf[:, 3] = 1.0
    s.tf[:, :3] = 2.0  # colours above 1: the final clamp caps them
    n = s.dims[0]
    cells = np.full((n - 1, n - 1, n - 1), 0.5, np.float32)
    o = Oracle(s, field=cells)
    img, lit = o.view_march_cells()
    hit = img[..., 3] > 0
    assert lit == int(hit.sum())
    assert np.all(img[hit] == 1.0)
