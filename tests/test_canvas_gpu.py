"""The canvas side of the mapper: depth clipping of the camera rays
(MapCanvasToRays -> MaxDistance, MapperLightedVolume.cxx:151-152) and the
background blend (:185-188), against the oracle.

Bars: with per-pixel ray limits the image matches the oracle's march under the
same limits like every exact-form image (max |dRGBA| <= 2e-3, >= 99.9% of pixels
bit-identical); window depths unproject to the oracle's float64 distances within
a relative 1e-4 (float32 arithmetic, near/far ratio 100); a window-depth render
equals the render under the distances it unprojects to, bit for bit; the blended
image equals the oracle's Porter-Duff over of the unblended image, bit for bit.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, blend_background, render_bricks
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def renderer(s):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    return r


def limits(s, seed):
    """Per-pixel limits: no limit, before the volume, and cuts through it."""
    rng = np.random.default_rng(seed)
    c = float(np.linalg.norm(np.asarray(s.cam_pos) - 0.5))
    lim = rng.uniform(c - 0.9, c + 0.9, (s.height, s.width)).astype(np.float32)
    lim[rng.random(lim.shape) < 0.15] = np.inf
    lim[rng.random(lim.shape) < 0.05] = np.nan  # reads as no limit
    return lim


def check(img, oimg):
    err = np.abs(img - oimg)
    same = np.mean(np.all(img == oimg, axis=-1))
    assert err.max() <= TOL, f"max |d| {err.max()}"
    assert same > 0.999, f"only {same:.4f} of pixels bit-identical"


@pytest.mark.parametrize("seed,light_kind,slab64", [(0, 0, True), (3, 1, True), (5, 0, False)])
def test_ray_distance_limits_match_oracle(cuda_device, seed, light_kind, slab64):
    s = scenes.small(seed, n=40, image=96, m=20, kind="noise" if seed % 2 else "blobs", light_kind=light_kind)
    s.slab_fp64 = slab64
    r = renderer(s)
    lim = limits(s, seed)
    r.set_depth_buffer(lim, B.DEPTH_RAY_DISTANCE)
    img, t = r.render(s.camera())
    m = r.get_shadow_map((s.map_m + 1) ** 3)
    o = Oracle(s)
    o.set_ray_limits(np.where(np.isnan(lim), np.inf, lim))
    oimg, olit = o.view_march(m)
    check(img, oimg)
    assert t["lit_samples"] == olit
    # clearing the buffer restores the unclipped image
    r.set_depth_buffer(None)
    full, tf = r.render(s.camera())
    o.set_ray_limits(None)
    ofull, _ = o.view_march(m)
    check(full, ofull)
    assert tf["lit_samples"] > t["lit_samples"]


def test_window_depth_unprojects_like_oracle_and_clips_like_distances(cuda_device):
    s = scenes.small(7, n=40, image=80, m=16)
    r = renderer(s)
    rng = np.random.default_rng(7)
    near, far = 0.05, 5.0
    depth = rng.uniform(0.9, 1.0, (s.height, s.width)).astype(np.float32)
    depth[:4] = 1.0
    depth[4:6] = np.nan
    r.set_depth_buffer(depth, B.DEPTH_WINDOW, near, far)
    cam = s.camera()
    lim = r.get_ray_limits(cam)
    want = Oracle(s).window_depth_to_distance(depth, near, far)
    assert np.max(np.abs(lim - want) / want) < 1e-4
    img, _ = r.render(cam)
    q = renderer(s)
    q.set_depth_buffer(lim, B.DEPTH_RAY_DISTANCE)
    img2, _ = q.render(cam)
    assert np.array_equal(img, img2)


def test_depth_buffer_size_must_match_camera(cuda_device):
    s = scenes.small(1, n=24, image=32, m=8)
    r = renderer(s)
    r.set_depth_buffer(np.ones((16, 16), np.float32), B.DEPTH_RAY_DISTANCE)
    with pytest.raises(B.BeamsError):
        r.render(s.camera())
    with pytest.raises(B.BeamsError):
        r.set_depth_buffer(np.ones((s.height, s.width), np.float32), B.DEPTH_WINDOW, 1.0, 0.5)


@pytest.mark.parametrize("bg", [(1.0, 1.0, 1.0, 1.0), (0.2, 0.5, 0.9, 0.6)])
def test_background_blend_matches_oracle(cuda_device, bg):
    s = scenes.small(2, n=32, image=64, m=12)
    r = renderer(s)
    plain, _ = r.render(s.camera())
    r.set_background(True, bg)
    blended, t = r.render(s.camera())
    assert np.array_equal(blended, blend_background(plain, bg))
    r.set_background(False)
    again, _ = r.render(s.camera())
    assert np.array_equal(again, plain)


def test_bricks_with_depth_limits_and_background(cuda_device):
    s = scenes.small(31, n=41, image=80, m=12, kind="blobs")
    bricks = scenes.split_bricks(s, (2, 2, 2))
    r = B.Renderer(0)
    r.set_bricks([(b.field_numpy(), b.origin, b.spacing, b.value_range) for b in bricks])
    bricks[0].configure(r)
    lim = limits(s, 31)
    r.set_depth_buffer(lim, B.DEPTH_RAY_DISTANCE)
    bg = (0.1, 0.2, 0.3, 1.0)
    r.set_background(True, bg)
    img, _ = r.render(bricks[0].camera())
    orgba, _, _, _, _ = render_bricks(bricks, ray_limits=np.where(np.isnan(lim), np.inf, lim))
    check(img, blend_background(orgba, bg))


def test_depth_limits_in_the_precision_and_learned_forms(cuda_device):
    """The limits apply in every single-volume form: the alpha channel never
    depends on the shading, so under the same limits the precision form's
    alpha matches the oracle's precision mode and the learned form's alpha
    equals the exact form's bit for bit, with equal lit-sample counts."""
    from oracle.oracle import quantize
    s = scenes.small(9, n=40, image=64, m=16, kind="noise")
    lim = limits(s, 9)
    r = renderer(s)
    r.set_depth_buffer(lim, B.DEPTH_RAY_DISTANCE)
    exact, te = r.render(s.camera())
    r.set_form(B.FORM_PRECISION, B.BF16)
    prec, tp = r.render(s.camera())
    m = r.get_shadow_map((s.map_m + 1) ** 3)
    o = Oracle(s, field=quantize(s.field_numpy(), "bf16"), precision=True)
    o.set_ray_limits(np.where(np.isnan(lim), np.inf, lim))
    oimg, olit = o.view_march(m.reshape((s.map_m + 1,) * 3))
    check(prec, oimg)
    assert tp["lit_samples"] == olit
    r.set_form(B.FORM_EXACT)
    r.mlp_train(B.mlp_options(samples_log2=14, n_lights=1, scene_light=1, epochs=1))
    r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.0))
    learned, tl = r.render(s.camera())
    assert np.array_equal(learned[..., 3], exact[..., 3])
    assert tl["lit_samples"] == te["lit_samples"]
