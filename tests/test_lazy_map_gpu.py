"""The exact form's lazy map (beams_set_lazy_shadow_map): a view march without
shading marks the map cells the frame's rays read and the light march builds
only their corners. The reference builds every vertex (TransmittanceMap.h:565-621)
and reads the map only at lit samples (LightedVolumeRenderer.cxx:456-475), whose
set and order do not depend on the map, so the image must equal the full map's
bit for bit.

Each lazy frame follows a frame that left other lights' maps in the map
buffer, so a vertex that the lazy build skips but the view march reads would
change the image.

Bars: lazy image == full-map image (np.array_equal) with equal lit-sample
counts, on uniform and rectilinear fields, point and directional lights, the
multi-light extension, canvas depth limits and both empty-skip settings; fewer
vertices built than (M+1)^3 when the view sees part of the volume; one lazy
image also checked directly against the oracle (max |dRGBA| <= 2e-3, >= 99.9%
bit-identical pixels, the exact form's bar).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def renderer(s, coords=None):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    if coords is not None:
        r.set_volume_coordinates(*coords)
    s.configure(r)
    return r


POISON_LIGHTS = [((0.3, 0.9, -0.3), (1.0, 0.2, 0.2), 1.0), ((-0.8, 0.1, 0.6), (0.2, 1.0, 0.2), 1.0),
                 ((0.1, -0.7, -0.7), (0.2, 0.2, 1.0), 1.0)]


def poison(r, cam, nlights=1):
    """Leaves other directional lights' full maps in the map buffer, so that a
    vertex the lazy build skips but the view march reads changes the image."""
    r.set_lazy_shadow_map(False)
    r.clear_lights()
    for d, c, i in POISON_LIGHTS[:nlights]:
        r.add_directional_light(d, c, i)
    r.render(cam)


def full_and_lazy(r, cam, restore, nlights=1):
    """restore(r) puts back the scene's lights after the poisoning frame."""
    r.set_lazy_shadow_map(False)
    full, tf = r.render(cam)
    poison(r, cam, nlights)
    restore(r)
    r.set_lazy_shadow_map(True)
    lazy, tl = r.render(cam)
    r.set_lazy_shadow_map(False)
    return full, tf, lazy, tl


def assert_same(full, tf, lazy, tl, nvert):
    assert np.array_equal(lazy, full), f"lazy image differs by {np.max(np.abs(lazy - full))}"
    assert tl["lit_samples"] == tf["lit_samples"]
    assert tf["map_vertices"] == nvert
    assert 0 < tl["map_vertices"] <= nvert


CASES = [
    dict(seed=0, kind="blobs", light_kind=0, fov=30.0),
    dict(seed=1, kind="blobs", light_kind=1, fov=30.0),
    dict(seed=2, kind="noise", light_kind=0, fov=9.0),
    dict(seed=3, kind="noise", light_kind=1, fov=6.0),
]


@pytest.mark.parametrize("c", CASES, ids=lambda c: f"{c['kind']}-L{c['light_kind']}-fov{c['fov']:g}")
def test_lazy_map_image_equals_full_map_image(cuda_device, c):
    s = scenes.small(c["seed"], n=40, image=96, m=20, kind=c["kind"], light_kind=c["light_kind"])
    s.fov_y_deg = c["fov"]
    r = renderer(s)
    nv = (s.map_m + 1) ** 3
    full, tf, lazy, tl = full_and_lazy(r, s.camera(), s.configure)
    assert_same(full, tf, lazy, tl, nv)
    if c["fov"] < 10:  # a zoomed view reads part of the volume
        assert tl["map_vertices"] < nv
    print(f"{c}: built {tl['map_vertices']} of {nv} vertices")


def test_lazy_map_image_matches_oracle(cuda_device):
    s = scenes.small(4, n=40, image=96, m=20, kind="noise", light_kind=0)
    s.fov_y_deg = 12.0
    r = renderer(s)
    poison(r, s.camera())
    s.configure(r)
    r.set_lazy_shadow_map(True)
    img, t = r.render(s.camera())
    o = Oracle(s)
    om, _ = o.light_march()
    oimg, olit = o.view_march(om)
    err = np.abs(img - oimg)
    assert err.max() <= TOL, f"max |d| {err.max()}"
    assert np.mean(np.all(img == oimg, axis=-1)) > 0.999
    assert t["lit_samples"] == olit


def test_lazy_map_is_not_readable_or_reused(cuda_device):
    s = scenes.small(5, n=32, image=64, m=16)
    r = renderer(s)
    r.set_reuse_shadow_map(True)
    r.set_lazy_shadow_map(True)
    a, ta = r.render(s.camera())
    with pytest.raises(B.BeamsError):
        r.get_shadow_map((s.map_m + 1) ** 3)
    b, tb = r.render(s.camera())  # rebuilt, never reused
    assert tb["map_vertices"] == ta["map_vertices"] > 0
    assert np.array_equal(a, b)
    r.set_lazy_shadow_map(False)
    c, tc = r.render(s.camera())  # a full map again, readable
    assert np.array_equal(a, c)
    assert tc["map_vertices"] == (s.map_m + 1) ** 3
    assert r.get_shadow_map((s.map_m + 1) ** 3).size == (s.map_m + 1) ** 3


@pytest.mark.parametrize("skip", [True, False])
def test_lazy_map_with_and_without_empty_skip(cuda_device, skip):
    s = scenes.small(6, n=48, image=80, m=24, kind="blobs", light_kind=0)
    s.fov_y_deg = 14.0
    r = renderer(s)
    r.set_tuning(light_brick=8, empty_skip=skip, view_skip=skip)
    full, tf, lazy, tl = full_and_lazy(r, s.camera(), s.configure)
    assert_same(full, tf, lazy, tl, (s.map_m + 1) ** 3)


@pytest.mark.parametrize("brick", [0, 16, 32])
def test_lazy_map_under_every_vertex_order(cuda_device, brick):
    """The vertex list follows the light march's order: rows, or cubic bricks."""
    s = scenes.small(8, n=56, image=96, m=40, kind="noise", light_kind=0)
    s.fov_y_deg = 11.0
    r = renderer(s)
    r.set_tuning(light_brick=brick, empty_skip=False, view_skip=False)
    full, tf, lazy, tl = full_and_lazy(r, s.camera(), s.configure)
    assert_same(full, tf, lazy, tl, (s.map_m + 1) ** 3)
    assert tl["map_vertices"] < (s.map_m + 1) ** 3


def test_lazy_map_rectilinear(cuda_device):
    s = scenes.small(21, n=40, image=80, m=16, kind="noise", light_kind=1)
    rng = np.random.default_rng(21)
    coords = []
    for _ in range(3):
        w = rng.uniform(0.4, 1.6, s.dims[0] - 1)
        cc = np.concatenate([[0.0], np.cumsum(w)])
        coords.append(np.float32(cc / cc[-1]))
    s.fov_y_deg = 10.0
    r = renderer(s, coords)
    full, tf, lazy, tl = full_and_lazy(r, s.camera(), s.configure)
    assert_same(full, tf, lazy, tl, (s.map_m + 1) ** 3)


def test_lazy_map_multi_light(cuda_device):
    s = scenes.small(2, n=40, image=96, m=20, kind="noise")
    s.fov_y_deg = 12.0
    r = renderer(s)

    def lights(q):
        s.configure(q)
        q.add_point_light((1.6, 0.2, -0.4), (0.9, 0.5, 0.2), 0.8)
        q.add_directional_light((-0.3, -1.0, 0.2), (0.2, 0.4, 1.0), 0.6)

    lights(r)
    r.set_multi_light(True)
    nv = (s.map_m + 1) ** 3
    full, tf, lazy, tl = full_and_lazy(r, s.camera(), lights, nlights=3)
    assert np.array_equal(lazy, full)
    assert tl["lit_samples"] == tf["lit_samples"]
    assert tf["map_vertices"] == 3 * nv
    assert 0 < tl["map_vertices"] < 3 * nv and tl["map_vertices"] % 3 == 0


def test_lazy_map_with_depth_limits(cuda_device):
    s = scenes.small(3, n=40, image=96, m=20, kind="noise", light_kind=1)
    r = renderer(s)
    rng = np.random.default_rng(3)
    c = float(np.linalg.norm(np.asarray(s.cam_pos) - 0.5))
    lim = rng.uniform(c - 0.6, c, (s.height, s.width)).astype(np.float32)  # most rays end inside
    lim[rng.random(lim.shape) < 0.1] = np.inf
    r.set_lazy_shadow_map(True)
    _, t_nolim = r.render(s.camera())
    r.set_depth_buffer(lim, B.DEPTH_RAY_DISTANCE)
    full, tf, lazy, tl = full_and_lazy(r, s.camera(), s.configure)
    assert_same(full, tf, lazy, tl, (s.map_m + 1) ** 3)
    assert tl["map_vertices"] < t_nolim["map_vertices"]  # clipped rays read fewer cells


@pytest.mark.parametrize("dt,skip", [(B.BF16, False), (B.F16, True)])
def test_lazy_map_in_the_precision_form(cuda_device, dt, skip):
    """The precision form marks over its 16-bit field and builds its binary16
    map over the list: the same image as its full map, after a frame that left
    another light's map in the buffer, and straight after an exact-form frame
    (the buffer then held a float32 map, whose bits read as binary16 can be
    NaN: the masked build clears it)."""
    s = scenes.small(7, n=48, image=80, m=24, kind="noise", light_kind=0)
    s.fov_y_deg = 12.0
    r = renderer(s)
    r.set_tuning(light_brick=8, empty_skip=skip, view_skip=skip)
    r.render(s.camera())  # exact form: a float32 map in the buffer
    r.set_form(B.FORM_PRECISION, field_dtype=dt)
    full, tf = r.render(s.camera())
    poison(r, s.camera())
    s.configure(r)
    r.set_lazy_shadow_map(True)
    lazy, tl = r.render(s.camera())
    assert np.array_equal(lazy, full), f"differs by {np.max(np.abs(lazy - full))}"
    assert tl["lit_samples"] == tf["lit_samples"]
    assert 0 < tl["map_vertices"] < tf["map_vertices"] == (s.map_m + 1) ** 3
    with pytest.raises(B.BeamsError):
        r.get_shadow_map((s.map_m + 1) ** 3)
    r.set_lazy_shadow_map(False)
    again, _ = r.render(s.camera())
    assert np.array_equal(again, full)
    assert r.get_shadow_map((s.map_m + 1) ** 3).size == (s.map_m + 1) ** 3
    # straight from an exact-form frame (a float32 map) to a lazy precision frame
    q = renderer(s)
    q.set_tuning(light_brick=8, empty_skip=skip, view_skip=skip)
    q.render(s.camera())
    q.set_form(B.FORM_PRECISION, field_dtype=dt)
    q.set_lazy_shadow_map(True)
    direct, _ = q.render(s.camera())
    assert np.array_equal(direct, full), f"differs by {np.max(np.abs(direct - full))}"


def test_kept_marks_follow_every_view_input(cuda_device):
    """Mode 2 keeps the marked cells across frames while the view's inputs are
    unchanged: a moving light re-marks nothing (one launch fewer) and matches
    the full map; a change of camera, colour map, canvas depth, sample distance,
    termination alpha or volume marks again."""
    s = scenes.small(9, n=40, image=96, m=20, kind="noise", light_kind=1)
    s.fov_y_deg = 14.0
    r = renderer(s)
    q = renderer(s)  # full maps, same settings
    for x in (r, q):  # fixed launch choices; layouts built before counting launches
        x.set_tuning(light_brick=8, empty_skip=False, view_skip=False)
        x.render(s.camera())

    def both(cam):
        r.set_lazy_shadow_map(True, keep_marks=True)
        a, ta = r.render(cam)
        b, tb = q.render(cam)
        assert np.array_equal(a, b), f"kept-mark frame differs by {np.max(np.abs(a - b))}"
        assert ta["lit_samples"] == tb["lit_samples"]
        return ta

    cam = s.camera()
    t0 = both(cam)
    t1 = both(cam)
    assert t1["kernel_launches"] == t0["kernel_launches"] - 1  # marks kept
    for i, d in enumerate([(0.2, 0.9, 0.3), (-0.7, 0.1, 0.7), (0.5, -0.5, -0.7)]):  # a light orbit
        for x in (r, q):
            x.clear_lights()
            x.add_directional_light(d, (1.0, 0.9, 0.8), 1.2)
        t = both(cam)
        assert t["kernel_launches"] == t1["kernel_launches"]
    # each view input marks again
    s2 = scenes.small(9, n=40, image=96, m=20, kind="noise", light_kind=1)
    s2.fov_y_deg = 9.0
    t = both(s2.camera())
    assert t["kernel_launches"] == t0["kernel_launches"]
    t = both(cam)
    assert t["kernel_launches"] == t0["kernel_launches"]
    tf = np.array(s.tf, np.float32).copy()
    tf[:, 3] = np.clip(tf[:, 3] * 1.7, 0, 1)
    for x in (r, q):
        x.set_color_map(tf)
    assert both(cam)["kernel_launches"] == t0["kernel_launches"]
    for x in (r, q):
        x.set_sample_distance(0.7 / 39)
    assert both(cam)["kernel_launches"] == t0["kernel_launches"]
    for x in (r, q):
        x.set_termination_alpha(0.9)
    assert both(cam)["kernel_launches"] == t0["kernel_launches"]
    c = float(np.linalg.norm(np.asarray(s.cam_pos) - 0.5))
    lim = np.random.default_rng(9).uniform(c - 0.5, c + 0.3, (s.height, s.width)).astype(np.float32)
    for x in (r, q):
        x.set_depth_buffer(lim, B.DEPTH_RAY_DISTANCE)
    t = both(cam)
    assert t["kernel_launches"] == t0["kernel_launches"] + 1  # the ray-limit kernel
    assert both(cam)["kernel_launches"] == t0["kernel_launches"]  # kept again (limits still computed)
    f2 = s.field_numpy() * np.float32(0.8)
    for x in (r, q):
        x.set_depth_buffer(None)
        x.set_volume(f2, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    t = both(cam)
    assert t["kernel_launches"] > t0["kernel_launches"] - 1
    # the form and its field's type move the samples: the precision form marks
    # again, and again after its dtype changes
    for dt in (B.BF16, B.F16):
        for x in (r, q):
            x.set_form(B.FORM_PRECISION, field_dtype=dt)
        both(cam)  # a new quad copy and marks
        t = both(cam)
        assert t["kernel_launches"] == t0["kernel_launches"] - 1  # marks kept within the form
    with pytest.raises(B.BeamsError):
        r._check(r._L.beams_set_lazy_shadow_map(r._h, 3))


@pytest.mark.parametrize("skip", [True, False])
def test_lazy_first_frame_with_transparent_colour_map_range(cuda_device, skip):
    """Samples of alpha 0 mark no cell (they add exactly 0 whatever finite map
    value they read; a masked build's new map buffer is zeroed): a colour map
    transparent below 0.45 leaves many samples unmarked. The lazy frame is the
    renderer's first, so an unbuilt vertex holds only what the allocation left,
    and it must equal a full-map render from another renderer."""
    s = scenes.small(10, n=48, image=96, m=24, kind="blobs", light_kind=0)
    tf = np.array(s.tf, np.float32).copy()
    tf[: int(0.45 * len(tf)), 3] = 0.0
    s.tf = tf
    lazy_r, full_r = renderer(s), renderer(s)
    for x in (lazy_r, full_r):
        x.set_tuning(light_brick=8, empty_skip=skip, view_skip=skip)
    lazy_r.set_lazy_shadow_map(True)
    lazy, tl = lazy_r.render(s.camera())
    full, tfull = full_r.render(s.camera())
    assert np.array_equal(lazy, full), f"differs by {np.max(np.abs(lazy - full))}"
    assert tl["lit_samples"] == tfull["lit_samples"]
    assert 0 < tl["map_vertices"] < tfull["map_vertices"]
    assert np.all(np.isfinite(lazy))
