"""Explicit rectilinear coordinates (beams_set_volume_coordinates): the
reference's RenderCells takes a rectilinear coordinate system, the Cartesian
product of three coordinate arrays, which its locators search
(LightedVolumeRenderer.cxx:45-186, RectilinearMeshOracle.h:140-176).

Bars: maps bit-exact against the oracle on the same coordinates, images within
the exact form's bar (max |dRGBA| <= 2e-3, >= 99.9% of pixels bit-identical),
equal lit-sample counts; explicit coordinates equal to the generated uniform
ones give the uniform image bit for bit.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, quantize
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def stretched(n, kind, seed):
    t = np.linspace(0.0, 1.0, n)
    if kind == "power":
        return tuple(np.float32(t ** p) for p in (1.5, 1.0, 0.7))
    rng = np.random.default_rng(seed)  # jittered: every spacing in [0.4, 1.6] of the mean
    out = []
    for _ in range(3):
        w = rng.uniform(0.4, 1.6, n - 1)
        c = np.concatenate([[0.0], np.cumsum(w)])
        out.append(np.float32(c / c[-1]))
    return tuple(out)


def render(s, form=B.FORM_EXACT, dt=B.BF16):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    if getattr(s, "coords", None) is not None:
        r.set_volume_coordinates(*s.coords)
    s.configure(r)
    if form == B.FORM_PRECISION:
        r.set_form(B.FORM_PRECISION, field_dtype=dt)
    img, t = r.render(s.camera())
    m = r.get_shadow_map((s.map_m + 1) ** 3).reshape((s.map_m + 1,) * 3)
    return img, m, t, r


def check(img, oimg):
    assert np.max(np.abs(img - oimg)) <= TOL, f"max |d| {np.max(np.abs(img - oimg))}"
    assert np.mean(np.all(img == oimg, axis=-1)) > 0.999


@pytest.mark.parametrize("kind,light_kind,slab64", [("power", 0, True), ("jitter", 1, True), ("jitter", 0, False)])
def test_rectilinear_exact_matches_oracle(cuda_device, kind, light_kind, slab64):
    s = scenes.small(21, n=40, image=80, m=16, kind="noise" if kind == "jitter" else "blobs", light_kind=light_kind)
    s.slab_fp64 = slab64
    s.coords = stretched(s.dims[0], kind, 21)
    img, m, t, _ = render(s)
    o = Oracle(s)
    om, _ = o.light_march()
    assert np.array_equal(m, om), f"map: {np.sum(m != om)} of {m.size} differ"
    oimg, olit = o.view_march(om)
    check(img, oimg)
    assert t["lit_samples"] == olit


@pytest.mark.parametrize("dt,name", [(B.BF16, "bf16"), (B.F16, "f16")])
def test_rectilinear_precision_matches_oracle(cuda_device, dt, name):
    s = scenes.small(22, n=40, image=80, m=16, kind="blobs")
    s.coords = stretched(s.dims[0], "jitter", 22)
    img, m, t, _ = render(s, B.FORM_PRECISION, dt)
    o = Oracle(s, field=quantize(s.field_numpy(), name), precision=True)
    om, _ = o.light_march()
    assert np.array_equal(m, om), f"map: {np.sum(m != om)} of {m.size} differ"
    oimg, olit = o.view_march(om)
    check(img, oimg)
    assert t["lit_samples"] == olit


def test_explicit_uniform_coordinates_give_the_uniform_image(cuda_device):
    s = scenes.small(23, n=40, image=80, m=16)
    base, bm, _, _ = render(s)
    c = np.float32(s.origin[0]) + np.float32(s.spacing[0]) * np.arange(s.dims[0], dtype=np.float32)
    s.coords = (c, c.copy(), c.copy())
    img, m, _, r = render(s)
    assert np.array_equal(m, bm) and np.array_equal(img, base)
    # clearing the coordinates (or a new volume) returns to the uniform grid
    r.set_volume_coordinates()
    again, _ = r.render(s.camera())
    assert np.array_equal(again, base)


def test_rectilinear_rejections(cuda_device):
    s = scenes.small(24, n=24, image=32, m=8)
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    c = np.linspace(0, 1, s.dims[0], dtype=np.float32)
    bad = c.copy()
    bad[5] = bad[4]
    with pytest.raises(B.BeamsError):
        r.set_volume_coordinates(bad, c, c)
    r.set_volume_coordinates(c, c, c)
    with pytest.raises(B.BeamsError):
        r.mlp_train(B.mlp_options(samples_log2=12, epochs=1))
