"""Multi-light extension of the exact form (off by default).

The reference shades with the first light only (LightedVolumeRenderer.cxx:836-840
reads Locations[0]; the source carries a note to refactor for several lights).
With beams_set_multi_light(1) the renderer builds one map per light (K1 once per
light, maps stacked in light order) and K2 shades each sample with
sum_l (1 - opacity_l) * colour_l * intensity_l, accumulated in light order.

Bars: each stacked map equals the single-light oracle map of that light bit for
bit; the image equals the oracle's multi-light march bit for bit on >= 99.9% of
pixels and within 2e-3 everywhere (the exact form's K2 bar); with the switch off
the first light alone shades the image, as in the reference.
"""
import copy

import numpy as np
import pytest

from oracle.oracle import Oracle
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3

EXTRA = [
    # (kind, position or direction, colour, intensity)
    (0, (1.6, 0.2, -0.4), (0.9, 0.5, 0.2), 0.8),
    (1, (-0.3, -1.0, 0.2), (0.2, 0.4, 1.0), 0.6),
]


def light_scene(s, kind, pos, color, intensity):
    t = copy.copy(s)
    t.light_kind, t.light, t.light_color, t.light_intensity = kind, tuple(pos), tuple(color), float(intensity)
    return t


def setup(s, lights, multi):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    for kind, pos, color, inten in lights:
        if kind == 0:
            r.add_point_light(pos, color, inten)
        else:
            r.add_directional_light(pos, color, inten)
    r.set_multi_light(multi)
    return r


@pytest.mark.parametrize("seed,nextra", [(0, 1), (2, 2)])
def test_multi_light_maps_and_image_match_oracle(cuda_device, seed, nextra):
    s = scenes.small(seed, n=40, image=96, m=20, kind="blobs" if seed == 0 else "noise")
    lights = EXTRA[:nextra]
    r = setup(s, lights, True)
    img, t = r.render(s.camera())
    nv = (s.map_m + 1) ** 3
    nl = 1 + nextra
    maps = r.get_shadow_map(nl * nv).reshape(nl, nv)
    scenes_l = [s] + [light_scene(s, *L) for L in lights]
    for l, sl in enumerate(scenes_l):
        om, _ = Oracle(sl).light_march()
        assert np.array_equal(maps[l], om.reshape(-1)), f"light {l}: map differs by {np.max(np.abs(maps[l] - om))}"
    lc = np.stack([np.float32(sl.light_color) * np.float32(sl.light_intensity) for sl in scenes_l])
    oimg, olit = Oracle(s).view_march_multi(maps, lc)
    err = np.abs(img - oimg)
    same = np.mean(np.all(img == oimg, axis=-1))
    assert err.max() <= TOL, f"max |d| {err.max()}"
    assert same > 0.999, f"only {same:.4f} of pixels bit-identical"
    assert t["lit_samples"] == olit
    print(f"multi-light seed {seed}: {nl} lights, identical {same:.5f}, max|d| {err.max():.2e}")


def test_multi_light_off_shades_with_first_light_only(cuda_device):
    s = scenes.small(1, n=32, image=64, m=16)
    img_off, _ = setup(s, EXTRA, False).render(s.camera())
    r1 = B.Renderer(0)
    r1.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r1)
    img_one, _ = r1.render(s.camera())
    assert np.array_equal(img_off, img_one)


def test_two_half_lights_equal_one_full_light(cuda_device):
    s = scenes.small(3, n=32, image=64, m=16, light_kind=1)
    r1 = B.Renderer(0)
    r1.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r1)
    full, _ = r1.render(s.camera())
    h = copy.copy(s)
    h.light_intensity = s.light_intensity * 0.5
    r2 = setup(h, [(h.light_kind, h.light, h.light_color, h.light_intensity)], True)
    two, _ = r2.render(s.camera())
    assert np.array_equal(full, two)


def test_multi_light_rejected_outside_exact_form(cuda_device):
    s = scenes.small(4, n=24, image=32, m=8)
    r = setup(s, EXTRA[:1], True)
    r.set_form(B.FORM_PRECISION, B.BF16)
    with pytest.raises(B.BeamsError):
        r.render(s.camera())
