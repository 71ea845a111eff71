"""Precision form: the field in bfloat16 or binary16, optical depth accumulated in
float32 with Kahan compensation, the map as binary16 transmittance.

Parity: against the oracle's precision mode on the same quantized field — the
map (binary16 transmittance) bit-exact and the image max |dRGBA| <= 2e-3
(expected bit-exact). Accuracy: reported against the FP64 oracle on the
unquantized field, beside the exact FP32 path's."""
import numpy as np
import pytest

from oracle.oracle import Oracle, psnr, quantize
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def render_prec(s, dt, field=None):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy() if field is None else field, origin=s.origin, spacing=s.spacing,
                 value_range=s.value_range)
    s.configure(r)
    r.set_form(B.FORM_PRECISION, field_dtype=dt)
    img, t = r.render(s.camera())
    m = r.get_shadow_map((s.map_m + 1) ** 3).reshape((s.map_m + 1,) * 3)
    return img, m, t


@pytest.mark.parametrize("dt,name", [(B.BF16, "bf16"), (B.F16, "f16")])
@pytest.mark.parametrize("kind,light_kind", [("blobs", 0), ("noise", 1)])
def test_precision_matches_oracle_precision_mode(cuda_device, dt, name, kind, light_kind):
    s = scenes.small(41, n=40, image=96, m=20, kind=kind, light_kind=light_kind)
    img, m, t = render_prec(s, dt)
    q = quantize(s.field_numpy(), name)
    o = Oracle(s, field=q, precision=True)
    om, _ = o.light_march()
    assert np.array_equal(m, om), f"map: {np.sum(m != om)} of {m.size} differ, max {np.abs(m - om).max()}"
    oimg, lit = o.view_march(om)
    assert np.max(np.abs(img - oimg)) <= TOL
    assert np.mean(np.all(img == oimg, axis=-1)) > 0.999
    assert t["lit_samples"] == lit
    # accuracy against the FP64 oracle on the unquantized field, beside the FP32 exact path
    o64 = Oracle(s)
    ref64, _ = o64.view_march(o64.light_march(fp64=True)[0], fp64=True)
    with B.Renderer(0) as rr:
        rr.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(rr)
        exact, _ = rr.render(s.camera())
    p_prec, p_exact = psnr(img, ref64), psnr(exact, ref64)
    print(f"{name} {kind}: PSNR vs f64 precision {p_prec:.1f} dB, exact {p_exact:.1f} dB, "
          f"max|d| {np.abs(img - ref64).max():.2e} mean {np.abs(img - ref64).mean():.2e}")
    assert p_prec > 35


def test_16bit_volume_input_equals_converted_float_input(cuda_device):
    import torch
    s = scenes.small(42, n=32, image=64, m=16)
    img_a, m_a, _ = render_prec(s, B.BF16)
    fb = torch.from_numpy(s.field_numpy()).cuda().to(torch.bfloat16)
    img_b, m_b, _ = render_prec(s, B.BF16, field=fb)
    assert np.array_equal(m_a, m_b) and np.array_equal(img_a, img_b)


def test_precision_transmittance_is_monotone_kahan_sum(cuda_device):
    """A constant field gives T = exp(-k tau) for whole k along each light ray."""
    s = scenes.small(43, n=16, image=8, m=8, light_kind=1)
    s.light = (0.013, 0.021, 1.0)
    s.array = np.full((16, 16, 16), 0.45, np.float32)
    _, m, _ = render_prec(s, B.F16)
    idx = int(np.float32(np.float32(0.45)) * np.float32(255))
    a = np.float32(s.tf[idx, 3]) / np.float32(s.tf[:, 3].max())
    tau = -np.log1p(-np.float64(a))
    k = -np.log(np.maximum(m.astype(np.float64), 1e-30)) / tau
    ok = m > 1e-3
    assert np.allclose(k[ok], np.round(k[ok]), atol=0.02)
