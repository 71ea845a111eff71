"""Fault handling without faulting the GPU: NaN fields and out-of-range values
render like the oracle, an injected allocation failure returns BEAMS_ERR_OOM and
the next call works, and the batch kernel's bounded wait (a map item that never
publishes its completion) ends with BEAMS_ERR_TIMEOUT on a context that stays usable."""
import time

import numpy as np
import pytest

from oracle.oracle import Oracle
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
OOM, TIMEOUT = 4, 5


def _renderer(s, field=None):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy() if field is None else field, origin=s.origin, spacing=s.spacing,
                 value_range=s.value_range)
    s.configure(r)
    return r


def test_nan_field_renders_like_the_oracle(cuda_device):
    s = scenes.small(91, n=32, image=48, m=12, kind="blobs")
    f = s.field_numpy().copy()
    f[10:14, :, 5:20] = np.nan
    s.array = f
    with _renderer(s, f) as r:
        img, t = r.render(s.camera())
        m = r.get_shadow_map((s.map_m + 1) ** 3)
    o = Oracle(s)
    om, _ = o.light_march()
    oimg, lit = o.view_march(om)
    assert np.array_equal(m, om.ravel(), equal_nan=True)
    assert np.array_equal(img, oimg, equal_nan=True) and t["lit_samples"] == lit


def test_values_outside_the_range_render_like_the_oracle(cuda_device):
    s = scenes.small(92, n=32, image=48, m=12, kind="noise")
    s.value_range = (0.2, 0.6)  # the field spans [0, 1]: TF indices fall outside the table
    with _renderer(s) as r:
        img, t = r.render(s.camera())
        m = r.get_shadow_map((s.map_m + 1) ** 3)
    o = Oracle(s)
    om, _ = o.light_march()
    oimg, lit = o.view_march(om)
    assert np.array_equal(m, om.ravel()) and np.array_equal(img, oimg) and t["lit_samples"] == lit


def test_injected_allocation_failure_is_reported_and_recovered(cuda_device):
    s = scenes.small(93, n=24, image=32, m=8)
    with _renderer(s) as r:
        ref, _ = r.render(s.camera())
        r.set_shadow_map_size(10)          # the next render needs a new map buffer
        B.lib().beams_test_fail_allocation(1)
        with pytest.raises(B.BeamsError) as e:
            r.render(s.camera())
        assert e.value.status == OOM and "injected" in str(e.value)
        img, _ = r.render(s.camera())     # the same call succeeds once memory is available
        r.set_shadow_map_size(s.map_m)
        img2, _ = r.render(s.camera())
        assert np.array_equal(img2, ref)
    B.lib().beams_test_fail_allocation(0)


def test_batch_wait_times_out_and_the_context_survives(cuda_device):
    vols = [scenes.small(94, n=24, kind="blobs")]
    cam = B.Renderer.camera((0.5, 0.5, 2.0), (0.5, 0.5, 0.5), (0, 1, 0), 30.0, 32, 32)
    with B.Renderer(0) as r:
        r.set_color_map(scenes.tf_table())
        r.batch_set_volumes([(s.field_numpy(), s.origin, s.spacing, s.value_range) for s in vols])
        r.set_batch_options(_withhold=True)
        t0 = time.time()
        with pytest.raises(B.BeamsError) as e:
            r.render_batch([B.Renderer.request(0, cam, (0.5, 3.0, 0.5), map_cells=8)])
        waited = time.time() - t0
        assert e.value.status == TIMEOUT and waited < 60
        r.set_batch_options()
        outs, t = r.render_batch([B.Renderer.request(0, cam, (0.5, 3.0, 0.5), map_cells=8)])
        assert t["lit_samples"] > 0 and np.isfinite(outs[0]).all()
