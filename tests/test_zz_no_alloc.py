"""beams_render_noalloc: the render entry point for callers that may not
allocate device memory themselves (a plugin or custom call living inside
another framework's memory management, or a frame loop that must not stall on
cudaMalloc/cudaFree). Its only scratch, the frame's transmittance map, is a
static device array of at most BEAMS_NOALLOC_MAX_MAP_CELLS = 128 cells per axis.

The test calls it through the C ABI twice in a row, on two different scenes,
and checks each image against the regular entry point (beams_render) bit for
bit: both run the same march code (march_vertex, view_march_pixel), this one
on the plain field with cell tables computed in shared memory. It lives in its
own file, collected last, and passes alone in a fresh process as well as after
the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
MAX_CELLS = 128


def _fn():
    f = B.lib().beams_render_noalloc
    P = C.c_void_p
    f.argtypes = [C.POINTER(B.Volume), P, C.c_int, P, P, C.c_float, C.c_int, C.c_float, C.c_float,
                  C.POINTER(B.Camera), P, P]
    f.restype = C.c_int
    return f


def _render_noalloc(s, field_dev, tf_dev, out_dev, data_offset=0, tf_n=None, light_color=None):
    import torch
    nz, ny, nx = field_dev.shape
    vol = B.Volume(C.c_void_p(field_dev.data_ptr() + data_offset), B.F32, (C.c_int * 3)(nx, ny, nz),
                   (C.c_double * 3)(*s.origin), (C.c_double * 3)(*s.spacing),
                   (C.c_double * 2)(*s.value_range), B.ASSOC_POINTS, 1)
    cam = s.camera()
    light = (C.c_double * 3)(*s.light)
    color = (C.c_float * 3)(*(s.light_color if light_color is None else light_color))
    n = tf_dev.shape[0] if tf_n is None else tf_n
    st = _fn()(C.byref(vol), C.c_void_p(tf_dev.data_ptr()), n, light, color, s.light_intensity,
               s.map_m, s.sample_distance, s.cutoff, C.byref(cam), C.c_void_p(out_dev.data_ptr()),
               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st


def _render_regular(s):
    with B.Renderer(0) as r:
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        img, _ = r.render(s.camera())
    return img


def test_noalloc_matches_regular_render_two_calls_in_a_row(cuda_device):
    import torch
    a = scenes.small(21, n=40, image=72, m=24, kind="blobs", light_kind=0)
    b = scenes.small(22, n=33, image=64, m=MAX_CELLS, kind="noise", light_kind=0)
    b.cutoff = 0.99
    outs = []
    for s in (a, b):  # two calls in a row, sharing the one static scratch map
        fd = torch.from_numpy(s.field_numpy()).cuda()
        tf = torch.from_numpy(np.ascontiguousarray(s.tf, np.float32)).cuda()
        out = torch.full((s.height, s.width, 4), -1.0, dtype=torch.float32, device="cuda")
        assert _render_noalloc(s, fd, tf, out) == 0, B.lib().beams_last_error(None)
        outs.append((s, fd, tf, out))
    torch.cuda.synchronize()
    for s, _, _, out in outs:
        got = out.cpu().numpy()
        ref = _render_regular(s)
        assert np.array_equal(got, ref), f"{s.name}: max |d| {float(np.max(np.abs(got - ref)))}"
        assert np.all(got[..., 3] >= 0.0)
    # The second call's map (M = 128, the limit) overwrote the first one's; a
    # repeat of the first scene must still match (each call rewrites its map).
    s, fd, tf, out = outs[0]
    out.fill_(-1.0)
    assert _render_noalloc(s, fd, tf, out) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), _render_regular(s))


def test_noalloc_rejects_maps_beyond_the_static_scratch(cuda_device):
    import torch
    s = scenes.small(23, n=16, image=8, m=MAX_CELLS + 1)
    fd = torch.from_numpy(s.field_numpy()).cuda()
    tf = torch.from_numpy(np.ascontiguousarray(s.tf, np.float32)).cuda()
    out = torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda")
    st = _render_noalloc(s, fd, tf, out)
    assert st == 1  # BEAMS_ERR_INVALID_ARG
    assert b"128" in B.lib().beams_last_error(None)
    # Arguments the call checks on the host before it launches anything: a
    # field pointer that is not 4-byte aligned, a non-finite light colour, and a
    # colour map size outside [1, 1024].
    ok = scenes.small(24, n=16, image=8, m=8)
    fd = torch.from_numpy(ok.field_numpy()).cuda()
    assert _render_noalloc(ok, fd, tf, out, data_offset=2) == 1
    assert b"aligned" in B.lib().beams_last_error(None)
    assert _render_noalloc(ok, fd, tf, out, light_color=(1.0, float("nan"), 1.0)) == 1
    assert _render_noalloc(ok, fd, tf, out, tf_n=0) == 1
    assert _render_noalloc(ok, fd, tf, out, tf_n=1025) == 1
    assert _render_noalloc(ok, fd, tf, out) == 0
    torch.cuda.synchronize()
    # axes too long for the shared-memory cell tables: refused before any launch
    # (the buffer holds the whole claimed volume all the same)
    big = torch.zeros((2, 4000, 8192), dtype=torch.float32, device="cuda")
    assert _render_noalloc(ok, big, tf, out) == 2  # BEAMS_ERR_UNSUPPORTED
    assert b"shared-memory" in B.lib().beams_last_error(None)
