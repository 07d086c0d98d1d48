"""The allocation-free render entry point (sheen_scene_render_region_noalloc).

Callers that cannot let the library allocate GPU memory mid-frame (a frame
recorded into a CUDA graph, where cudaMalloc is not allowed during capture;
a real-time loop whose device memory is all reserved at start-up) render
small regions through this entry point, whose scratch lives in a fixed
device array.  This file is collected last so that a failure here cannot
hide a failure elsewhere; it initialises the device itself and runs the same
way alone or after the other tests.

The check: two calls in a row on the same region give the image the regular
region entry point gives, within the pixel bar of the parity tests (mean
absolute error <= 1e-3), and requests beyond the stated limit are refused.
"""
import ctypes

import numpy as np
import pytest

import sheen_b200 as sb

pytestmark = pytest.mark.gpu


def _noalloc():
    L = sb.lib()
    f = L.sheen_scene_render_region_noalloc
    f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("config,detail,aa", [(1, 4, 4), (0, 0, 1)])
def test_noalloc_matches_regular_entry_point(config, detail, aa):
    import torch
    sb.init(0, 100)
    scene = sb.generate_scene(config, 5, detail)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    W, H = 320, 180
    x0, y0, x1, y1 = (96, 40, 160, 104) if aa == 4 else (64, 32, 192, 160)
    ref = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    ds.render_region(W, H, aa, x0, y0, x1, y1, ref.data_ptr(), 0)
    torch.cuda.synchronize()
    f = _noalloc()
    for _ in range(2):   # the shared scratch keeps the last call's contents
        out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        rc = f(ds.handle, W, H, aa, x0, y0, x1, y1, out.data_ptr(), None)
        assert rc == 0, sb.last_error()
        torch.cuda.synchronize()
        a = ref[y0:y1, x0:x1].cpu().numpy()
        b = out[y0:y1, x0:x1].cpu().numpy()
        assert np.isfinite(b).all()
        assert np.abs(a[..., :3] - b[..., :3]).mean() <= 1e-3
        # pixels outside the region are untouched
        assert float(out[:y0].abs().sum()) == 0.0
    ds.close()


def test_noalloc_rejects_oversized_requests():
    import torch
    sb.init(0, 100)
    scene = sb.generate_scene(0, 1)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    out = torch.zeros((480, 640, 4), dtype=torch.float32, device="cuda")
    f = _noalloc()
    assert f(ds.handle, 640, 480, 1, 0, 0, 640, 480, out.data_ptr(), None) == -1
    assert "at most 16384 samples" in sb.last_error()
    plain = sb.DeviceScene(scene, sb.FORM_PLAIN)
    assert f(plain.handle, 640, 480, 1, 0, 0, 64, 64, out.data_ptr(), None) == -1
    assert "SHEEN_FORM_WAVEFRONT" in sb.last_error()
    ds.close()
    plain.close()
