"""The allocation-free render entry point (sheen_scene_render_region_noalloc).

Some callers cannot let the library allocate GPU memory while they draw: a
real-time loop that reserves all of its device memory at start-up and treats
any later allocation as a fault, or an application whose own memory manager
must own every byte on the device.  They render small regions through this
entry point, whose scratch lives in a fixed array in the library's device
globals.  This file is collected last so that a failure here cannot hide a
failure elsewhere; it initialises the device itself and runs the same way
alone or after the other tests.

The checks: two calls in a row on the same region give exactly the image the
regular region entry point gives (the same queue kernels run on the same
inputs, so the bar is bit equality, which is inside the parity tests' 1e-3
mean absolute error); the Moller-Trumbore and watertight triangle variants,
the all-categories variant and the megakernel fallback (media) are covered;
requests beyond the stated limit are refused; and the entry point still
works after sheen_cleanup and a second sheen_init in the same process.
"""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import sheen_b200 as sb
from cases import CASES
from helpers import load_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _noalloc():
    L = sb.lib()
    f = L.sheen_scene_render_region_noalloc
    f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _scene(kind):
    if kind == "features_b":
        return load_case(next(c for c in CASES if c["name"] == "features_b"))
    cfg, seed, detail = {"mesh": (1, 5, 4), "spheres": (0, 5, 0), "analytic": (2, 5, 0)}[kind.split("_")[0]]
    return sb.generate_scene(cfg, seed, detail)


@pytest.mark.parametrize("kind,aa,region", [
    ("mesh", 4, (96, 40, 160, 104)),
    ("mesh_watertight", 4, (96, 40, 160, 104)),
    ("spheres", 1, (64, 32, 192, 160)),
    ("analytic", 1, (100, 50, 228, 178)),
    ("features_b", 4, (0, 0, 64, 64)),          # media: the megakernel fallback
])
def test_noalloc_matches_regular_entry_point(kind, aa, region):
    import torch
    sb.init(0, 100)
    scene = _scene(kind)
    if kind.endswith("watertight"):
        sb.tune_set("trace.watertight", 1)
    try:
        ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    finally:
        sb.tune_set("trace.watertight", 0)
    W, H = 320, 180
    x0, y0, x1, y1 = region
    ref = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    ds.render_region(W, H, aa, x0, y0, x1, y1, ref.data_ptr(), 0)
    torch.cuda.synchronize()
    a = ref[y0:y1, x0:x1].cpu().numpy()
    assert np.isfinite(a).all() and float(np.abs(a[..., :3]).sum()) > 0
    f = _noalloc()
    for _ in range(2):   # the shared scratch keeps the last call's contents
        out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        rc = f(ds.handle, W, H, aa, x0, y0, x1, y1, out.data_ptr(), None)
        assert rc == 0, sb.last_error()
        torch.cuda.synchronize()
        b = out[y0:y1, x0:x1].cpu().numpy()
        assert np.array_equal(a, b), float(np.abs(a - b).max())
        # pixels outside the region are untouched
        assert float(out[:y0].abs().sum()) == 0.0 and float(out[y1:].abs().sum()) == 0.0
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
    # 64x64 at 4 spp is exactly the limit; 72x64 pads to 80x64 and is over it
    assert f(ds.handle, 640, 480, 4, 0, 0, 64, 64, out.data_ptr(), None) == 0, sb.last_error()
    assert f(ds.handle, 640, 480, 4, 0, 0, 72, 64, out.data_ptr(), None) == -1
    plain = sb.DeviceScene(scene, sb.FORM_PLAIN)
    assert f(plain.handle, 640, 480, 1, 0, 0, 64, 64, out.data_ptr(), None) == -1
    assert "SHEEN_FORM_WAVEFRONT" in sb.last_error()
    torch.cuda.synchronize()
    ds.close()
    plain.close()


# Run in a child process that never touches torch: sheen_cleanup resets the
# device (as the reference's cleanup does), which would invalidate memory a
# torch allocator in the same process still holds.  Device memory for the
# allocation-free call comes from the CUDA driver API directly.
_CYCLE = textwrap.dedent(r"""
    import ctypes, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    import sheen_b200 as sb
    cu = ctypes.CDLL("libcuda.so.1")
    f = sb.lib().sheen_scene_render_region_noalloc
    f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    W, H, aa, R = 160, 96, 4, (32, 16, 96, 80)

    def noalloc(ds):
        ptr = ctypes.c_uint64()
        assert cu.cuMemAlloc_v2(ctypes.byref(ptr), W * H * 16) == 0
        assert cu.cuMemsetD8_v2(ptr, 0, W * H * 16) == 0
        assert f(ds.handle, W, H, aa, *R, ctypes.c_void_p(ptr.value), None) == 0, sb.last_error()
        host = np.empty((H, W, 4), np.float32)
        assert cu.cuMemcpyDtoH_v2(host.ctypes.data_as(ctypes.c_void_p), ptr, W * H * 16) == 0
        assert cu.cuMemFree_v2(ptr) == 0
        return host[R[1]:R[3], R[0]:R[2]]

    def run(png):
        sb.init(0, 100)
        scene = sb.generate_scene(1, 5, 4)
        ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)    # device BVH build
        img, _ = ds.render_host(W, H, aa)
        reg = noalloc(ds)
        ds.close()
        sb.render_scene(sb.generate_scene(0, 1), 64, 48, 1, png)   # device sRGB pack
        return img, reg, open(png, "rb").read()

    a = run(sys.argv[2] + "/a.png")
    sb.cleanup()
    b = run(sys.argv[2] + "/b.png")
    assert np.array_equal(a[0], b[0]), "regular render differs after cleanup"
    assert np.array_equal(a[1], b[1]), "allocation-free render differs after cleanup"
    assert np.array_equal(b[1], b[0][R[1]:R[3], R[0]:R[2]]), "allocation-free != regular"
    assert a[2] == b[2], "PNG bytes differ after cleanup"
    sb.cleanup()
    print("cycle ok")
""")


def test_noalloc_after_cleanup_and_reinit(tmp_path):
    r = subprocess.run([sys.executable, "-c", _CYCLE, ROOT, str(tmp_path)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "cycle ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
