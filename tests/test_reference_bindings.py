"""The reference's own bindings driving this library (B200 only).

1. The Blender add-on's ctypes contract (c_api_contract.py, passed by
   engine.py:88-147 to sheen_render_scene): a scene built with those
   classes, recorded as raw bytes in golden/contract_scene.npz by
   golden/make_contract_fixture.py, is handed to sheen_render_scene as the
   add-on would.  The PNG equals the one this library writes for the same
   scene through its own contract, and the image matches the reference's own
   code built for the host.  The contract's HeightField is 72 bytes against
   64 in C (a pointer-alignment tail), so an add-on scene with more than one
   heightfield is misread from the second one on; the fixture has exactly
   one, and the sizes are asserted here to document the defect.
2. The reference's native module (api/sheen_py_module.cpp, built unchanged
   against this library into oracle/_ref by oracle/Makefile) imported as
   `sheen`: init / render_scene / cleanup on the same scene, in a child
   process (cleanup resets the device), writes the same PNG.
"""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import sheen_b200 as sb
from helpers import contract_scene
from oracle_bindings import RefHost, image_error

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
W, H, AA = 160, 120, 4


def test_addon_contract_scene_renders_through_the_drop_in(tmp_path):
    buf, keep, f = contract_scene()
    assert int(f["sizeof_SheenScene"]) == 344 and int(f["sizeof_HeightField"]) == 72
    from sheen_b200 import contract
    assert contract.HEIGHTFIELD.itemsize == 64               # the C layout, which this library keeps
    addr = ctypes.addressof(buf)
    sb.init(0, 100)
    p = tmp_path / "addon.png"
    sb.render_scene(addr, W, H, AA, str(p))
    img, st = sb.render_rgba(addr, W, H, AA, sb.FORM_PLAIN)
    assert st["primary_rays"] == W * H * AA and np.isfinite(img).all()
    q = tmp_path / "own.png"
    sb.write_png(str(q), img)
    from test_abi import _png_rows
    assert np.array_equal(_png_rows(str(p)), _png_rows(str(q)))
    assert RefHost.available(), "oracle/_ref/libsheen_ref_host.so is not built"
    ref = RefHost()
    h = ref.scene(addr)
    r = ref.render(h, W, H, AA)
    h.close()
    err = image_error(img, r)
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.01, err
    wimg, _ = sb.render_rgba(addr, W, H, AA, sb.FORM_WAVEFRONT)
    assert image_error(wimg, r)["mean_abs"] <= 1e-3


_MODULE = textwrap.dedent(r"""
    import sys
    sys.path.insert(0, sys.argv[1] + "/oracle/_ref")
    sys.path.insert(0, sys.argv[1] + "/tests")
    import sheen                      # the reference's native module
    from helpers import contract_scene
    buf, keep, f = contract_scene()
    sheen.init(0, 100)
    sheen.render_scene(buf, 160, 120, 4, sys.argv[2])
    sheen.cleanup()
    print("module ok", sheen.__file__)
""")


def test_reference_native_module_renders_through_this_library(tmp_path):
    mods = [n for n in os.listdir(os.path.join(ROOT, "oracle", "_ref")) if n.startswith("sheen.") and n.endswith(".so")]
    assert mods, "oracle/_ref/sheen*.so (the reference's module) is not built"
    out = tmp_path / "module.png"
    r = subprocess.run([sys.executable, "-c", _MODULE, ROOT, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "module ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    buf, keep, _ = contract_scene()
    sb.init(0, 100)
    own = tmp_path / "own.png"
    sb.render_scene(ctypes.addressof(buf), W, H, AA, str(own))
    from test_abi import _png_rows
    assert np.array_equal(_png_rows(str(out)), _png_rows(str(own)))
