"""The .sheen loader (sheen_load_scene_file) against the reference loader
(api/scene_io.cpp, built for the host from the reference tree) on every
reference scene that loads here, and on this repository's fixtures; plus
error reporting (CPU only)."""
import ctypes
import glob
import os

import numpy as np
import pytest

import sheen_b200 as sb
from sheen_b200 import contract as C
from oracle_bindings import RefHost

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _arrays(view):
    out = {}
    for name, dt in C.ARRAY_FIELDS:
        n, p = getattr(view, "num_" + name), getattr(view, name)
        out[name] = (np.frombuffer((ctypes.c_ubyte * (n * dt.itemsize)).from_address(p), dt).copy()
                     if n else np.zeros(0, dt))
    return out


def _compare(ref_view, mine_view):
    a, b = _arrays(ref_view), _arrays(mine_view)
    for name, dt in C.ARRAY_FIELDS:
        assert a[name].shape == b[name].shape, name
        for f in dt.names:
            if f == "image":
                continue
            assert np.array_equal(a[name][f], b[name][f]), (name, f)
    assert bytes(ref_view.camera) == bytes(mine_view.camera)
    assert ref_view.csg_root == mine_view.csg_root
    assert ref_view.num_textures == mine_view.num_textures
    for i in range(ref_view.num_textures):
        wa = ctypes.cast(ref_view.texture_widths, ctypes.POINTER(ctypes.c_int))[i]
        wb = ctypes.cast(mine_view.texture_widths, ctypes.POINTER(ctypes.c_int))[i]
        assert wa == wb


def _load_both(path, cwd):
    ref = RefHost()
    old = os.getcwd()
    os.chdir(cwd)
    try:
        h = ref.lib.sheen_ref_load_scene_file(path.encode())
        try:
            mine = sb.load_scene_file(path)
        except RuntimeError:
            mine = None
    finally:
        os.chdir(old)
    return ref, h, mine


@pytest.mark.skipif(not RefHost.available(), reason="reference host build absent")
def test_reference_scenes_load_identically(reference_tree):
    loaded = 0
    for path in sorted(glob.glob(os.path.join(reference_tree, "scenes", "*.sheen"))):
        ref, h, mine = _load_both(path, reference_tree)
        if not h:
            # scenes whose side files are missing (/tmp/cliff64.pgm, ...) fail in both
            assert mine is None, path
            continue
        _compare(C.SheenScene.from_address(ref.lib.sheen_ref_loaded_view(h)), mine.view)
        st = (ctypes.c_int * 4)()
        ref.lib.sheen_ref_loaded_settings(h, st)
        m = mine.settings
        assert list(st) == [m["width"], m["height"], m["aa"], m["photons"]], path
        ref.lib.sheen_ref_loaded_free(h)
        loaded += 1
    assert loaded >= 10


@pytest.mark.skipif(not RefHost.available(), reason="reference host build absent")
@pytest.mark.parametrize("name", ["features_a.sheen", "features_b.sheen"])
def test_fixture_scenes_load_identically(name):
    ref, h, mine = _load_both(name, GOLDEN)
    assert h and mine is not None
    _compare(C.SheenScene.from_address(ref.lib.sheen_ref_loaded_view(h)), mine.view)
    ref.lib.sheen_ref_loaded_free(h)


def test_fixture_contents():
    old = os.getcwd()
    os.chdir(GOLDEN)
    try:
        s = sb.load_scene_file("features_b.sheen")
    finally:
        os.chdir(old)
    v = s.view
    assert v.num_textures == 2 and v.num_heightfields == 1 and v.num_media == 1
    assert v.num_sweep_strands == 41 and v.num_lights == 4
    assert s.settings["aa"] == 4 and s.settings["width"] == 80


def test_errors_name_the_line(tmp_path):
    p = tmp_path / "bad.sheen"
    p.write_text("material 0.5 0.5 0.5 0 8 0.1\nsphere 0 0 0 1 0\nbogus 1 2 3\n")
    with pytest.raises(RuntimeError, match="line 3"):
        sb.load_scene_file(str(p))
    with pytest.raises(RuntimeError, match="cannot open"):
        sb.load_scene_file(str(tmp_path / "missing.sheen"))
    p.write_text("material 0.5 0.5 0.5 0 8 0.1\nsphere 0 0 0 1 7\nplane 0 1 0 0 -3\n")
    s = sb.load_scene_file(str(p))
    objs = np.frombuffer((ctypes.c_ubyte * 48).from_address(s.view.objects), C.OBJECT)
    assert objs["material_id"][0] == 0   # out-of-range material ids fall back to 0
