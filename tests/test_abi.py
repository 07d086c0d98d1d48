"""The drop-in boundary: struct layout and exported symbols (CPU only).

Ports the reference's layout asserts (tests/sizes_main.cpp:5-21) and extends
them to every struct of the scene contract and to SheenScene itself, checked
three ways: a C probe compiled against include/sheen_c_api.h, the numpy /
ctypes contract of sheen_b200.contract, and (when the reference tree is
present) a probe compiled against the reference's own types.h.
"""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import sheen_b200
from sheen_b200 import contract as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    # name: (size, {field: offset})
    "CameraData": (64, {"position": 0, "right": 12, "up": 24, "forward": 36, "focal_length": 48,
                        "sensor_width": 52, "shift_x": 56, "shift_y": 60}),
    "Material": (112, {"specular": 12, "texture_id": 24, "anisotropy": 32, "reflect": 60, "transmission": 64,
                       "ior": 68, "emission_color": 72, "emission": 84, "mask_id": 88, "normal_id": 92,
                       "normal_strength": 96}),
    "Triangle": (112, {"v0": 0, "n0": 36, "uv0": 72, "uv1": 80, "uv2": 88, "material_id": 96}),
    "Object": (48, {"type": 0, "material_id": 4, "param1": 8, "param2": 20}),
    "Light": (96, {"direction": 0, "position": 12, "u_axis": 24, "v_axis": 36, "color": 48, "intensity": 60,
                   "radius": 64, "angle": 68, "blend": 72, "beam": 76, "type": 80, "flags": 84, "texture_id": 88}),
    "Medium": (48, {"center": 0, "half": 12, "sigma_s": 24, "sigma_t": 36, "samples": 40}),
    "Plane": (32, {"normal": 0, "d": 12, "material_id": 16}),
    "SweepPoint": (16, {"position": 0, "radius": 12}),
    "SweepStrand": (16, {"point_offset": 0, "point_count": 4, "material_id": 8}),
    "HeightField": (64, {"center": 0, "size_x": 12, "height": 20, "octaves": 28, "seed": 32, "material_id": 36,
                         "image": 40, "img_w": 48, "img_h": 52}),
    "LathePoint": (16, {"y": 0, "radius": 4}),
    "Lathe": (32, {"center": 0, "point_offset": 12, "point_count": 16, "material_id": 20}),
    "PrismPoint": (16, {"x": 0, "z": 4}),
    "Prism": (48, {"center": 0, "y_min": 12, "y_max": 16, "sweep": 20, "point_offset": 24, "point_count": 28,
                   "material_id": 32}),
    "CSGNode": (32, {"op": 0, "leaf_kind": 4, "leaf_index": 8, "left": 12, "right": 16}),
    "Superellipsoid": (48, {"center": 0, "a": 12, "b": 16, "c": 20, "n": 24, "material_id": 28}),
    "SheenScene": (352, {"camera": 0, "objects": 64, "num_objects": 72, "triangles": 112, "csg_nodes": 224,
                         "csg_root": 232, "num_csg_nodes": 236, "materials": 256, "texture_pixels": 272,
                         "num_textures": 296, "lights": 304, "num_lights": 312, "photons": 316,
                         "photon_cell": 320, "caustics": 324, "media": 328, "num_media": 336}),}


def _probe(header_dir_args, prelude, lang="c"):
    lines = [prelude, "#include <stdio.h>", "#include <stddef.h>", "int main(void){"]
    for name, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe." + ("c" if lang == "c" else "cpp"))
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        comp = "gcc" if lang == "c" else "g++"
        subprocess.run([comp, "-w", *header_dir_args, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.strip().splitlines())}


def test_c_header_layout():
    got = _probe(["-I", os.path.join(ROOT, "include")], '#include "sheen_c_api.h"')
    for name, (size, fields) in STRUCTS.items():
        assert got[name] == size, name
        for f, off in fields.items():
            assert got[f"{name}.{f}"] == off, (name, f)


def test_reference_layout_matches(reference_tree):
    # The reference's own header is the authority for every size and offset.
    prelude = ('#include <cmath>\n#include <cuda_runtime.h>\n'
               'inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }\n#include "sheen_c_api.h"')
    got = _probe(["-I", reference_tree, "-I", "/usr/local/cuda/include"], prelude, lang="cpp")
    mine = _probe(["-I", os.path.join(ROOT, "include")], '#include "sheen_c_api.h"')
    for k, v in got.items():
        assert mine[k] == v, k


def test_numpy_and_ctypes_contract():
    dts = {"Material": C.MATERIAL, "Triangle": C.TRIANGLE, "Object": C.OBJECT, "Light": C.LIGHT,
           "Medium": C.MEDIUM, "Plane": C.PLANE, "SweepPoint": C.SWEEP_POINT, "SweepStrand": C.SWEEP_STRAND,
           "HeightField": C.HEIGHTFIELD, "LathePoint": C.LATHE_POINT, "Lathe": C.LATHE,
           "PrismPoint": C.PRISM_POINT, "Prism": C.PRISM, "CSGNode": C.CSG_NODE,
           "Superellipsoid": C.SUPERELLIPSOID, "CameraData": C.CAMERA}
    for name, dt in dts.items():
        size, fields = STRUCTS[name]
        assert dt.itemsize == size, name
        for f, off in fields.items():
            assert dt.fields[f][1] == off, (name, f)
    assert ctypes.sizeof(C.SheenScene) == 352
    for f, off in STRUCTS["SheenScene"][1].items():
        assert getattr(C.SheenScene, f).offset == off, f


def _declared_symbols():
    names = set()
    for h in ("sheen_c_api.h",):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(sheen_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(sheen_b200.LIB_PATH)
    declared = _declared_symbols()
    assert {"sheen_init", "sheen_cleanup", "sheen_render_scene", "sheen_get_last_error"} <= declared
    for name in sorted(declared):
        assert hasattr(lib, name), name


def test_errors_without_device_work():
    lib = sheen_b200.lib()
    s = sheen_b200.SceneArrays()
    v = s.view()
    # parameter checks run before any device call (api/sheen_c_api.cu:189-193)
    assert lib.sheen_render_scene(ctypes.addressof(v), 0, 10, 1, b"/tmp/x.png") == -1
    assert sheen_b200.last_error() == "bad render params"
    assert lib.sheen_render_scene(ctypes.addressof(v), 10, 10, 65, b"/tmp/x.png") == -1
    assert lib.sheen_render_scene(ctypes.addressof(v), 10, 10, 1, None) == -1
    assert lib.sheen_render_scene(ctypes.addressof(v), 10, 10, 1, b"/tmp/x.png") == -1
    assert sheen_b200.last_error() == "no materials"
    assert lib.sheen_render_scene(None, 10, 10, 1, b"/tmp/x.png") == -1
    assert sheen_b200.last_error() == "null scene"


def test_png_writer(tmp_path):
    img = np.zeros((3, 4, 4), np.float32)
    img[..., 0] = np.linspace(0, 1.2, 4)[None, :]
    img[..., 3] = 1
    p = tmp_path / "t.png"
    sheen_b200.write_png(str(p), img)
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    import zlib
    i = data.index(b"IDAT")
    n = int.from_bytes(data[i - 4:i], "big")
    raw = zlib.decompress(data[i + 4:i + 4 + n])
    row = np.frombuffer(raw[1:1 + 12], np.uint8).reshape(4, 3)
    # png_color.h:11-20: 0 -> 0, clamp above 1 -> 255, sRGB curve in between
    assert row[0, 0] == 0 and row[3, 0] == 255
    c = 0.4
    want = int((1.055 * c ** (1 / 2.4) - 0.055) * 255 + 0.5)
    assert abs(int(row[1, 0]) - want) <= 1


def _png_rows(path):
    """RGB8 pixels of a PNG written by this library (one IDAT, filter 0)."""
    import struct
    import zlib
    b = open(path, "rb").read()
    assert b[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(b):
        n = struct.unpack(">I", b[pos:pos + 4])[0]
        tag = b[pos + 4:pos + 8]
        data = b[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h = struct.unpack(">II", data[:8])
        elif tag == b"IDAT":
            idat += data
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert (raw[:, 0] == 0).all()
    return raw[:, 1:].reshape(h, w, 3)


def test_srgb_thresholds_are_the_host_conversion_steps(tmp_path):
    """At every threshold the host conversion steps up by one byte value, so
    counting thresholds reproduces it (the device packs that way)."""
    L = sheen_b200.lib()
    thr = np.zeros(255, np.float32)
    L.sheen_srgb_thresholds.argtypes = [ctypes.c_void_p]
    L.sheen_srgb_thresholds.restype = None
    L.sheen_srgb_thresholds(thr.ctypes.data)
    assert (np.diff(thr) > 0).all() and thr[-1] <= 1.0 and thr[0] > 0.0
    below = np.nextafter(thr, np.float32(-1.0))
    rng = np.random.default_rng(2)
    extra = np.r_[rng.random(5000).astype(np.float32), [0.0, -1.0, 1.0, 2.0, np.inf, np.nan, 1e-30]]
    vals = np.r_[thr, below, extra].astype(np.float32)
    n = len(vals)
    img = np.zeros((1, n, 4), np.float32)
    img[0, :, 0] = vals
    img[0, :, 1] = vals[::-1]
    img[0, :, 2] = vals
    p = str(tmp_path / "steps.png")
    L.sheen_write_png_srgb.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    assert L.sheen_write_png_srgb(p.encode(), img.ctypes.data, n, 1) == 0
    got = _png_rows(p)[0]
    def by_table(v):
        v = np.where(np.isnan(v) | (v <= 0), -1.0, v)
        return np.where(v > 0, np.searchsorted(thr, v, side="right"), 0).astype(np.uint8)
    assert np.array_equal(got[:, 0], by_table(vals))
    assert np.array_equal(got[:, 1], by_table(vals[::-1]))
    assert np.array_equal(got[:255, 0], np.arange(1, 256, dtype=np.uint8))   # each threshold: its byte
    assert np.array_equal(got[255:510, 0], np.arange(0, 255, dtype=np.uint8))  # one ulp below: the byte before


def test_contract_fixture_is_the_addons_layout(reference_tree):
    """golden/contract_scene.npz holds what the reference's ctypes contract
    (c_api_contract.py) builds for its scene: regenerated here byte for byte
    (pointer fields excepted, which hold this process's addresses)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_contract_fixture", os.path.join(os.path.dirname(__file__), "golden", "make_contract_fixture.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sc, keep = mod.build()
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "contract_scene.npz"))
    now = np.frombuffer(ctypes.string_at(ctypes.addressof(sc), ctypes.sizeof(sc)), np.uint8).copy()
    rec = f["scene_bytes"].copy()
    for k in f.files:
        if k.startswith("ptr_"):
            o = int(f[k])
            now[o:o + 8] = 0
            rec[o:o + 8] = 0
            arr = keep[k[4:]]
            assert bytes(f["arr_" + k[4:]]) == ctypes.string_at(ctypes.addressof(arr), ctypes.sizeof(arr))
    assert np.array_equal(now, rec)
    assert int(f["sizeof_HeightField"]) == 72 and int(f["sizeof_SheenScene"]) == 344
