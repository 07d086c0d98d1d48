"""Reflect + refract recursion (SheenSceneExt.max_depth; an extension with no
counterpart in the reference, whose mirror ray stops at depth 1).

The mesh workload's extended form (config 1: its tori instanced, max_depth
4; every surface but the glass reflects 0.2, the glass tori refract) is
rendered by both renderer forms and compared with the oracle's restatement
of the same rules (oracle/sheen_oracle.c, render_deep).  The depth-1
baseline is the same extension with max_depth 0.

CPU: the ctypes view of SheenSceneExt against the C header, the range check
on max_depth (run before any device call), and properties of the oracle's
recursion -- depth 1 is the reference's path bit for bit, sky pixels keep
their colour, deeper paths change the image, FP32 and FP64 agree.
GPU: images and ray counts against the oracle, depth 1 equal to depth 0,
batch jobs of such scenes equal to their single renders.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

import sheen_b200 as sb
from sheen_b200 import contract as C
from oracle_bindings import Oracle, image_error

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FORMS = [sb.FORM_PLAIN, sb.FORM_WAVEFRONT]
FORM_IDS = ["plain", "wavefront"]
W, H, AA = 96, 54, 2


@pytest.fixture(scope="module")
def deep_scene():
    return sb.generate_scene(1, 3, 3, extended=True)


def _ext(scene, max_depth):
    x = C.SheenSceneExt.from_buffer_copy(ctypes.string_at(scene.ext_ptr, ctypes.sizeof(C.SheenSceneExt)))
    x.max_depth = max_depth
    return x


def _oracle_render(scene, ext, fp64=False, w=W, h=H, aa=AA):
    o = Oracle(fp64=fp64)
    hd = o.scene(scene.view_ptr, ext_ptr=ctypes.addressof(ext) if ext is not None else None)
    img = o.render(hd, w, h, aa)
    hd.close()
    return img


# ------------------------------------------------------------------ CPU


def test_ext_ctypes_layout_matches_header():
    fields = [f for f, _ in C.SheenSceneExt._fields_]
    lines = ['#include "sheen_c_api.h"', "#include <stdio.h>", "#include <stddef.h>", "int main(void){",
             'printf("size %zu\\n", sizeof(SheenSceneExt));']
    lines += [f'printf("{f} %zu\\n", offsetof(SheenSceneExt, {f}));' for f in fields]
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "p.c"), os.path.join(d, "p")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-w", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = {k: int(v) for k, v in (ln.split() for ln in out.strip().splitlines())}
    assert got["size"] == ctypes.sizeof(C.SheenSceneExt)
    for f in fields:
        assert got[f] == getattr(C.SheenSceneExt, f).offset, f


def test_generator_sets_depth_four(deep_scene):
    assert _ext(deep_scene, 4).max_depth == 4
    x = C.SheenSceneExt.from_buffer_copy(ctypes.string_at(deep_scene.ext_ptr, ctypes.sizeof(C.SheenSceneExt)))
    assert x.max_depth == 4
    plain = sb.generate_scene(1, 3, 3)
    assert ctypes.string_at(plain.view.triangles, 64) == ctypes.string_at(deep_scene.view.triangles, 64)


@pytest.mark.parametrize("depth", [-1, 9, 1000])
def test_depth_outside_range_is_refused(deep_scene, depth):
    L = sb.lib()
    L.sheen_scene_create_ext.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p)]
    L.sheen_scene_create_ext.restype = ctypes.c_int
    h = ctypes.c_void_p()
    x = _ext(deep_scene, depth)
    rc = L.sheen_scene_create_ext(deep_scene.view_ptr, ctypes.addressof(x), sb.FORM_WAVEFRONT, ctypes.byref(h))
    assert rc == -1 and "max_depth outside 0..8" in sb.last_error()


def test_oracle_depth_one_is_the_reference_path(deep_scene):
    base = _oracle_render(deep_scene, _ext(deep_scene, 0), w=64, h=36, aa=1)
    one = _oracle_render(deep_scene, _ext(deep_scene, 1), w=64, h=36, aa=1)
    assert np.array_equal(base, one)


def test_oracle_recursion_changes_bouncing_pixels_only(deep_scene):
    w, h = 64, 36
    base = _oracle_render(deep_scene, _ext(deep_scene, 0), w=w, h=h, aa=1)
    deep = _oracle_render(deep_scene, _ext(deep_scene, 4), w=w, h=h, aa=1)
    o = Oracle()
    x0 = _ext(deep_scene, 0)
    hd = o.scene(deep_scene.view_ptr, ext_ptr=ctypes.addressof(x0))
    cat, _, _ = o.primary_hits(hd, w, h, 1)
    hd.close()
    sky = (cat.reshape(h, w) < 0)
    assert sky.any() and (~sky).any()
    # a primary miss has no children: its colour is the sky's in both
    assert np.array_equal(deep[sky], base[sky])
    # a hit whose mirror ray leaves for the sky (most of the ground) ends at
    # depth 1 in both; the others gather a second bounce (weight 0.2 x 0.2
    # on the reflective surfaces, the full transmission through the glass)
    diff = np.abs(deep - base)[..., :3].max(axis=-1)
    assert (diff[~sky] > 1e-4).mean() > 0.1 and diff.max() > 1e-2
    assert np.isfinite(deep).all()


def test_oracle_recursion_fp32_matches_fp64(deep_scene):
    a = _oracle_render(deep_scene, _ext(deep_scene, 4), w=64, h=36, aa=1)
    b = _oracle_render(deep_scene, _ext(deep_scene, 4), fp64=True, w=64, h=36, aa=1)
    err = image_error(a, b)
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.02, err


# ------------------------------------------------------------------ GPU


@pytest.fixture(scope="module")
def device():
    sb.init(0, 100)
    yield


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("depth", [2, 4, 8])
def test_recursion_matches_oracle(device, deep_scene, form, depth):
    x = _ext(deep_scene, depth)
    ds = sb.DeviceScene(deep_scene, form, ext=x)
    img, st = ds.render_host(W, H, AA, count_rays=True)
    ds.close()
    ref = _oracle_render(deep_scene, x)
    err = image_error(img, ref)
    assert st["primary_rays"] == W * H * AA
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.01, err
    base, _ = sb.DeviceScene(deep_scene, form, ext=_ext(deep_scene, 0)).render_host(W, H, AA)
    assert image_error(img, base)["mean_abs"] > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_recursion_ray_count_matches_oracle(device, deep_scene, form):
    import torch
    x = _ext(deep_scene, 4)
    ds = sb.DeviceScene(deep_scene, form, ext=x)
    out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    st = ds.render_region(W, H, AA, 0, 0, W, H, out.data_ptr(), 0, count_rays=True)
    torch.cuda.synchronize()
    ds.close()
    o = Oracle()
    hd = o.scene(deep_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    _, queries = o.render_region(hd, W, H, AA, 0, 0, W, H)
    hd.close()
    assert abs(st["total_rays"] - queries) <= max(2, 1e-3 * queries), (st, queries)
    # more secondary rays than the reference's depth-1 rules issue
    base = sb.DeviceScene(deep_scene, form, ext=_ext(deep_scene, 0))
    bst = base.render_region(W, H, AA, 0, 0, W, H, out.data_ptr(), 0, count_rays=True)
    torch.cuda.synchronize()
    base.close()
    assert st["total_rays"] > bst["total_rays"]


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_depth_one_equals_depth_zero(device, deep_scene, form):
    a, _ = sb.DeviceScene(deep_scene, form, ext=_ext(deep_scene, 0)).render_host(64, 36, 1)
    b, _ = sb.DeviceScene(deep_scene, form, ext=_ext(deep_scene, 1)).render_host(64, 36, 1)
    assert np.array_equal(a, b)


@pytest.mark.gpu
def test_frame_path_reports_the_megakernel(device, deep_scene):
    deep = sb.DeviceScene(deep_scene, sb.FORM_WAVEFRONT, ext=_ext(deep_scene, 4))
    flat = sb.DeviceScene(deep_scene, sb.FORM_WAVEFRONT, ext=_ext(deep_scene, 0))
    plain = sb.DeviceScene(deep_scene, sb.FORM_PLAIN, ext=_ext(deep_scene, 4))
    assert deep.frame_path(1920, 1080, 4) == sb.PATH_MEGAKERNEL
    assert flat.frame_path(1920, 1080, 4) == sb.PATH_QUEUES
    assert plain.frame_path(1920, 1080, 4) == sb.PATH_PLAIN
    with pytest.raises(RuntimeError):
        flat.frame_path(0, 1080, 4)
    for d in (deep, flat, plain):
        d.close()


@pytest.mark.gpu
def test_batch_renders_recursion_scenes_alone(device, deep_scene):
    import torch
    deep = sb.DeviceScene(deep_scene, sb.FORM_WAVEFRONT, ext=_ext(deep_scene, 4))
    flat = sb.DeviceScene(deep_scene, sb.FORM_WAVEFRONT, ext=_ext(deep_scene, 0))
    outs = [torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    sb.render_batch([(deep, W, H, AA, None, outs[0].data_ptr()), (flat, W, H, AA, None, outs[1].data_ptr())])
    torch.cuda.synchronize()
    a, _ = deep.render_host(W, H, AA)
    b, _ = flat.render_host(W, H, AA)
    deep.close()
    flat.close()
    assert np.array_equal(outs[0].cpu().numpy(), a)
    assert np.array_equal(outs[1].cpu().numpy(), b)
