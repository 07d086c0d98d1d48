"""Launch parameters of the wavefront form (sheen_tune_set / sheen_tune_get).

Every queue-pipeline setting must give the same image: the shadow-stage
variants only schedule the same queries differently (32-ray batches per
warp, or lanes that take new rays as theirs finish) and the pixel tile only
changes the order in which samples are taken, so images are compared bit
for bit.  The small-frame switch (wave.mega_samples) runs the same queries
in the BVH4 megakernel, whose separately compiled shading agrees to 1e-5.
"""
import ctypes
import json

import numpy as np
import pytest

import sheen_b200 as sb

DEFAULTS = {"wave.shadow_kernel": 1, "wave.refill_min": 16, "wave.shadow_blocks_per_sm": 0, "wave.shadow_stack": 0,
            "wave.inner_min": 10, "wave.tile_w": 16, "wave.mega_samples": 327680}


@pytest.fixture
def restore_tuning():
    yield
    for k, v in DEFAULTS.items():
        sb.tune_set(k, v)


def test_keys_defaults_and_ranges(restore_tuning):
    assert set(sb.TUNE_KEYS) == set(DEFAULTS)
    for k, v in DEFAULTS.items():
        assert sb.tune_get(k) == v
    sb.tune_set("wave.refill_min", 32)
    assert sb.tune_get("wave.refill_min") == 32
    with pytest.raises(RuntimeError, match="out of range"):
        sb.tune_set("wave.refill_min", 0)
    with pytest.raises(RuntimeError, match="out of range"):
        sb.tune_set("wave.shadow_kernel", 2)
    with pytest.raises(RuntimeError, match="unknown tuning key"):
        sb.tune_set("wave.nope", 1)
    with pytest.raises(RuntimeError, match="unknown tuning key"):
        sb.tune_get("wave.nope")


SCENES = [(0, 3, 0, 0, 1), (1, 4, 3, 0, 4), (2, 5, 0, 0, 2), (3, 6, 0, 20000, 4)]   # config, seed, detail, photons, spp


@pytest.mark.gpu
@pytest.mark.parametrize("config,seed,detail,photons,spp", SCENES, ids=["spheres", "mesh", "analytic", "caustics"])
def test_shadow_variants_give_identical_images(config, seed, detail, photons, spp, restore_tuning):
    sb.init(0, 100)
    scene = sb.generate_scene(config, seed, detail, photons)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    W, H = 240, 136
    sb.tune_set("wave.shadow_kernel", 0)
    ref, st0 = ds.render_host(W, H, spp, count_rays=True)
    assert np.isfinite(ref).all()
    sb.tune_set("wave.shadow_kernel", 1)
    for refill, per_sm, stack, inner in ((1, 0, 0, 0), (8, 0, 0, 0), (32, 0, 0, 0), (8, 1, 0, 0), (8, 0, 1, 0),
                                         (1, 0, 1, 0), (24, 2, 1, 0), (16, 0, 0, 10), (16, 0, 1, 10), (1, 0, 0, 32),
                                         (32, 0, 0, 1), (8, 1, 1, 20)):
        sb.tune_set("wave.refill_min", refill)
        sb.tune_set("wave.shadow_blocks_per_sm", per_sm)
        sb.tune_set("wave.shadow_stack", stack)
        sb.tune_set("wave.inner_min", inner)
        img, st = ds.render_host(W, H, spp, count_rays=True)
        assert np.array_equal(img, ref), (refill, per_sm, stack, inner, float(np.abs(img - ref).max()))
        assert st["total_rays"] == st0["total_rays"]
    for tw in (8, 32, 16):    # pixel tiles 8x16, 32x4 and back to 16x8
        sb.tune_set("wave.tile_w", tw)
        img, st = ds.render_host(W, H, spp, count_rays=True)
        assert np.array_equal(img, ref), (tw, float(np.abs(img - ref).max()))
        assert st["total_rays"] == st0["total_rays"]
    with pytest.raises(RuntimeError, match="8, 16 or 32"):
        sb.tune_set("wave.tile_w", 12)
    ds.close()
    scene.close()


def test_autotune_rejects_bad_calls():
    L = sb.lib()
    L.sheen_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(sb.TuneResult)]
    L.sheen_autotune.restype = ctypes.c_int
    r = sb.TuneResult()
    assert L.sheen_autotune(None, 64, 64, 1, 1, ctypes.byref(r)) == -1
    assert sb.last_error() == "null scene or result"


def test_autotune_cache_hit_applies_without_timing(tmp_path, restore_tuning):
    class FakeScene:          # a cache hit never touches the scene
        device_bytes = 123
        handle = None
    cache = tmp_path / "tune.json"
    key = "k1"
    cache.write_text(json.dumps({key: {"wave.shadow_kernel": 0, "wave.refill_min": 16,
                                       "wave.shadow_blocks_per_sm": 2, "best_ms": 1.0}}))
    res = sb.autotune(FakeScene(), 64, 64, 1, cache=str(cache), key=key)
    assert res["cached"] is True
    assert sb.tune_get("wave.shadow_kernel") == 0
    assert sb.tune_get("wave.refill_min") == 16
    assert sb.tune_get("wave.shadow_blocks_per_sm") == 2


@pytest.mark.gpu
def test_autotune_keeps_a_setting_no_slower_than_default(tmp_path, restore_tuning):
    sb.init(0, 100)
    scene = sb.generate_scene(1, 8, 4)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    ref, _ = ds.render_host(320, 180, 4)
    cache = str(tmp_path / "tune.json")
    res = sb.autotune(ds, 320, 180, 4, reps=2, cache=cache)
    assert res["cached"] is False and res["candidates"] >= 2
    assert res["best_ms"] <= res["default_ms"]
    for k in sb.TUNE_KEYS:
        assert sb.tune_get(k) == res[k]
    img, _ = ds.render_host(320, 180, 4)
    if res["wave.mega_samples"] == 0 or 320 * 184 * 4 > res["wave.mega_samples"] // 4:
        assert np.array_equal(img, ref)       # queue stages: any tile, any shadow setting
    else:
        assert np.abs(img - ref).mean() <= 1e-5
    again = sb.autotune(ds, 320, 180, 4, cache=cache)
    assert again["cached"] is True
    ds.close()
    scene.close()
