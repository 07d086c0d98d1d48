"""Launch parameters of the wavefront form (sheen_tune_set / sheen_tune_get).

Every setting must give the same image: the shadow-stage variants only
schedule the same queries differently (32-ray batches per warp, or lanes
that take new rays as theirs finish), so images are compared bit for bit.
"""
import numpy as np
import pytest

import sheen_b200 as sb

DEFAULTS = {"wave.shadow_kernel": 1, "wave.refill_min": 8, "wave.shadow_blocks_per_sm": 0}


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
    for refill, per_sm in ((1, 0), (8, 0), (32, 0), (8, 1)):
        sb.tune_set("wave.refill_min", refill)
        sb.tune_set("wave.shadow_blocks_per_sm", per_sm)
        img, st = ds.render_host(W, H, spp, count_rays=True)
        assert np.array_equal(img, ref), (refill, per_sm, float(np.abs(img - ref).max()))
        assert st["total_rays"] == st0["total_rays"]
    ds.close()
    scene.close()
