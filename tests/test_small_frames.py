"""Small frames of the wavefront form run on the BVH4 megakernel (B200 only).

Below wave.mega_samples samples (tile-padded pixels x spp; a quarter of it
for scenes with triangles) one megakernel launch replaces the eight queue
stages, whose fixed cost dominates such frames.  Checks: the default rule
picks the megakernel for the 640x480 1-spp spheres frame and the queue
stages for a 640x480 frame of the mesh scene; the megakernel's images meet
the parity bars against the reference's render (the committed golden
fixtures) and agree with the queue pipeline's to 1e-5.
"""
import numpy as np
import pytest

import sheen_b200 as sb
from cases import CASES
from helpers import golden, load_case
from oracle_bindings import image_error

pytestmark = [pytest.mark.gpu, pytest.mark.small_frames]


@pytest.fixture(scope="module", autouse=True)
def device():
    sb.init(0, 100)
    yield


def _render(ds, W, H, aa, mega):
    old = sb.tune_get("wave.mega_samples")
    if mega is not None:
        sb.tune_set("wave.mega_samples", (1 << 30) if mega else 0)
    try:
        img, _ = ds.render_host(W, H, aa)
    finally:
        sb.tune_set("wave.mega_samples", old)
    return img


def test_default_rule_picks_the_megakernel_for_small_frames():
    assert sb.tune_get("wave.mega_samples") == 327680
    spheres = sb.DeviceScene(sb.generate_scene(0, 1), sb.FORM_WAVEFRONT)
    assert spheres.frame_path(640, 480, 1) == sb.PATH_MEGAKERNEL
    assert spheres.frame_path(1920, 1080, 1) == sb.PATH_QUEUES
    d = _render(spheres, 640, 480, 1, None)
    assert np.array_equal(d, _render(spheres, 640, 480, 1, True))
    spheres.close()
    mesh = sb.DeviceScene(sb.generate_scene(1, 1, 4), sb.FORM_WAVEFRONT)
    assert mesh.frame_path(640, 480, 1) == sb.PATH_QUEUES
    assert mesh.frame_path(320, 240, 1) == sb.PATH_MEGAKERNEL
    d = _render(mesh, 640, 480, 1, None)           # 307200 samples > 327680 / 4
    assert np.array_equal(d, _render(mesh, 640, 480, 1, False))
    d = _render(mesh, 320, 240, 1, None)           # 76800 samples <= 81920
    assert np.array_equal(d, _render(mesh, 320, 240, 1, True))
    mesh.close()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_megakernel_matches_reference_and_queue_pipeline(case):
    s = load_case(case)
    ds = sb.DeviceScene(s, sb.FORM_WAVEFRONT)
    W, H, aa = case["W"], case["H"], case["aa"]
    mega = _render(ds, W, H, aa, True)
    queue = _render(ds, W, H, aa, False)
    ds.close()
    err = image_error(mega, golden(case)["rgba"])
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.01, err
    assert image_error(mega, queue)["mean_abs"] <= 1e-5


def test_full_spheres_frame_matches_reference():
    """The 640x480 1-spp spheres workload, rendered by the default rule (the
    megakernel), against the reference's host build over the whole frame."""
    from bench import quiet_stdout
    from oracle_bindings import RefHost
    assert RefHost.available(), "oracle/_ref/libsheen_ref_host.so is not built"
    scene = sb.generate_scene(0, 1)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    img = _render(ds, 640, 480, 1, None)
    ds.close()
    ref = RefHost()
    with quiet_stdout():
        h = ref.scene(scene.view_ptr)
        r = ref.render(h, 640, 480, 1)
    h.close()
    err = image_error(img, r)
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.01, err
