"""Parity of the CUDA renderer forms with the oracle (B200 only).

Bars:
  - per-pixel RGB (linear float4 before sRGB): mean absolute error <= 1e-3
    against the reference's render (committed golden fixtures rendered by
    the reference's own code) and against the oracle, with at most 1% of
    pixels off by more than 1e-2 (terminators and silhouettes);
  - primary-ray hits: identical (object id, material id) except on grazing
    hits whose t agrees to 1e-5 relative; hit-versus-miss disagreements
    (silhouettes) on at most 0.2% of samples;
  - hit distance against the FP64 oracle: maximum relative error reported,
    99% of samples within 1e-5.
Every call goes through the C-ABI of libsheen_c_api.so.
"""
import numpy as np
import pytest

import sheen_b200 as sb
from cases import CASES
from helpers import golden, load_case
from oracle_bindings import MISS, Oracle, RefHost, image_error

pytestmark = pytest.mark.gpu

FORMS = [sb.FORM_PLAIN, sb.FORM_WAVEFRONT]
FORM_IDS = ["plain", "wavefront"]


@pytest.fixture(scope="module", autouse=True)
def device():
    sb.init(0, 100)
    yield


def _hits(ds, W, H, aa):
    return ds.primary_hits(W, H, aa)


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_image_matches_reference(case, form):
    s = load_case(case)
    img, st = sb.render_rgba(s, case["W"], case["H"], case["aa"], form)
    assert np.isfinite(img).all()
    err = image_error(img, golden(case)["rgba"])
    assert err["mean_abs"] <= 1e-3, err
    assert err["frac_px_over_1e-2"] <= 0.01, err


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_image_matches_oracle(case, form):
    s = load_case(case)
    img, _ = sb.render_rgba(s, case["W"], case["H"], case["aa"], form)
    o = Oracle()
    ref = o.render(o.scene(s.view_ptr), case["W"], case["H"], case["aa"])
    err = image_error(img, ref)
    assert err["mean_abs"] <= 1e-3, err
    assert err["frac_px_over_1e-2"] <= 0.01, err


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("case", [c for c in CASES if c["name"] != "caustics_20k"],
                         ids=[c["name"] for c in CASES if c["name"] != "caustics_20k"])
def test_primary_hit_ids(case, form):
    s = load_case(case)
    ds = sb.DeviceScene(s, form)
    obj, mat, t = _hits(ds, case["W"], case["H"], case["aa"])
    g = golden(case)
    gobj, gmat, gt = g["obj"], g["mat"], g["t"]
    both = (obj != MISS) & (gobj != MISS)
    same = both & (obj == gobj) & (mat == gmat)
    rel = np.abs(t.astype(np.float64) - gt) / np.maximum(np.abs(gt), 1e-6)
    differ = both & ~same
    # A different primitive is allowed where the two distances agree (shared
    # edge, grazing hit); where they do not, one side grazed a silhouette
    # (a thin strand, a box edge) that the other missed: those count with the
    # hit-versus-miss samples against the silhouette budget.
    silhouette = (differ & (rel > 1e-5)) | ((obj != MISS) != (gobj != MISS))
    assert silhouette.mean() <= 0.002, (case["name"], int(silhouette.sum()))
    assert (same | (differ & (rel <= 1e-5))).sum() >= 0.99 * both.sum()
    ds.close()


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_hit_distance_vs_fp64_oracle(form):
    case = next(c for c in CASES if c["name"] == "mesh_l3")
    s = load_case(case)
    ds = sb.DeviceScene(s, form)
    obj, mat, t = _hits(ds, case["W"], case["H"], case["aa"])
    o64 = Oracle(fp64=True)
    cat, prim, t64 = o64.primary_hits(o64.scene(s.view_ptr), case["W"], case["H"], case["aa"])
    tri = (cat == 2) & (obj == -(prim + 1))
    rel = np.abs(t[tri] - t64[tri]) / t64[tri]
    print(f"max relative hit-t error vs FP64 oracle ({FORM_IDS[form]}): {rel.max():.3e}")
    assert tri.sum() > 100
    assert np.quantile(rel, 0.99) <= 1e-5 and rel.max() <= 2e-3
    ds.close()


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_deterministic_and_resident(form):
    case = next(c for c in CASES if c["name"] == "caustics_20k")
    s = load_case(case)
    a, st_a = sb.render_rgba(s, case["W"], case["H"], case["aa"], form)
    b, _ = sb.render_rgba(s, case["W"], case["H"], case["aa"], form)
    assert np.array_equal(a, b)           # photon map order is deterministic
    ds = sb.DeviceScene(s, form)
    c, st = ds.render_host(case["W"], case["H"], case["aa"], count_rays=True)
    assert np.array_equal(a, c)
    assert st["primary_rays"] == case["W"] * case["H"] * max(1, case["aa"])
    assert st["total_rays"] >= st["primary_rays"]
    ds.close()


def test_reused_buffers_do_not_leak_between_frames():
    """A resident wavefront scene reuses its queues and slots across frames;
    a frame must not read anything a previous frame of another shape left."""
    s = sb.generate_scene(0, 4)
    ds = sb.DeviceScene(s, sb.FORM_WAVEFRONT)
    ds.render_host(96, 72, 4)                 # fills the buffers
    a, _ = ds.render_host(64, 48, 1)          # smaller frame on the same buffers
    ds.close()
    b, _ = sb.render_rgba(s, 64, 48, 1, sb.FORM_WAVEFRONT)   # fresh buffers
    assert np.array_equal(a, b)


def test_forms_agree_on_rays_and_pixels():
    case = next(c for c in CASES if c["name"] == "mesh_l3")
    s = load_case(case)
    out = []
    for form in FORMS:
        ds = sb.DeviceScene(s, form)
        img, st = ds.render_host(case["W"], case["H"], case["aa"], count_rays=True)
        out.append((img, st))
        ds.close()
    (a, sa), (b, sb_) = out
    assert sa["primary_rays"] == sb_["primary_rays"]
    # both forms issue the reference's queries; ties at shared edges can move a glass pass
    assert abs(sa["total_rays"] - sb_["total_rays"]) <= 0.001 * sa["total_rays"]
    assert image_error(a, b)["mean_abs"] <= 1e-3


def test_full_size_workload_properties():
    """The headline workload at full size: 2,110,720 triangles, 1920x1080,
    4 spp.  Size-independent checks: finite non-negative pixels, alpha 1,
    the expected primary-ray count, both forms within the pixel bar of each
    other, and sampled rows against the reference's host build when present."""
    s = sb.generate_scene(1, 1, 8)
    W, H, aa = 1920, 1080, 4
    imgs = {}
    for form in FORMS:
        ds = sb.DeviceScene(s, form)
        img, st = ds.render_host(W, H, aa, count_rays=True)
        assert st["primary_rays"] == W * H * aa
        assert np.isfinite(img).all() and (img[..., :3] >= 0).all() and (img[..., 3] == 1).all()
        imgs[form] = img
        ds.close()
    assert image_error(imgs[0], imgs[1])["mean_abs"] <= 1e-3
    if RefHost.available():
        ref = RefHost()
        h = ref.scene(s.view_ptr)
        rows = ref.render(h, W, H, aa, 0, 30, 32)   # block rows 30..31 (pixel rows 480..511)
        err = image_error(rows[480:512], imgs[0][480:512])
        assert err["mean_abs"] <= 1e-3, err


def test_c_api_png(tmp_path):
    """The drop-in PNG call packs sRGB on the device; its pixels are exactly
    the host conversion (png_color.h:11-20) of the same render."""
    from test_abi import _png_rows
    s = sb.generate_scene(0, 1)
    p = tmp_path / "spheres.png"
    sb.render_scene(s, 160, 120, 1, str(p))
    assert p.read_bytes()[:8] == b"\x89PNG\r\n\x1a\n"
    img, _ = sb.render_rgba(s, 160, 120, 1, sb.FORM_PLAIN)
    q = tmp_path / "host.png"
    sb.write_png(str(q), img)
    assert np.array_equal(_png_rows(str(p)), _png_rows(str(q)))
    with pytest.raises(RuntimeError, match="bad render params"):
        sb.render_scene(s, 160, 120, 0, str(p))
