"""Many tiles, frames and scenes in one pass of the wavefront queue kernels
(sheen_render_batch).

Every sample of a batched job runs the same code on the same inputs as when
the job is rendered alone.  The batch and single-frame kernels are separate
compiled instances, and the compiler may fuse a multiply and an add in one
and not the other, so a pixel can differ in its last bits; rarely such a
difference moves a shadow-ray origin across an edge.  The bar (BATCH_TOL):
mean absolute difference <= 1e-6, at most 0.1% of pixels off by more than
1e-4, none by more than 2e-2.  Jobs run under the kernel variant their
scene would use alone (the triangle/sphere/plane variant or the full one),
so mixing scenes never changes which variant renders a job.
"""
import numpy as np
import pytest

import sheen_b200 as sb


def _close(a, b):
    d = np.abs(a - b)
    return {"mean": float(d.mean()), "frac_1e4": float((d.max(-1) > 1e-4).mean()), "max": float(d.max()),
            "exact": bool(np.array_equal(a, b))}


def _assert_batch_tol(a, b, what):
    e = _close(a, b)
    assert e["mean"] <= 1e-6 and e["frac_1e4"] <= 1e-3 and e["max"] <= 2e-2, (what, e)
    return e


def _uneven_tiles(W, H, n, seed):
    """n rectangles covering a W x H frame: rows of uneven height, each cut
    into tiles of uneven width."""
    rng = np.random.default_rng(seed)
    rows = int(np.sqrt(n))
    cols = [n // rows + (1 if r < n % rows else 0) for r in range(rows)]
    ys = np.sort(rng.choice(np.arange(1, H), rows - 1, replace=False)).tolist()
    ys = [0] + ys + [H]
    tiles = []
    for r in range(rows):
        xs = np.sort(rng.choice(np.arange(1, W), cols[r] - 1, replace=False)).tolist()
        xs = [0] + xs + [W]
        for c in range(cols[r]):
            tiles.append((xs[c], ys[r], xs[c + 1], ys[r + 1]))
    return tiles


def test_uneven_tiles_cover_the_frame():
    for n in (1, 7, 16, 64):
        tiles = _uneven_tiles(320, 200, n, n)
        assert len(tiles) == n
        cover = np.zeros((200, 320), np.int32)
        for x0, y0, x1, y1 in tiles:
            assert 0 <= x0 < x1 <= 320 and 0 <= y0 < y1 <= 200
            cover[y0:y1, x0:x1] += 1
        assert (cover == 1).all()


@pytest.mark.gpu
@pytest.mark.parametrize("config,detail,photons,spp,ntiles", [(1, 4, 0, 2, 16), (3, 0, 20000, 4, 64), (2, 0, 0, 1, 7)],
                         ids=["mesh-16", "caustics-64", "analytic-7"])
def test_tiles_in_one_batch_equal_the_frame(config, detail, photons, spp, ntiles):
    import torch
    sb.init(0, 100)
    scene = sb.generate_scene(config, 3, detail, photons)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    W, H = 320, 200
    ref = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    st_ref = ds.render_device(W, H, spp, ref.data_ptr(), count_rays=True)
    out = torch.full((H, W, 4), -1.0, dtype=torch.float32, device="cuda")
    tiles = _uneven_tiles(W, H, ntiles, 11)
    st = sb.render_batch([(ds, W, H, spp, t, out.data_ptr()) for t in tiles], stats=True)
    torch.cuda.synchronize()
    a, b = out.cpu().numpy(), ref.cpu().numpy()
    assert (a[..., 3] == 1.0).all()          # every pixel written by exactly the tiles
    e = _assert_batch_tol(a, b, (config, ntiles))
    print(f"tiles {ntiles}: {e}")
    assert st["total_rays"] == st_ref["total_rays"]
    ds.close()


@pytest.mark.gpu
def test_mixed_scenes_and_shapes_equal_each_alone():
    import torch
    sb.init(0, 100)
    specs = [((0, 2, 0, 0), 160, 120, 1), ((1, 5, 4, 0), 240, 136, 4), ((3, 4, 0, 20000), 200, 200, 2),
             ((2, 6, 0, 0), 96, 64, 3), ((1, 5, 4, 0), 64, 48, 9)]
    scenes, jobs, refs, outs = [], [], [], []
    for (cfg, seed, detail, photons), W, H, spp in specs:
        sc = sb.generate_scene(cfg, seed, detail, photons)
        ds = sb.DeviceScene(sc, sb.FORM_WAVEFRONT)
        scenes.append((sc, ds))
        ref = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        ds.render_device(W, H, spp, ref.data_ptr())
        refs.append(ref)
        out = torch.full((H, W, 4), -1.0, dtype=torch.float32, device="cuda")
        outs.append(out)
        jobs.append((ds, W, H, spp, None, out.data_ptr()))
    # the same scene twice in one batch, and a plain-form job beside them
    sc_plain = sb.generate_scene(0, 9, 0, 0)
    ds_plain = sb.DeviceScene(sc_plain, sb.FORM_PLAIN)
    ref_p = torch.zeros((100, 120, 4), dtype=torch.float32, device="cuda")
    ds_plain.render_device(120, 100, 2, ref_p.data_ptr())
    out_p = torch.zeros_like(ref_p)
    jobs.append((ds_plain, 120, 100, 2, None, out_p.data_ptr()))
    sb.render_batch(jobs)
    torch.cuda.synchronize()
    for k, (o, r) in enumerate(zip(outs + [out_p], refs + [ref_p])):
        a, b = o.cpu().numpy(), r.cpu().numpy()
        if k == len(outs):
            assert np.array_equal(a, b)        # the plain-form job runs its own kernel, alone
        else:
            print(f"job {k}: {_assert_batch_tol(a, b, k)}")
    for sc, ds in scenes:
        ds.close()
    ds_plain.close()


def test_batch_rejects_bad_jobs():
    L = sb.lib()
    import ctypes
    assert L.sheen_render_batch(None, 1, None, None) == -1
    arr = (sb.BatchJob * 1)()
    arr[0] = sb.BatchJob(None, 64, 64, 1, 0, 0, 0, 0, None)
    assert L.sheen_render_batch(arr, 1, None, None) == -1
    assert "null scene" in sb.last_error()
    assert L.sheen_render_batch(arr, 0, None, None) == 0
