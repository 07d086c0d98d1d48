"""Host-side paths around a frame: the first frame of a shape launched
directly and later ones replayed from a captured CUDA graph, and images
read back into pageable host memory through the pinned ring."""
import numpy as np
import pytest

import sheen_b200 as sb


@pytest.mark.gpu
def test_direct_and_graph_frames_identical():
    """The first frame of a shape is launched directly, the second captured
    and replayed, the third replayed: the same image bit for bit."""
    import torch
    sb.init(0, 100)
    scene = sb.generate_scene(1, 12, 3)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    W, H, spp = 320, 200, 2
    imgs = []
    for _ in range(3):
        out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        ds.render_device(W, H, spp, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        imgs.append(out.cpu())
    # a new shape between, then the first shape again (still captured)
    out = torch.zeros((100, 160, 4), dtype=torch.float32, device="cuda")
    ds.render_device(160, 100, spp, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    ds.render_device(W, H, spp, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    imgs.append(out.cpu())
    ds.close()
    for img in imgs[1:]:
        assert torch.equal(img, imgs[0])


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(1024, 1024), (1000, 777)])
def test_pageable_readback_through_ring(W, H):
    """Images of 8 MB or more read into pageable memory go through the
    pinned ring (several threads, 4 MB chunks, a ragged last chunk): the
    same bytes as the device image."""
    import torch
    sb.init(0, 100)
    scene = sb.generate_scene(0, 3, 0)
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT)
    host, _ = ds.render_host(W, H, 1)
    assert host.nbytes >= 8 << 20
    dev = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    ds.render_device(W, H, 1, dev.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ds.close()
    assert np.array_equal(host, dev.cpu().numpy())
    assert np.isfinite(host).all() and host.any()


@pytest.mark.gpu
def test_kept_queue_block_reused_across_scenes():
    """A released scene's queue block is kept and handed to the next scene
    that fits (other lights, a smaller frame): images equal those rendered
    with freshly allocated blocks (mem.pool_keep_mb 0 keeps nothing)."""
    sb.init(0, 100)
    a = sb.generate_scene(1, 21, 3)        # 4 lights
    b = sb.generate_scene(0, 22, 0)        # spheres, other lights
    shapes = [(a, 320, 200, 2), (b, 256, 128, 1), (a, 160, 100, 4), (b, 320, 200, 2)]

    def run():
        imgs = []
        for sc, W, H, spp in shapes:
            ds = sb.DeviceScene(sc, sb.FORM_WAVEFRONT)
            img, _ = ds.render_host(W, H, spp)
            img2, _ = ds.render_host(W, H, spp)   # the captured graph over the same block
            assert np.array_equal(img, img2)
            ds.close()
            imgs.append(img)
        return imgs

    kept = run()
    sb.tune_set("mem.pool_keep_mb", 0)
    try:
        fresh = run()
    finally:
        sb.tune_set("mem.pool_keep_mb", 16384)
    for k, f in zip(kept, fresh):
        assert np.array_equal(k, f)
