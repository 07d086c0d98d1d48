"""The request loop (sheen_server_*): layout, host-side checks and, on a B200,
continuous batching.

Bars:
  - a request's image is bit-identical alone and in a mix of concurrent
    requests on several scenes (every sample's random numbers depend on its
    pixel, sample index and bounce only, and each in-flight request has its
    own queues), whatever the band size;
  - a request rendered by the server matches the same scene rendered by the
    resident-scene entry point of the same form: max absolute difference
    <= 1e-6 per channel (the same kernels over the same samples);
  - admission: with a budget that fits one request beside the scenes, no two
    requests are on the GPU at once and all complete; a request that can
    never fit is refused at submit.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

import sheen_b200 as sb
from sheen_b200 import serve

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_layout(structs):
    lines = ['#include "sheen_c_api.h"', "#include <stdio.h>", "#include <stddef.h>", "int main(void){"]
    for name, fields in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "p.c"), os.path.join(d, "p")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-w", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.strip().splitlines())}


def test_server_struct_layout_matches_header():
    types = {"SheenServerConfig": serve.ServerConfig, "SheenRequestInfo": serve.RequestInfo,
             "SheenServerStats": serve.ServerStats}
    got = _c_layout({n: [f for f, _ in t._fields_] for n, t in types.items()})
    for name, t in types.items():
        assert got[name] == ctypes.sizeof(t), name
        for f, _ in t._fields_:
            assert got[f"{name}.{f}"] == getattr(t, f).offset, (name, f)


def test_server_calls_reject_bad_handles():
    L = serve._lib()
    rid = ctypes.c_ulonglong()
    assert L.sheen_server_submit(None, 0, 16, 16, 1, None, ctypes.byref(rid)) == -1
    assert sb.last_error() == "unknown server handle"
    assert L.sheen_server_poll(12345, 1) == -1
    assert L.sheen_server_wait(12345, 1, 0.0, None) == -1
    assert L.sheen_server_remove_scene(None, 0) == -1
    L.sheen_server_destroy(None)     # unknown handles are ignored


def test_request_stream_is_seeded_and_in_range():
    a = serve.request_stream(64, 20.0, seed=3)
    b = serve.request_stream(64, 20.0, seed=3)
    assert a == b
    assert a[0]["t"] == 0.0
    assert all(x["t"] <= y["t"] for x, y in zip(a, a[1:]))
    for r in a:
        assert (r["width"], r["height"]) in serve.STREAM_RESOLUTIONS
        assert r["spp"] in serve.STREAM_SPP
        assert r["config"] in (0, 1, 2, 3)
    # mean inter-arrival time close to 1/rate
    s = serve.request_stream(4000, 20.0, seed=5)
    assert abs(s[-1]["t"] / 3999 - 0.05) < 0.005


# ---------------------------------------------------------------- GPU ----

def _scenes():
    """Small scenes of every generator: spheres, mesh (level-3 icosphere),
    analytic + CSG, and the caustic scene with a small photon map."""
    return [sb.generate_scene(0, 11), sb.generate_scene(1, 12, 3), sb.generate_scene(2, 13),
            sb.generate_scene(3, 14, 0, 20000)]


MIX = [  # (scene index, W, H, spp)
    (0, 160, 96, 1), (1, 200, 120, 4), (2, 128, 128, 4), (3, 96, 64, 16),
    (1, 96, 96, 1), (0, 250, 40, 4), (2, 64, 200, 1), (3, 120, 72, 4),
]


@pytest.mark.gpu
@pytest.mark.parametrize("form", [sb.FORM_WAVEFRONT, sb.FORM_PLAIN], ids=["wavefront", "plain"])
def test_same_alone_and_in_mix(form):
    sb.init(0, 100)
    scenes = _scenes()
    # Small bands so that most requests span several launches.
    with serve.Server(form=form, max_inflight=4, tile_samples=8192) as srv:
        ids = [srv.add_scene(s) for s in scenes]
        alone = []
        for si, W, H, spp in MIX:
            img, info = srv.submit(ids[si], W, H, spp).wait()
            assert info["status"] == serve.REQ_DONE and info["rays"] > 0
            alone.append(img.copy())
        reqs = [srv.submit(ids[si], W, H, spp) for si, W, H, spp in MIX]
        for k, r in enumerate(reqs):
            img, info = r.wait()
            assert np.isfinite(img).all()
            assert np.array_equal(img, alone[k]), (k, float(np.abs(img - alone[k]).max()))
        st = srv.stats()
        assert st["completed"] == 2 * len(MIX) and st["failed"] == 0
        assert st["inflight_peak"] >= 2      # the mix did overlap
    # Different band sizes give the same image.
    with serve.Server(form=form, max_inflight=2, tile_samples=1 << 22) as srv:
        sid = srv.add_scene(scenes[1])
        img, info = srv.submit(sid, 200, 120, 4).wait()
        assert info["tiles"] == 1
        assert np.array_equal(img, alone[1])
    for s in scenes:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", [sb.FORM_WAVEFRONT, sb.FORM_PLAIN], ids=["wavefront", "plain"])
def test_server_matches_resident_scene_render(form):
    sb.init(0, 100)
    scene = sb.generate_scene(1, 21, 3)
    ds = sb.DeviceScene(scene, form)
    ref, _ = ds.render_host(320, 200, 4)
    with serve.Server(form=form, tile_samples=20000) as srv:
        sid = srv.add_scene(scene)
        img, info = srv.submit(sid, 320, 200, 4).wait()
    assert info["tiles"] > 1
    assert float(np.abs(img - ref).max()) <= 1e-6
    ds.close()
    scene.close()


@pytest.mark.gpu
def test_admission_by_hbm_footprint():
    sb.init(0, 100)
    scene = sb.generate_scene(1, 31, 3)
    probe = serve.Server(max_inflight=4)
    sid = probe.add_scene(scene)
    img, info = probe.submit(sid, 256, 256, 4).wait()
    scene_bytes = probe.stats()["scene_bytes"]
    probe.close()
    # Room for the scene and one such request, not two.
    budget = scene_bytes + int(1.5 * info["hbm_bytes"])
    with serve.Server(max_inflight=4, hbm_budget=budget) as srv:
        sid = srv.add_scene(scene)
        reqs = [srv.submit(sid, 256, 256, 4) for _ in range(6)]
        for r in reqs:
            out, _ = r.wait()
            assert np.array_equal(out, img)
        st = srv.stats()
        assert st["completed"] == 6
        assert st["inflight_peak"] == 1
        assert st["hbm_peak"] <= budget
        # A request that could never fit is refused at once.
        with pytest.raises(RuntimeError, match="exceeds the server's HBM budget"):
            srv.submit(sid, 2048, 2048, 64)
    scene.close()


@pytest.mark.gpu
def test_remove_scene_and_shutdown():
    sb.init(0, 100)
    scene = sb.generate_scene(0, 41)
    srv = serve.Server(max_inflight=1)
    sid = srv.add_scene(scene)
    bytes0 = srv.stats()["scene_bytes"]
    assert bytes0 > 0
    reqs = [srv.submit(sid, 640, 480, 16) for _ in range(3)]
    srv.remove_scene(sid)                  # in use: freed after the last request
    with pytest.raises(RuntimeError, match="unknown scene id"):
        srv.submit(sid, 64, 64, 1)
    for r in reqs:
        r.wait()
    assert srv.stats()["scene_bytes"] == 0
    # Shutdown with queued work: pending requests fail, running ones finish.
    sid = srv.add_scene(scene)
    reqs = [srv.submit(sid, 640, 480, 64) for _ in range(4)]
    assert srv.stats()["pending"] >= 1     # one slot: the rest are queued
    srv.close()                            # returns once the running request is done
    assert serve._lib().sheen_server_poll(None, reqs[0].id) == -1
    scene.close()
