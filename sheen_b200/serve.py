"""Request loop (continuous batching) over the C-ABI's sheen_server_* calls.

The reference has no serving path: each ``sheen_render_scene`` call rebuilds
and re-uploads its scene and renders one frame (api/sheen_c_api.cu:187-361).
A :class:`Server` keeps scenes resident on the device and renders requests of
any resolution and sample count as they arrive; requests are admitted onto
the GPU by free slot and HBM footprint and overlap there with the ones
already running.

    srv = Server(max_inflight=4)
    sid = srv.add_scene(sheen_b200.generate_scene(1, seed=7))
    req = srv.submit(sid, 1920, 1080, 4)      # returns at once
    img, info = req.wait()                     # (H, W, 4) float32, dict
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import FORM_WAVEFRONT, _check, _scene_ptr, lib, last_error

REQ_PENDING, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class ServerConfig(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int), ("max_inflight", ctypes.c_int),
                ("hbm_budget", ctypes.c_ulonglong), ("tile_samples", ctypes.c_longlong)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("scene_id", ctypes.c_int), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("aa_samples", ctypes.c_int), ("tiles", ctypes.c_int),
                ("rays", ctypes.c_ulonglong), ("hbm_bytes", ctypes.c_ulonglong),
                ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("error", ctypes.c_char * 128)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["error"] = self.error.decode("utf-8", "replace")
        return d


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_ulonglong), ("completed", ctypes.c_ulonglong),
                ("failed", ctypes.c_ulonglong), ("rays", ctypes.c_ulonglong),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("busy_ms", ctypes.c_double), ("hbm_budget", ctypes.c_ulonglong),
                ("hbm_used", ctypes.c_ulonglong), ("hbm_peak", ctypes.c_ulonglong),
                ("scene_bytes", ctypes.c_ulonglong), ("inflight_peak", ctypes.c_int),
                ("inflight", ctypes.c_int), ("pending", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        P, I = ctypes.c_void_p, ctypes.c_int
        U64 = ctypes.c_ulonglong
        L.sheen_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(P)]
        L.sheen_server_create.restype = I
        L.sheen_server_destroy.argtypes = [P]
        L.sheen_server_destroy.restype = None
        L.sheen_server_add_scene.argtypes = [P, P, ctypes.POINTER(I)]
        L.sheen_server_add_scene.restype = I
        L.sheen_server_remove_scene.argtypes = [P, I]
        L.sheen_server_remove_scene.restype = I
        L.sheen_server_submit.argtypes = [P, I, I, I, I, P, ctypes.POINTER(U64)]
        L.sheen_server_submit.restype = I
        L.sheen_server_poll.argtypes = [P, U64]
        L.sheen_server_poll.restype = I
        L.sheen_server_wait.argtypes = [P, U64, ctypes.c_double, ctypes.POINTER(RequestInfo)]
        L.sheen_server_wait.restype = I
        L.sheen_server_stats.argtypes = [P, ctypes.POINTER(ServerStats)]
        L.sheen_server_stats.restype = I
        _bound = True
    return L


class Request:
    """A submitted request; owns the host buffer its image is written into."""

    def __init__(self, server, rid, image):
        self.server = server
        self.id = rid
        self.image = image
        self.info = None

    def poll(self) -> int:
        if self.info is not None:
            return self.info["status"]
        rc = _lib().sheen_server_poll(self.server.handle, self.id)
        if rc < 0:
            raise RuntimeError(last_error())
        return rc

    def wait(self, timeout_ms: float = -1.0):
        """(image, info) once finished; None on timeout.  A failed request
        raises RuntimeError with its error text."""
        if self.info is None:
            info = RequestInfo()
            rc = _lib().sheen_server_wait(self.server.handle, self.id, float(timeout_ms), ctypes.byref(info))
            if rc < 0:
                raise RuntimeError(last_error())
            if rc == 0:
                return None
            self.info = info.as_dict()
            self.server._live.pop(self.id, None)
        if self.info["status"] != REQ_DONE:
            raise RuntimeError(self.info["error"] or "request failed")
        return self.image, self.info


class Server:
    """sheen_server_* handle.  form: FORM_WAVEFRONT or FORM_PLAIN; hbm_budget
    in bytes (0: 90% of free device memory); tile_samples per band of rows."""

    def __init__(self, form: int = FORM_WAVEFRONT, max_inflight: int = 4, hbm_budget: int = 0,
                 tile_samples: int = 0):
        cfg = ServerConfig(form, max_inflight, hbm_budget, tile_samples)
        h = ctypes.c_void_p()
        self._live = {}
        self.handle = None
        _check(_lib().sheen_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h.value

    def add_scene(self, scene) -> int:
        ptr, keep = _scene_ptr(scene)
        sid = ctypes.c_int()
        _check(_lib().sheen_server_add_scene(self.handle, ptr, ctypes.byref(sid)))
        del keep
        return sid.value

    def remove_scene(self, scene_id: int) -> None:
        _check(_lib().sheen_server_remove_scene(self.handle, scene_id))

    def submit(self, scene_id: int, width: int, height: int, aa: int) -> Request:
        image = np.empty((height, width, 4), np.float32)
        rid = ctypes.c_ulonglong()
        _check(_lib().sheen_server_submit(self.handle, scene_id, width, height, aa, image.ctypes.data,
                                          ctypes.byref(rid)))
        req = Request(self, rid.value, image)
        # The library writes into `image` when the request completes: keep it
        # alive until then even if the caller drops the Request.
        self._live[rid.value] = image
        return req

    def stats(self) -> dict:
        st = ServerStats()
        _check(_lib().sheen_server_stats(self.handle, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        if self.handle:
            # Destroy waits for in-flight requests; only then are their
            # buffers free to go.
            _lib().sheen_server_destroy(self.handle)
            self.handle = None
        self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Serving workload: the request mix of the serving benchmark.
STREAM_RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080), (2048, 2048))
STREAM_SPP = (1, 4, 16, 64)


def request_stream(n: int = 512, rate: float = 20.0, seed: int = 2024, configs=(0, 1, 2, 3),
                   seeds_per_config: int = 4):
    """Seeded request stream: Poisson arrivals at `rate` per second; each
    request draws a scene generator from `configs` with a seed from a pool of
    `seeds_per_config` (so scenes repeat and the device cache matters), a
    resolution from STREAM_RESOLUTIONS and a sample count from STREAM_SPP.
    Returns a list of dicts sorted by arrival time (seconds from the start)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    t = np.cumsum(gaps) - gaps[0]
    out = []
    for i in range(n):
        cfg = int(configs[rng.integers(len(configs))])
        w, h = STREAM_RESOLUTIONS[rng.integers(len(STREAM_RESOLUTIONS))]
        out.append({"t": float(t[i]), "config": cfg, "seed": int(1000 + rng.integers(seeds_per_config)),
                    "width": w, "height": h, "spp": int(STREAM_SPP[rng.integers(len(STREAM_SPP))])})
    return out
