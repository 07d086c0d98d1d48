"""sheen_b200 -- B200 renderer core for Sheen's per-pixel ray-casting path.

Host-side mirror of the reference's Python entry points.  The reference's
native module (api/sheen_py_module.cpp:57-87) exposes ``init(device_id,
cuda_arch)``, ``cleanup()`` and ``render_scene(scene, width, height, aa,
output_path)`` over libsheen_c_api.so; the same three functions are here with
the same argument meaning and errors (RuntimeError carrying
sheen_get_last_error()).  Beside them: RGBA output, resident device scenes
with a choice of renderer form, the .sheen loader, the synthetic workload
generators, and the request loop (``sheen_b200.serve``).

Everything goes through the C-ABI of the in-tree ``libsheen_c_api.so``
(built for sm_100a by ``__graft_entry__.build()`` / ``make -C
sheen_b200/csrc``).  There is no CPU fallback: if the library is missing,
loading fails loudly.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import contract
from .contract import SceneArrays, SheenScene

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsheen_c_api.so")

FORM_PLAIN = 0
FORM_WAVEFRONT = 1
PATH_PLAIN, PATH_QUEUES, PATH_MEGAKERNEL = 0, 1, 2   # sheen_scene_frame_path
RENDER_COUNT_RAYS = 1
RENDER_COUNT_NODES = 2


def _flags(count_rays, count_nodes):
    return (RENDER_COUNT_RAYS if count_rays else 0) | (RENDER_COUNT_NODES if count_nodes else 0)

_lib = None


class RenderStats(ctypes.Structure):
    _fields_ = [("primary_rays", ctypes.c_ulonglong), ("shadow_rays", ctypes.c_ulonglong),
                ("secondary_rays", ctypes.c_ulonglong), ("total_rays", ctypes.c_ulonglong),
                ("node_visits", ctypes.c_ulonglong), ("prim_tests", ctypes.c_ulonglong),
                ("build_ms", ctypes.c_double), ("upload_ms", ctypes.c_double),
                ("photon_ms", ctypes.c_double), ("render_ms", ctypes.c_double),
                ("device_bytes", ctypes.c_ulonglong), ("upload_bytes", ctypes.c_ulonglong),
                ("shadow_node_visits", ctypes.c_ulonglong), ("shadow_prim_tests", ctypes.c_ulonglong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("aa_samples", ctypes.c_int), ("x0", ctypes.c_int), ("y0", ctypes.c_int), ("x1", ctypes.c_int),
                ("y1", ctypes.c_int), ("out_rgba_device", ctypes.c_void_p)]


class StageProfile(ctypes.Structure):
    _fields_ = [("primary_ms", ctypes.c_double), ("shadow_ms", ctypes.c_double * 3), ("reflect_ms", ctypes.c_double),
                ("refract_ms", ctypes.c_double), ("resolve_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("primary_rays", ctypes.c_ulonglong), ("shadow_rays", ctypes.c_ulonglong * 3),
                ("reflect_rays", ctypes.c_ulonglong), ("refract_rays", ctypes.c_ulonglong)]

    def as_dict(self):
        d = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            d[k] = list(v) if not isinstance(v, (int, float)) else v
        return d


class SceneSettings(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("aa", ctypes.c_int),
                ("photons", ctypes.c_int), ("photon_cell", ctypes.c_float),
                ("caustics", ctypes.c_float), ("output", ctypes.c_char * 512)]


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libsheen_c_api.so not built ({LIB_PATH}); run __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    P, I, U, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint, ctypes.c_float
    L.sheen_init.argtypes = [I, I]
    L.sheen_init.restype = I
    L.sheen_cleanup.argtypes = []
    L.sheen_cleanup.restype = None
    L.sheen_render_scene.argtypes = [P, I, I, I, ctypes.c_char_p]
    L.sheen_render_scene.restype = I
    L.sheen_get_last_error.argtypes = []
    L.sheen_get_last_error.restype = ctypes.c_char_p
    L.sheen_render_scene_rgba.argtypes = [P, I, I, I, I, P, ctypes.POINTER(RenderStats)]
    L.sheen_render_scene_rgba.restype = I
    L.sheen_scene_create.argtypes = [P, I, ctypes.POINTER(P)]
    L.sheen_scene_create.restype = I
    L.sheen_scene_destroy.argtypes = [P]
    L.sheen_scene_destroy.restype = None
    L.sheen_scene_device_bytes.argtypes = [P]
    L.sheen_scene_device_bytes.restype = ctypes.c_ulonglong
    L.sheen_scene_form.argtypes = [P]
    L.sheen_scene_form.restype = I
    L.sheen_scene_frame_path.argtypes = [P, I, I, I]
    L.sheen_scene_frame_path.restype = I
    L.sheen_scene_render_device.argtypes = [P, I, I, I, P, P, I, ctypes.POINTER(RenderStats)]
    L.sheen_scene_render_device.restype = I
    L.sheen_scene_render_region.argtypes = [P, I, I, I, I, I, I, I, P, P, I, ctypes.POINTER(RenderStats)]
    L.sheen_scene_render_region.restype = I
    L.sheen_scene_render_host.argtypes = [P, I, I, I, P, I, ctypes.POINTER(RenderStats)]
    L.sheen_scene_render_host.restype = I
    L.sheen_load_scene_file.argtypes = [ctypes.c_char_p, ctypes.POINTER(P)]
    L.sheen_load_scene_file.restype = I
    L.sheen_owned_view.argtypes = [P]
    L.sheen_owned_view.restype = P
    L.sheen_owned_settings.argtypes = [P]
    L.sheen_owned_settings.restype = ctypes.POINTER(SceneSettings)
    L.sheen_owned_free.argtypes = [P]
    L.sheen_owned_free.restype = None
    L.sheen_generate_scene.argtypes = [I, U, I, I, ctypes.POINTER(P)]
    L.sheen_generate_scene.restype = I
    L.sheen_generate_scene_ext.argtypes = [I, U, I, I, I, ctypes.POINTER(P)]
    L.sheen_generate_scene_ext.restype = I
    L.sheen_owned_ext.argtypes = [P]
    L.sheen_owned_ext.restype = P
    L.sheen_scene_create_ext.argtypes = [P, P, I, ctypes.POINTER(P)]
    L.sheen_scene_create_ext.restype = I
    L.sheen_scene_primary_hits.argtypes = [P, I, I, I, P, P, P]
    L.sheen_scene_profile_stages.argtypes = [P, I, I, I, P, P, ctypes.POINTER(StageProfile)]
    L.sheen_render_batch.argtypes = [ctypes.POINTER(BatchJob), I, P, ctypes.POINTER(RenderStats)]
    L.sheen_scene_trace.argtypes = [P, P, I, P, P, P]
    L.sheen_scene_trace.restype = I
    L.sheen_render_batch.restype = I
    L.sheen_scene_profile_stages.restype = I
    L.sheen_scene_primary_hits.restype = I
    L.sheen_write_png_srgb.argtypes = [ctypes.c_char_p, P, I, I]
    L.sheen_write_png_srgb.restype = I
    _lib = L
    return L


def last_error() -> str:
    return lib().sheen_get_last_error().decode("utf-8", "replace")


def _check(rc):
    if rc != 0:
        raise RuntimeError(last_error())


def _scene_ptr(scene):
    """Accepts a ctypes SheenScene, SceneArrays, OwnedScene or a raw address."""
    if isinstance(scene, SceneArrays):
        v = scene.view()
        return ctypes.addressof(v), v
    if isinstance(scene, OwnedScene):
        return scene.view_ptr, scene
    if isinstance(scene, SheenScene):
        return ctypes.addressof(scene), scene
    if isinstance(scene, int):
        return scene, None
    raise TypeError("scene must be a SheenScene, SceneArrays, OwnedScene or address")


# --- reference-compatible entry points (api/sheen_py_module.cpp:33-87) ---

def init(device_id: int = 0, cuda_arch: int = 100) -> None:
    _check(lib().sheen_init(device_id, cuda_arch))


def cleanup() -> None:
    lib().sheen_cleanup()


def render_scene(scene, width: int, height: int, aa: int, output_path: str) -> None:
    ptr, keep = _scene_ptr(scene)
    _check(lib().sheen_render_scene(ptr, width, height, aa, output_path.encode()))
    del keep


# --- additions ---

def render_rgba(scene, width: int, height: int, aa: int, form: int = FORM_PLAIN):
    """Linear RGBA float32 image (height, width, 4) and the render stats."""
    ptr, keep = _scene_ptr(scene)
    out = np.empty((height, width, 4), np.float32)
    st = RenderStats()
    _check(lib().sheen_render_scene_rgba(ptr, width, height, aa, form, out.ctypes.data, ctypes.byref(st)))
    del keep
    return out, st.as_dict()


class DeviceScene:
    """A scene resident in HBM (SheenDeviceScene).  With ext=True, an
    OwnedScene's extension arrays (sheen_owned_ext) are passed to
    sheen_scene_create_ext; ext may also be a contract.SheenSceneExt."""

    def __init__(self, scene, form: int = FORM_PLAIN, ext=False):
        ptr, keep = _scene_ptr(scene)
        h = ctypes.c_void_p()
        if isinstance(ext, contract.SheenSceneExt):
            _check(lib().sheen_scene_create_ext(ptr, ctypes.addressof(ext), form, ctypes.byref(h)))
        elif ext:
            if not isinstance(scene, OwnedScene):
                raise TypeError("scene extensions come from an OwnedScene")
            _check(lib().sheen_scene_create_ext(ptr, scene.ext_ptr, form, ctypes.byref(h)))
        else:
            _check(lib().sheen_scene_create(ptr, form, ctypes.byref(h)))
        del keep
        self.handle = h.value
        self.form = form

    def frame_path(self, width, height, aa) -> int:
        """PATH_PLAIN, PATH_QUEUES or PATH_MEGAKERNEL: the kernels that render
        a whole frame of this size (sheen_scene_frame_path)."""
        r = lib().sheen_scene_frame_path(self.handle, width, height, aa)
        if r < 0:
            raise RuntimeError(last_error())
        return r

    @property
    def device_bytes(self) -> int:
        return int(lib().sheen_scene_device_bytes(self.handle))

    def render_host(self, width, height, aa, count_rays=False, count_nodes=False):
        out = np.empty((height, width, 4), np.float32)
        st = RenderStats()
        _check(lib().sheen_scene_render_host(self.handle, width, height, aa, out.ctypes.data,
                                             _flags(count_rays, count_nodes), ctypes.byref(st)))
        return out, st.as_dict()

    def render_device(self, width, height, aa, out_ptr: int, stream: int = 0, count_rays=False, stats=False,
                      count_nodes=False):
        """Render into a device buffer (width*height float4).  With count_rays,
        count_nodes or stats the call synchronises and returns the stats."""
        st = RenderStats() if (stats or count_rays or count_nodes) else None
        _check(lib().sheen_scene_render_device(self.handle, width, height, aa, out_ptr, stream,
                                               _flags(count_rays, count_nodes),
                                               ctypes.byref(st) if st is not None else None))
        return st.as_dict() if st is not None else None

    def render_region(self, width, height, aa, x0, y0, x1, y1, out_ptr: int, stream: int = 0,
                      count_rays=False, stats=False):
        """Render pixels [x0, x1) x [y0, y1) of a width x height image into the
        device buffer at out_ptr (whole image, width*height float4)."""
        st = RenderStats() if (stats or count_rays) else None
        _check(lib().sheen_scene_render_region(self.handle, width, height, aa, x0, y0, x1, y1, out_ptr, stream,
                                               _flags(count_rays, False),
                                               ctypes.byref(st) if st is not None else None))
        return st.as_dict() if st is not None else None

    def profile_stages(self, width, height, aa, out_ptr: int, stream: int = 0) -> dict:
        """One wavefront frame into the device buffer at out_ptr with per-stage
        device times (CUDA events) and per-kernel ray counts."""
        p = StageProfile()
        _check(lib().sheen_scene_profile_stages(self.handle, width, height, aa, out_ptr, stream, ctypes.byref(p)))
        return p.as_dict()

    def trace(self, rays: np.ndarray):
        """Closest hits of arbitrary rays (n x 8 float32: origin, t_min,
        direction, t_max): object ids, material ids, t (-1 on a miss)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        obj = np.empty(n, np.int32)
        mat = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        _check(lib().sheen_scene_trace(self.handle, rays.ctypes.data, n, obj.ctypes.data, mat.ctypes.data,
                                       t.ctypes.data))
        return obj, mat, t

    def primary_hits(self, width, height, aa):
        """Per-sample primary closest hits: object id, material id, t."""
        ns = max(1, min(aa, 64))
        n = width * height * ns
        obj = np.zeros(n, np.int32)
        mat = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        _check(lib().sheen_scene_primary_hits(self.handle, width, height, aa, obj.ctypes.data,
                                              mat.ctypes.data, t.ctypes.data))
        return obj, mat, t

    def close(self):
        if self.handle:
            lib().sheen_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OwnedScene:
    """Host scene owned by the library (.sheen loader or generator)."""

    def __init__(self, handle):
        self.handle = handle

    @property
    def view_ptr(self) -> int:
        return lib().sheen_owned_view(self.handle)

    @property
    def view(self) -> SheenScene:
        return SheenScene.from_address(self.view_ptr)

    @property
    def ext_ptr(self) -> int:
        """Address of the scene's SheenSceneExt (zero-filled when it has none)."""
        return lib().sheen_owned_ext(self.handle)

    @property
    def settings(self) -> dict:
        s = lib().sheen_owned_settings(self.handle).contents
        return {"width": s.width, "height": s.height, "aa": s.aa, "photons": s.photons,
                "photon_cell": s.photon_cell, "caustics": s.caustics,
                "output": s.output.decode("utf-8", "replace")}

    def close(self):
        if self.handle:
            lib().sheen_owned_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_scene_file(path: str) -> OwnedScene:
    h = ctypes.c_void_p()
    _check(lib().sheen_load_scene_file(path.encode(), ctypes.byref(h)))
    return OwnedScene(h.value)


def generate_scene(config: int, seed: int = 1, detail: int = 0, photons: int = 0,
                   extended: bool = False) -> OwnedScene:
    """A workload scene; extended: with its extension column
    (sheen_generate_scene_ext) -- config 1 with reflect + refract recursion
    to 4 bounces, config 2 with the extension shapes."""
    h = ctypes.c_void_p()
    if extended:
        _check(lib().sheen_generate_scene_ext(config, seed, detail, photons, 1, ctypes.byref(h)))
    else:
        _check(lib().sheen_generate_scene(config, seed, detail, photons, ctypes.byref(h)))
    return OwnedScene(h.value)


def render_batch(jobs, stream: int = 0, stats: bool = False):
    """Render many jobs in one pass of the wavefront queue kernels
    (sheen_render_batch).  Each job is (scene, width, height, aa, region,
    out_ptr): a DeviceScene, the frame size, samples per pixel, a pixel
    rectangle (x0, y0, x1, y1) or None for the whole frame, and the address
    of a device buffer of width*height float4.  Returns the ray counts when
    stats is true (then it synchronises)."""
    arr = (BatchJob * max(len(jobs), 1))()
    for k, (scene, w, h, aa, region, out_ptr) in enumerate(jobs):
        x0, y0, x1, y1 = region if region is not None else (0, 0, 0, 0)
        arr[k] = BatchJob(scene.handle, w, h, aa, x0, y0, x1, y1, out_ptr)
    st = RenderStats() if stats else None
    _check(lib().sheen_render_batch(arr, len(jobs), stream, ctypes.byref(st) if st is not None else None))
    return st.as_dict() if st is not None else None


def tune_set(key: str, value: int) -> None:
    """Set a launch parameter of the wavefront form (see sheen_tune_set)."""
    L = lib()
    L.sheen_tune_set.argtypes = [ctypes.c_char_p, ctypes.c_int]
    L.sheen_tune_set.restype = ctypes.c_int
    _check(L.sheen_tune_set(key.encode(), int(value)))


def tune_get(key: str) -> int:
    L = lib()
    L.sheen_tune_get.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    L.sheen_tune_get.restype = ctypes.c_int
    v = ctypes.c_int()
    _check(L.sheen_tune_get(key.encode(), ctypes.byref(v)))
    return v.value


TUNE_KEYS = ("wave.shadow_kernel", "wave.refill_min", "wave.shadow_blocks_per_sm", "wave.shadow_stack",
             "wave.tile_w", "wave.mega_samples",
             "wave.inner_min")


class TuneResult(ctypes.Structure):
    _fields_ = [("shadow_kernel", ctypes.c_int), ("refill_min", ctypes.c_int),
                ("shadow_blocks_per_sm", ctypes.c_int), ("candidates", ctypes.c_int),
                ("best_ms", ctypes.c_double), ("default_ms", ctypes.c_double), ("shadow_stack", ctypes.c_int),
                ("inner_min", ctypes.c_int), ("tile_w", ctypes.c_int), ("mega_samples", ctypes.c_int)]


def autotune(scene: "DeviceScene", width: int, height: int, aa: int, reps: int = 3, cache: str | None = None,
             key: str | None = None) -> dict:
    """Pick the fastest launch parameters for a wavefront scene and frame
    shape (sheen_autotune) and keep them in force.  With `cache` (a JSON
    file), a setting found earlier under the same key is applied without
    timing, and new results are added to the file.  The default key is the
    scene's device footprint and the frame shape."""
    import json
    key = key or f"sm_100a|bytes={scene.device_bytes}|{width}x{height}x{aa}"
    table = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
        if key in table:
            for k in TUNE_KEYS:
                if k in table[key]:
                    tune_set(k, table[key][k])
            return dict(table[key], cached=True)
    L = lib()
    L.sheen_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(TuneResult)]
    L.sheen_autotune.restype = ctypes.c_int
    r = TuneResult()
    _check(L.sheen_autotune(scene.handle, width, height, aa, reps, ctypes.byref(r)))
    res = {"wave.shadow_kernel": r.shadow_kernel, "wave.refill_min": r.refill_min,
           "wave.shadow_blocks_per_sm": r.shadow_blocks_per_sm, "wave.shadow_stack": r.shadow_stack,
           "wave.inner_min": r.inner_min, "wave.tile_w": r.tile_w, "wave.mega_samples": r.mega_samples,
           "candidates": r.candidates,
           "best_ms": r.best_ms, "default_ms": r.default_ms}
    if cache:
        table[key] = res
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, cache)
    return dict(res, cached=False)


def write_png(path: str, rgba: np.ndarray) -> None:
    rgba = np.ascontiguousarray(rgba, np.float32)
    _check(lib().sheen_write_png_srgb(path.encode(), rgba.ctypes.data, rgba.shape[1], rgba.shape[0]))
