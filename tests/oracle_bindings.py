"""ctypes bindings for the parity checkers under oracle/ (test use only).

- ``Oracle``: this repository's C restatement of the path
  (oracle/libsheen_oracle.so, FP32; oracle/libsheen_oracle64.so, FP64).
- ``RefHost``: the reference's own per-pixel code compiled for the host
  cores (oracle/_ref/libsheen_ref_host.so, built from the reference sources
  by oracle/Makefile; absent on machines without the reference tree unless
  the built library was carried over).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double

MISS = -2147483648


def _load(path):
    return ctypes.CDLL(path) if os.path.exists(path) else None


class Oracle:
    def __init__(self, fp64: bool = False):
        path = os.path.join(ORACLE_DIR, "libsheen_oracle64.so" if fp64 else "libsheen_oracle.so")
        self.lib = _load(path)
        if self.lib is None:
            raise FileNotFoundError(path)
        L = self.lib
        L.oracle_scene_create.argtypes = [P]
        L.oracle_scene_create.restype = P
        L.oracle_scene_create_ext.argtypes = [P, P]
        L.oracle_scene_create_ext.restype = P
        L.oracle_scene_destroy.argtypes = [P]
        L.oracle_scene_photon_count.argtypes = [P]
        L.oracle_scene_photon_count.restype = I
        L.oracle_render.argtypes = [P, I, I, I, P, I, I, I]
        L.oracle_render.restype = I
        L.oracle_primary_hits.argtypes = [P, I, I, I, P, P, P, I]
        L.oracle_primary_hits.restype = I
        L.oracle_trace.argtypes = [P, I, P, P, P, P, I]
        L.oracle_trace.restype = I
        L.oracle_scene_set_centered.argtypes = [P, I]
        L.oracle_scene_set_centered.restype = None
        L.oracle_scene_set_knn.argtypes = [P, I]
        L.oracle_scene_set_knn.restype = None
        L.oracle_primary_hits_px.argtypes = [P, I, I, I, I, P, P, P, P, I]
        L.oracle_primary_hits_px.restype = I
        L.oracle_render_region.argtypes = [P, I, I, I, I, I, I, I, P, I, P]
        L.oracle_render_region.restype = I

    def scene(self, view_ptr: int, centered: bool = False, knn: int = 0, ext_ptr: int | None = None):
        ptr = (self.lib.oracle_scene_create_ext(view_ptr, ext_ptr) if ext_ptr
               else self.lib.oracle_scene_create(view_ptr))
        h = _Handle(self.lib, ptr, self.lib.oracle_scene_destroy)
        if centered:
            self.lib.oracle_scene_set_centered(h.ptr, 1)
        if knn:
            self.lib.oracle_scene_set_knn(h.ptr, knn)
        return h

    def render(self, h, W, H, aa, y0=0, y1=0, threads=0):
        out = np.zeros((H, W, 4), np.float32)
        assert self.lib.oracle_render(h.ptr, W, H, aa, out.ctypes.data, y0, y1, threads) == 0
        return out

    def trace(self, h, rays, threads=0):
        """Closest hits of rays given as (n, 6) doubles (origin, direction)."""
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
        n = len(rays)
        cat = np.zeros(n, np.int32)
        prim = np.zeros(n, np.int32)
        t = np.zeros(n, np.float64)
        assert self.lib.oracle_trace(h.ptr, n, rays.ctypes.data, cat.ctypes.data, prim.ctypes.data, t.ctypes.data,
                                     threads) == 0
        return cat, prim, t

    def primary_hits(self, h, W, H, aa, threads=0):
        ns = max(1, min(aa, 64))
        cat = np.zeros(W * H * ns, np.int32)
        prim = np.zeros(W * H * ns, np.int32)
        t = np.zeros(W * H * ns, np.float64)
        assert self.lib.oracle_primary_hits(h.ptr, W, H, aa, cat.ctypes.data, prim.ctypes.data,
                                            t.ctypes.data, threads) == 0
        return cat, prim, t

    def primary_hits_px(self, h, W, H, aa, pixels, threads=0):
        """Primary hits of the given pixels (flat indices y*W + x): arrays of
        len(pixels) * ns entries, index i*ns + s."""
        ns = max(1, min(aa, 64))
        px = np.ascontiguousarray(pixels, dtype=np.int32)
        n = len(px)
        cat = np.zeros(n * ns, np.int32)
        prim = np.zeros(n * ns, np.int32)
        t = np.zeros(n * ns, np.float64)
        assert self.lib.oracle_primary_hits_px(h.ptr, W, H, aa, n, px.ctypes.data, cat.ctypes.data,
                                               prim.ctypes.data, t.ctypes.data, threads) == 0
        return cat, prim, t

    def render_region(self, h, W, H, aa, x0, y0, x1, y1, threads=0):
        """RGBA of a pixel rectangle (whole-image array) and the number of
        scene queries it issued."""
        out = np.zeros((H, W, 4), np.float32)
        q = ctypes.c_ulonglong(0)
        assert self.lib.oracle_render_region(h.ptr, W, H, aa, x0, y0, x1, y1, out.ctypes.data, threads,
                                             ctypes.byref(q)) == 0
        return out, int(q.value)

    def photon_count(self, h):
        return self.lib.oracle_scene_photon_count(h.ptr)


class RefHost:
    PATH = os.path.join(ORACLE_DIR, "_ref", "libsheen_ref_host.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self):
        self.lib = _load(self.PATH)
        if self.lib is None:
            raise FileNotFoundError(self.PATH)
        L = self.lib
        L.sheen_ref_scene_create.argtypes = [P, I]
        L.sheen_ref_scene_create.restype = P
        L.sheen_ref_scene_destroy.argtypes = [P]
        L.sheen_ref_scene_render.argtypes = [P, I, I, I, P, I, I, I]
        L.sheen_ref_scene_render.restype = I
        L.sheen_ref_scene_primary_hits.argtypes = [P, I, I, I, P, P, P, I]
        L.sheen_ref_scene_primary_hits.restype = I
        L.sheen_ref_scene_photons.argtypes = [P]
        L.sheen_ref_scene_photons.restype = I
        L.sheen_ref_scene_photon_data.argtypes = [P, P, I]
        L.sheen_ref_scene_photon_data.restype = I
        L.sheen_ref_max_threads.restype = I
        L.sheen_ref_load_scene_file.argtypes = [ctypes.c_char_p]
        L.sheen_ref_load_scene_file.restype = P
        L.sheen_ref_loaded_view.argtypes = [P]
        L.sheen_ref_loaded_view.restype = P
        L.sheen_ref_loaded_settings.argtypes = [P, P]
        L.sheen_ref_loaded_free.argtypes = [P]

    def scene(self, view_ptr: int, threads=0):
        return _Handle(self.lib, self.lib.sheen_ref_scene_create(view_ptr, threads), self.lib.sheen_ref_scene_destroy)

    def render(self, h, W, H, aa, threads=0, by0=0, by1=0):
        out = np.zeros((H, W, 4), np.float32)
        assert self.lib.sheen_ref_scene_render(h.ptr, W, H, aa, out.ctypes.data, threads, by0, by1) == 0
        return out

    def primary_hits(self, h, W, H, aa, threads=0):
        ns = max(1, min(aa, 64))
        obj = np.zeros(W * H * ns, np.int32)
        mat = np.zeros(W * H * ns, np.int32)
        t = np.zeros(W * H * ns, np.float32)
        assert self.lib.sheen_ref_scene_primary_hits(h.ptr, W, H, aa, obj.ctypes.data, mat.ctypes.data,
                                                     t.ctypes.data, threads) == 0
        return obj, mat, t

    def photons(self, h):
        n = self.lib.sheen_ref_scene_photons(h.ptr)
        out = np.zeros((n, 12), np.float32)
        if n:
            self.lib.sheen_ref_scene_photon_data(h.ptr, out.ctypes.data, n)
        return out


class _Handle:
    def __init__(self, lib, ptr, free):
        self.lib, self.ptr, self._free = lib, ptr, free

    def close(self):
        if self.ptr:
            self._free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def image_error(a: np.ndarray, b: np.ndarray) -> dict:
    """Per-pixel RGB errors between two (H, W, 4) images."""
    d = np.abs(a[..., :3].astype(np.float64) - b[..., :3].astype(np.float64))
    mse = float((d ** 2).mean())
    return {"mean_abs": float(d.mean()), "max_abs": float(d.max()),
            "frac_px_over_1e-3": float((d.max(-1) > 1e-3).mean()),
            "frac_px_over_1e-2": float((d.max(-1) > 1e-2).mean()),
            "psnr": float(10 * np.log10(1.0 / mse)) if mse > 0 else float("inf")}
