"""Synthetic workload generators: deterministic, with the documented sizes."""
import ctypes

import numpy as np

import sheen_b200 as sb
from sheen_b200 import contract as C


def _bytes(view, name, dt):
    n = getattr(view, "num_" + name)
    return bytes((ctypes.c_ubyte * (n * dt.itemsize)).from_address(getattr(view, name))) if n else b""


def test_deterministic():
    for cfg, detail in ((0, 0), (1, 3), (2, 0), (3, 0)):
        a, b = sb.generate_scene(cfg, 7, detail, 1000), sb.generate_scene(cfg, 7, detail, 1000)
        for name, dt in C.ARRAY_FIELDS:
            assert _bytes(a.view, name, dt) == _bytes(b.view, name, dt), (cfg, name)
        c = sb.generate_scene(cfg, 8, detail, 1000)
        if cfg in (0, 1, 2):
            assert any(_bytes(a.view, n, d) != _bytes(c.view, n, d) for n, d in C.ARRAY_FIELDS)


def test_sizes():
    s = sb.generate_scene(0, 1)
    assert s.view.num_objects == 64 and s.view.num_planes == 1 and s.view.num_lights == 1
    assert s.settings["width"] == 640 and s.settings["aa"] == 1
    s = sb.generate_scene(1, 1, 8)
    assert s.view.num_triangles == 20 * 4 ** 8 + 16 * 50000 == 2110720
    assert s.view.num_lights == 4
    mats = np.frombuffer((ctypes.c_ubyte * (112 * s.view.num_materials)).from_address(s.view.materials), C.MATERIAL)
    tris = np.frombuffer((ctypes.c_ubyte * (112 * s.view.num_triangles)).from_address(s.view.triangles),
                         C.TRIANGLE)
    glass = mats["transmission"][tris["material_id"]] > 0
    assert glass.sum() == 4 * 50000
    s = sb.generate_scene(2, 1)
    v = s.view
    assert v.num_superellipsoids == 256 + 2 and v.num_lathes == 64 and v.num_prisms == 64
    assert v.num_sweep_strands == 32 and v.num_heightfields == 1 and v.csg_root >= 0
    s = sb.generate_scene(3, 1, 0, 4000000)
    assert s.view.photons == 4000000 and abs(s.view.photon_cell - 0.2) < 1e-7


def test_bvh4_structure():
    """The wavefront form's BVH4: every triangle in one leaf, decoded 8-bit
    child boxes contain everything below them, depth within the stack."""
    L = sb.lib()
    L.sheen_selfcheck_bvh4.argtypes = [ctypes.c_void_p]
    L.sheen_selfcheck_bvh4.restype = ctypes.c_int
    for detail in (3, 6):
        s = sb.generate_scene(1, 3, detail)
        d = L.sheen_selfcheck_bvh4(s.view_ptr)
        assert 1 <= d <= 15, d


def test_extended_per_primitive_arrays_cover_every_primitive():
    """SheenSceneExt's per-primitive arrays hold one entry per primitive (the
    library and the oracle read that many): the analytic workload's CSG-leaf
    superellipsoids carry n2 = 0 (single-exponent body), and two generations
    give the same bytes over the whole array."""
    import ctypes

    from sheen_b200 import contract as C

    def n2_bytes():
        s = sb.generate_scene(2, 1, 0, 0, extended=True)
        x = C.SheenSceneExt.from_buffer_copy(ctypes.string_at(s.ext_ptr, ctypes.sizeof(C.SheenSceneExt)))
        n = s.view.num_superellipsoids
        return np.frombuffer(ctypes.string_at(x.se_n2, 4 * n), np.float32).copy(), n

    a, n = n2_bytes()
    b, _ = n2_bytes()
    assert n == 258 and np.array_equal(a, b)
    assert (a[:256] > 0).all() and (a[256:] == 0).all()
