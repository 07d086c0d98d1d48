"""The wavefront form's triangle BVH4 built on the device.

The device builder (bvh4_gpu.cu) follows the host builder (bvh4.cpp) step
for step with the same rounded arithmetic, so the two must produce
byte-identical node and triangle arrays for the three triangle sets (all,
blocking, passable).  Cases cover both build phases (large nodes split level
by level, small subtrees built in one block), the list split taken when
every centroid coincides, tiny meshes, -0 coordinates, and a glass/opaque
mix that produces all three sets.
"""
import ctypes

import numpy as np
import pytest

import sheen_b200 as sb
from sheen_b200 import contract as C


def _compare(scene):
    L = sb.lib()
    L.sheen_bvh4_compare_builders.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    L.sheen_bvh4_compare_builders.restype = ctypes.c_int
    ptr, keep = sb._scene_ptr(scene)
    t = (ctypes.c_double * 2)()
    rc = L.sheen_bvh4_compare_builders(ptr, t)
    del keep
    return rc, (t[0], t[1])


def _mesh(verts, glass=None):
    """SceneArrays with triangles verts[i] = (v0, v1, v2); material 1 is glass."""
    s = C.SceneArrays()
    n = len(verts)
    t = np.zeros(n, C.TRIANGLE)
    t["v0"], t["v1"], t["v2"] = verts[:, 0], verts[:, 1], verts[:, 2]
    t["material_id"] = 0 if glass is None else glass.astype(np.int32)
    mats = np.zeros(2, C.MATERIAL)
    mats[0] = C.default_material()[0]
    mats[1] = C.default_material()[0]
    mats[1]["transmission"] = 1.0
    s.materials = mats
    s.triangles = t
    return s


def _soup(n, seed, spread=10.0, size=0.3):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3)).astype(np.float32)
    return (c + rng.normal(0.0, size, (n, 3, 3))).astype(np.float32)


def _init():
    sb.init(0, 100)


@pytest.mark.gpu
@pytest.mark.parametrize("detail", [3, 6, 8])
def test_mesh_workload_identical(detail):
    """The mesh workload's generator (icosphere + glass tori): three sets."""
    _init()
    s = sb.generate_scene(1, 3, detail)
    rc, (host_ms, dev_ms) = _compare(s)
    assert rc == 0, (rc, sb.last_error())
    print(f"detail {detail}: host {host_ms:.1f} ms, device {dev_ms:.1f} ms")


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 9, 1023, 1024, 1025, 5000, 70000])
def test_triangle_soups_identical(n):
    """Sizes around the small-subtree threshold and the chunk size, with a
    random glass mix."""
    _init()
    verts = _soup(n, n)
    glass = (np.random.default_rng(n + 1).random(n) < 0.2) if n >= 3 else None
    rc, _ = _compare(_mesh(verts, glass))
    assert rc == 0, (rc, sb.last_error())


@pytest.mark.gpu
def test_vertex_records_identical():
    """The watertight test's record layout ({v0}, {v1}, {v2}) from both builders."""
    _init()
    sb.tune_set("trace.watertight", 1)
    try:
        rc, _ = _compare(sb.generate_scene(1, 3, 5))
    finally:
        sb.tune_set("trace.watertight", 0)
    assert rc == 0, (rc, sb.last_error())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [40, 3000])
def test_coincident_centroids_identical(n):
    """Every centroid equal: no SAH candidate qualifies, the list is split in
    half (the host's fallback), in the small and in the large phase."""
    _init()
    offsets = np.array([[-1.0, -1.0, -1.0], [1.0, 1.0, 1.0], [1.0, -1.0, 0.0]], np.float32)
    scale = np.random.default_rng(7).uniform(0.5, 2.0, (n, 1, 1)).astype(np.float32)
    verts = (scale * offsets[None]).astype(np.float32)   # every box is centred on the origin
    rc, _ = _compare(_mesh(verts))
    assert rc == 0, (rc, sb.last_error())


@pytest.mark.gpu
def test_signed_zero_coordinates_identical():
    """Boxes touching -0 and +0: canonicalised the same way by both."""
    _init()
    verts = _soup(2000, 11, spread=1.0, size=0.5)
    verts[::3, 0, 0] = -0.0
    verts[1::3, 1, 1] = 0.0
    verts[2::3, 2, 2] = -0.0
    rc, _ = _compare(_mesh(verts))
    assert rc == 0, (rc, sb.last_error())


@pytest.mark.gpu
def test_flat_and_degenerate_axes_identical():
    """A planar grid (one flat axis) and zero-area triangles."""
    _init()
    g = np.stack(np.meshgrid(np.arange(60, dtype=np.float32), np.arange(60, dtype=np.float32)), -1).reshape(-1, 2)
    v0 = np.c_[g, np.zeros(len(g), np.float32)]
    verts = np.stack([v0, v0 + [1, 0, 0], v0 + [0, 1, 0]], 1).astype(np.float32)
    deg = np.repeat(v0[:50, None, :], 3, axis=1)   # points
    rc, _ = _compare(_mesh(np.concatenate([verts, deg]).astype(np.float32)))
    assert rc == 0, (rc, sb.last_error())


@pytest.mark.gpu
def test_device_built_scene_renders_like_host_built():
    """A resident wavefront scene built either way renders the same image
    bit for bit (the trees are identical)."""
    _init()
    s = sb.generate_scene(1, 5, 4)
    imgs = []
    for dev_build in (1, 0):
        sb.tune_set("build.device", dev_build)
        try:
            ds = sb.DeviceScene(s, sb.FORM_WAVEFRONT)
            img, _ = ds.render_host(160, 120, 2)
            ds.close()
        finally:
            sb.tune_set("build.device", 1)
        imgs.append(img)
    assert np.array_equal(imgs[0], imgs[1])


def _edge_cases():
    cases = {f"soup{n}": _mesh(_soup(n, n), (np.random.default_rng(n + 1).random(n) < 0.2) if n >= 3 else None)
             for n in (1, 2, 3, 9, 1025, 5000)}
    offsets = np.array([[-1.0, -1.0, -1.0], [1.0, 1.0, 1.0], [1.0, -1.0, 0.0]], np.float32)
    scale = np.random.default_rng(7).uniform(0.5, 2.0, (3000, 1, 1)).astype(np.float32)
    cases["coincident"] = _mesh((scale * offsets[None]).astype(np.float32))
    return cases


@pytest.mark.parametrize("name", sorted(_edge_cases()))
def test_host_builder_edge_cases(name):
    """The host builder (the device builder's reference) on the edge cases:
    structurally valid, depth within the traversal stack."""
    L = sb.lib()
    L.sheen_selfcheck_bvh4.argtypes = [ctypes.c_void_p]
    L.sheen_selfcheck_bvh4.restype = ctypes.c_int
    scene = _edge_cases()[name]
    ptr, keep = sb._scene_ptr(scene)
    d = L.sheen_selfcheck_bvh4(ptr)
    assert 1 <= d <= 15, d


def _kept_cases():
    cases = {}
    for n in (3, 9, 40, 1025, 5000):
        rng = np.random.default_rng(n + 3)
        cases[f"soup{n}_glass20"] = _mesh(_soup(n, n), rng.random(n) < 0.2)
    cases["soup3000_glass90"] = _mesh(_soup(3000, 5), np.random.default_rng(9).random(3000) < 0.9)
    cases["soup500_all_glass"] = _mesh(_soup(500, 6), np.ones(500, bool))
    cases["soup500_one_blocking"] = _mesh(_soup(500, 8), np.arange(500) != 17)
    cases["mesh_workload_detail4"] = sb.generate_scene(1, 3, 4)
    return cases


@pytest.mark.parametrize("name", sorted(_kept_cases()))
def test_derived_blocking_tree(name):
    """The blocking triangles' tree derived from the tree over all (leaves
    lose the passable triangles, one-child nodes are spliced out, boxes
    refitted): the tree over all is unchanged, the derived one holds every
    blocking triangle once, and each of its child boxes is exactly the
    quantised union of the triangles below it (a loose refit fails)."""
    L = sb.lib()
    L.sheen_selfcheck_bvh4_kept.argtypes = [ctypes.c_void_p]
    L.sheen_selfcheck_bvh4_kept.restype = ctypes.c_int
    scene = _kept_cases()[name]
    ptr, keep = sb._scene_ptr(scene)
    d = L.sheen_selfcheck_bvh4_kept(ptr)
    if name == "soup500_all_glass":
        assert d == 0
    else:
        assert 1 <= d <= 15, d


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["soup3000_glass90", "soup500_all_glass", "soup500_one_blocking", "soup40_glass20"])
def test_derived_blocking_tree_device_identical(name):
    """The device's derived blocking tree equals the host's byte for byte,
    including a mostly-passable mesh, an all-passable one (no blocking tree)
    and a single blocking triangle."""
    _init()
    rc, _ = _compare(_kept_cases()[name])
    assert rc == 0, (rc, sb.last_error())


@pytest.mark.parametrize("node_cost", [1, 8, 64])
def test_node_cost_setting_host_trees_valid(node_cost):
    """build.node_cost (the SAH price of a node visit against a triangle
    test) changes the leaf sizes; the trees stay valid and tight."""
    L = sb.lib()
    L.sheen_selfcheck_bvh4_kept.argtypes = [ctypes.c_void_p]
    L.sheen_selfcheck_bvh4_kept.restype = ctypes.c_int
    scene = _kept_cases()["mesh_workload_detail4"]
    ptr, keep = sb._scene_ptr(scene)
    sb.tune_set("build.node_cost", node_cost)
    try:
        d = L.sheen_selfcheck_bvh4_kept(ptr)
    finally:
        sb.tune_set("build.node_cost", 4)
    assert 1 <= d <= 15, d


@pytest.mark.gpu
@pytest.mark.parametrize("node_cost", [2, 8])
def test_node_cost_setting_device_identical(node_cost):
    """Both builders read build.node_cost and stay byte-identical."""
    _init()
    sb.tune_set("build.node_cost", node_cost)
    try:
        rc, _ = _compare(sb.generate_scene(1, 3, 6))
    finally:
        sb.tune_set("build.node_cost", 4)
    assert rc == 0, (rc, sb.last_error())
