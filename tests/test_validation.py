"""Scenes whose indices leave their arrays are refused at scene creation
(the device code trusts every index it reads, as the reference's does), so
a bad scene is an error message instead of a GPU fault.  The host checks
run before any device call; triangle material ids are checked on the
device after upload."""
import ctypes

import numpy as np
import pytest

import sheen_b200 as sb
from sheen_b200 import contract as C


def _create_error(view):
    L = sb.lib()
    L.sheen_scene_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.sheen_scene_create.restype = ctypes.c_int
    h = ctypes.c_void_p()
    rc = L.sheen_scene_create(ctypes.addressof(view), sb.FORM_WAVEFRONT, ctypes.byref(h))
    return rc, sb.last_error()


@pytest.fixture(scope="module")
def analytic():
    return sb.generate_scene(2, 1, 0, 0)


def _copy(scene):
    return C.SheenScene.from_buffer_copy(scene.view)


def test_csg_leaf_without_its_superellipsoids(analytic):
    v = _copy(analytic)
    assert v.csg_root >= 0
    v.num_superellipsoids = 0
    v.superellipsoids = None
    rc, err = _create_error(v)
    assert rc == -1 and "CSG superellipsoid leaf index out of range" in err


def test_csg_child_index_out_of_range(analytic):
    v = _copy(analytic)
    # a copy of the node array with the root's left child past the end
    raw = np.ctypeslib.as_array((ctypes.c_int32 * (8 * v.num_csg_nodes)).from_address(v.csg_nodes)).copy()
    raw = raw.reshape(v.num_csg_nodes, 8)
    root = v.csg_root
    assert raw[root, 1] < 0                       # interior node
    raw[root, 3] = v.num_csg_nodes + 5
    buf = np.ascontiguousarray(raw)
    v.csg_nodes = buf.ctypes.data
    rc, err = _create_error(v)
    assert rc == -1 and "CSG child index out of range" in err


def test_lathe_points_out_of_range(analytic):
    v = _copy(analytic)
    assert v.num_lathes > 0
    v.num_lathe_points = 1
    rc, err = _create_error(v)
    assert rc == -1 and "lathe points out of range" in err


def test_material_id_out_of_range(analytic):
    v = _copy(analytic)
    v.num_materials = 1          # other primitives use higher ids
    rc, err = _create_error(v)
    assert rc == -1 and "material_id out of range" in err


def test_null_array_with_count(analytic):
    v = _copy(analytic)
    v.prisms = None
    rc, err = _create_error(v)
    assert rc == -1 and "null array with a nonzero count" in err


@pytest.mark.gpu
def test_triangle_material_out_of_range_refused_on_device():
    sb.init(0, 100)
    s = C.SceneArrays()
    t = np.zeros(3, C.TRIANGLE)
    t["v0"] = [[0, 0, 0]] * 3
    t["v1"] = [[1, 0, 0]] * 3
    t["v2"] = [[0, 1, 0]] * 3
    t["material_id"] = [0, 0, 7]
    s.materials = np.zeros(1, C.MATERIAL)
    s.materials[0] = C.default_material()[0]
    s.triangles = t
    with pytest.raises(RuntimeError, match="triangle material_id out of range"):
        sb.DeviceScene(s, sb.FORM_WAVEFRONT)
    t["material_id"] = 0
    s.triangles = t
    ds = sb.DeviceScene(s, sb.FORM_WAVEFRONT)     # the same scene with valid ids
    ds.close()


@pytest.mark.gpu
def test_lathe_segment_table_hits_equal_plain_form(analytic):
    """The wavefront form tests lathes with the segment constants computed
    once per scene (lathe_segments_kernel) instead of per ray, after a box
    test against the surface's own bound about the Y axis; on a scene of
    lathes (and the ground plane) its primary hits equal the plain form's,
    which runs cone_test on every segment, bit for bit."""
    sb.init(0, 100)
    v = _copy(analytic)
    for k in ("num_objects", "num_sweep_strands", "num_triangles", "num_heightfields", "num_superellipsoids",
              "num_prisms"):
        setattr(v, k, 0)
    v.csg_root = -1
    hits = []
    for form in (sb.FORM_PLAIN, sb.FORM_WAVEFRONT):
        ds = sb.DeviceScene(v, form)
        hits.append(ds.primary_hits(640, 360, 1))
        ds.close()
    (o0, m0, t0), (o1, m1, t1) = hits
    assert (o0 < 0).sum() > 1000                    # lathe hits present
    assert np.array_equal(o0, o1) and np.array_equal(m0, m1)
    assert np.array_equal(t0, t1)


@pytest.mark.gpu
def test_superellipsoid_sign_shortcuts_hits_equal_plain_form(analytic):
    """The wavefront form decides most superellipsoid samples from two
    bounds on max|q| and sum|q| (SeSign) instead of three powf; the
    decisions equal F > 1's, so on a scene of superellipsoids (and the
    ground plane) its primary hits equal the plain form's bit for bit."""
    sb.init(0, 100)
    v = _copy(analytic)
    for k in ("num_objects", "num_sweep_strands", "num_triangles", "num_heightfields", "num_lathes",
              "num_prisms"):
        setattr(v, k, 0)
    v.csg_root = -1
    hits = []
    for form in (sb.FORM_PLAIN, sb.FORM_WAVEFRONT):
        ds = sb.DeviceScene(v, form)
        hits.append(ds.primary_hits(640, 360, 1))
        ds.close()
    (o0, m0, t0), (o1, m1, t1) = hits
    assert (o0 < 0).sum() > 1000                    # superellipsoid hits present
    assert np.array_equal(o0, o1) and np.array_equal(m0, m1)
    assert np.array_equal(t0, t1)


@pytest.mark.gpu
def test_csg_box_hits_equal_plain_form(analytic):
    """The wavefront form skips the CSG tree for rays that miss the box of
    its leaf solids; on a scene of spheres, superellipsoids, the CSG tree
    and the ground plane its primary hits equal the plain form's bit for
    bit (the plain form evaluates the tree for every ray, as the reference
    does)."""
    sb.init(0, 100)
    v = _copy(analytic)
    for k in ("num_sweep_strands", "num_triangles", "num_heightfields", "num_lathes", "num_prisms"):
        setattr(v, k, 0)
    assert v.csg_root >= 0
    hits = []
    for form in (sb.FORM_PLAIN, sb.FORM_WAVEFRONT):
        ds = sb.DeviceScene(v, form)
        hits.append(ds.primary_hits(640, 360, 1))
        img, _ = ds.render_host(160, 90, 1)
        hits[-1] = hits[-1] + (img,)
        ds.close()
    (o0, m0, t0, i0), (o1, m1, t1, i1) = hits
    assert np.array_equal(o0, o1) and np.array_equal(m0, m1)
    assert np.array_equal(t0, t1)
    assert np.abs(i0 - i1).mean() <= 1e-3


@pytest.mark.gpu
def test_strand_reach_cull_equals_plain_form(analytic):
    """The wavefront form skips the tests of strand pieces whose bounding
    sphere the ray's line misses (in the closest-hit test and in the
    optical depth of shadow rays); on a scene of the strands and the ground
    plane its primary hits equal the plain form's bit for bit, and the
    images, whose shadow rays carry the strands' optical depth, agree to the
    last bits of the two forms' separately compiled shading."""
    sb.init(0, 100)
    v = _copy(analytic)
    for k in ("num_objects", "num_superellipsoids", "num_triangles", "num_heightfields", "num_lathes",
              "num_prisms"):
        setattr(v, k, 0)
    v.csg_root = -1
    assert v.num_sweep_strands > 0
    res = []
    for form in (sb.FORM_PLAIN, sb.FORM_WAVEFRONT):
        ds = sb.DeviceScene(v, form)
        o, m, t = ds.primary_hits(640, 360, 1)
        img, _ = ds.render_host(320, 180, 1)
        ds.close()
        res.append((o, m, t, img))
    (o0, m0, t0, i0), (o1, m1, t1, i1) = res
    assert (o0 < 0).sum() > 1000                    # strand hits present
    assert np.array_equal(o0, o1) and np.array_equal(m0, m1) and np.array_equal(t0, t1)
    assert np.abs(i0 - i1).mean() <= 1e-5
