"""Instanced meshes in a two-level BVH (SheenSceneExt.instances; an extension
with no counterpart in the reference, whose loader flattens every copy).

The mesh workload's extended form (config 1) holds its 16 tori as instances
of one mesh.  Its check is the same scene flattened: the oracle flattens the
instances (oracle/sheen_oracle.c, flatten_instances), and the generator's
plain config 1 is that flattening up to the rounding of the transforms.

CPU: the range checks on instances (run before any device call) and the
oracle's instanced scene against the oracle's flattened one.
GPU (both forms): images and hit distances against the oracle, the
instanced render against the flattened render, ray counts, the queue
pipeline in use, batch jobs equal to single renders.
"""
import ctypes

import numpy as np
import pytest

import sheen_b200 as sb
from sheen_b200 import contract as C
from oracle_bindings import MISS, Oracle, image_error

FORMS = [sb.FORM_PLAIN, sb.FORM_WAVEFRONT]
FORM_IDS = ["plain", "wavefront"]
W, H, AA = 96, 54, 2


@pytest.fixture(scope="module")
def inst_scene():
    return sb.generate_scene(1, 3, 3, extended=True)


@pytest.fixture(scope="module")
def flat_scene():
    return sb.generate_scene(1, 3, 3)


def _ext(scene, max_depth=0):
    x = C.SheenSceneExt.from_buffer_copy(ctypes.string_at(scene.ext_ptr, ctypes.sizeof(C.SheenSceneExt)))
    x.max_depth = max_depth
    return x


def _instances(x):
    arr = (C.SheenInstance * x.num_instances).from_address(x.instances)
    return (C.SheenInstance * x.num_instances).from_buffer_copy(arr)


def _create_error(scene, x):
    L = sb.lib()
    L.sheen_scene_create_ext.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p)]
    L.sheen_scene_create_ext.restype = ctypes.c_int
    h = ctypes.c_void_p()
    rc = L.sheen_scene_create_ext(scene.view_ptr, ctypes.addressof(x), sb.FORM_WAVEFRONT, ctypes.byref(h))
    return rc, sb.last_error()


# ------------------------------------------------------------------ CPU


def test_generator_holds_sixteen_instances(inst_scene, flat_scene):
    x = _ext(inst_scene)
    assert x.num_instances == 16 and x.num_meshes == 1
    meshes = (C.SheenMesh * 1).from_address(x.meshes)
    n_tor = meshes[0].tri_count
    assert x.num_mesh_triangles == n_tor
    # the flattened scene holds the same tori after the icosphere
    assert flat_scene.view.num_triangles == inst_scene.view.num_triangles + 16 * n_tor


@pytest.mark.parametrize("case,message", [
    ("mesh", "instance mesh out of range"),
    ("material", "instance material_id out of range"),
    ("singular", "instance transform not invertible"),
    ("nan", "instance transform not finite"),
    ("range", "mesh triangles out of range"),
])
def test_bad_instances_are_refused(inst_scene, case, message):
    x = _ext(inst_scene)
    inst = _instances(x)
    meshes = (C.SheenMesh * 1).from_buffer_copy((C.SheenMesh * 1).from_address(x.meshes))
    if case == "mesh":
        inst[3].mesh = 1
    elif case == "material":
        inst[5].material_id = inst_scene.view.num_materials
    elif case == "singular":
        for k in range(12):
            inst[2].xform[k] = 0.0
    elif case == "nan":
        inst[7].xform[3] = float("nan")
    elif case == "range":
        meshes[0].tri_count = x.num_mesh_triangles + 1
    x.instances = ctypes.addressof(inst)
    x.meshes = ctypes.addressof(meshes)
    rc, err = _create_error(inst_scene, x)
    assert rc == -1 and message in err, err


def test_oracle_instances_are_the_flattened_scene(inst_scene, flat_scene):
    o = Oracle()
    x = _ext(inst_scene)
    h1 = o.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    a = o.render(h1, 64, 36, 1)
    h1.close()
    h2 = o.scene(flat_scene.view_ptr)
    b = o.render(h2, 64, 36, 1)
    h2.close()
    err = image_error(a, b)
    # the same triangles up to the transforms' rounding (double there, the
    # generator's float rotation here)
    assert err["mean_abs"] <= 1e-4 and err["frac_px_over_1e-2"] <= 0.005, err


# ------------------------------------------------------------------ GPU


@pytest.fixture(scope="module")
def device():
    sb.init(0, 100)
    yield


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_instanced_render_matches_oracle(device, inst_scene, flat_scene, form):
    x = _ext(inst_scene)
    ds = sb.DeviceScene(inst_scene, form, ext=x)
    img, st = ds.render_host(W, H, AA, count_rays=True)
    ds.close()
    o = Oracle()
    h = o.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    ref = o.render(h, W, H, AA)
    h.close()
    err = image_error(img, ref)
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.01, err
    # and against the flattened scene on the device
    flat, _ = sb.DeviceScene(flat_scene, form).render_host(W, H, AA)
    err2 = image_error(img, flat)
    assert err2["mean_abs"] <= 1e-3 and err2["frac_px_over_1e-2"] <= 0.01, err2


def _torus_rays(scene, n, seed=5):
    """float32 rays from the camera towards the instances' centres."""
    rng = np.random.default_rng(seed)
    x = _ext(scene)
    inst = _instances(x)
    cen = np.array([[i.xform[3], i.xform[7], i.xform[11]] for i in inst], np.float32)
    v = scene.view
    cam = np.array([v.camera.position.x, v.camera.position.y, v.camera.position.z], np.float32)
    tgt = cen[rng.integers(0, len(cen), n)] + rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32)
    d = tgt - cam
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = cam
    rays[:, 3] = 1e-3
    rays[:, 4:7] = d
    rays[:, 7] = 1e10
    return rays


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_instanced_hits_match_fp64_oracle(device, inst_scene, form):
    rays = _torus_rays(inst_scene, 20000)
    x = _ext(inst_scene)
    ds = sb.DeviceScene(inst_scene, form, ext=x)
    obj, mat, t = ds.trace(rays)
    ds.close()
    o = Oracle(fp64=True)
    h = o.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    cat, prim, t64 = o.trace(h, np.c_[rays[:, 0:3], rays[:, 4:7]].astype(np.float64))
    h.close()
    n_flat = inst_scene.view.num_triangles
    inst_hit = (obj != MISS) & (obj < -n_flat)        # device hits on instanced triangles
    assert inst_hit.sum() > 2000
    # object ids: spheres their index, everything else -(index + 1)
    want = np.where(cat == 0, prim, -(prim + 1))
    same = (cat >= 0) & (obj == want)
    both = (cat >= 0) & (obj != MISS)
    assert same.sum() >= 0.99 * both.sum()
    sel = same & inst_hit & (cat == 2)
    rel = np.abs(t[sel].astype(np.float64) - t64[sel]) / np.abs(t64[sel])
    assert np.quantile(rel, 0.99) <= 1e-5 and rel.max() <= 1e-4, (np.quantile(rel, 0.99), rel.max())


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_instanced_ray_count_matches_oracle(device, inst_scene, form):
    import torch
    x = _ext(inst_scene)
    ds = sb.DeviceScene(inst_scene, form, ext=x)
    out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    st = ds.render_region(W, H, AA, 0, 0, W, H, out.data_ptr(), 0, count_rays=True)
    torch.cuda.synchronize()
    ds.close()
    o = Oracle()
    h = o.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    _, queries = o.render_region(h, W, H, AA, 0, 0, W, H)
    h.close()
    assert abs(st["total_rays"] - queries) <= max(2, 1e-3 * queries), (st, queries)


@pytest.mark.gpu
def test_instanced_scene_runs_the_queue_stages(device, inst_scene):
    import torch
    ds = sb.DeviceScene(inst_scene, sb.FORM_WAVEFRONT, ext=_ext(inst_scene, 0))
    assert ds.frame_path(1920, 1080, 4) == sb.PATH_QUEUES
    out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    prof = ds.profile_stages(W, H, AA, out.data_ptr())
    ds.close()
    assert prof["primary_rays"] == W * H * AA and prof["refract_rays"] > 0
    deep = sb.DeviceScene(inst_scene, sb.FORM_WAVEFRONT, ext=_ext(inst_scene, 4))
    assert deep.frame_path(1920, 1080, 4) == sb.PATH_MEGAKERNEL
    deep.close()


@pytest.mark.gpu
def test_batch_with_instanced_scenes(device, inst_scene, flat_scene):
    import torch
    a = sb.DeviceScene(inst_scene, sb.FORM_WAVEFRONT, ext=_ext(inst_scene, 0))
    b = sb.DeviceScene(flat_scene, sb.FORM_WAVEFRONT)
    outs = [torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(3)]
    sb.render_batch([(a, W, H, AA, None, outs[0].data_ptr()), (b, W, H, AA, None, outs[1].data_ptr()),
                     (a, W, H, 1, (0, 0, W // 2, H), outs[2].data_ptr())])
    torch.cuda.synchronize()
    ia, _ = a.render_host(W, H, AA)
    ib, _ = b.render_host(W, H, AA)
    ic, _ = a.render_host(W, H, 1)
    a.close()
    b.close()
    assert np.array_equal(outs[0].cpu().numpy(), ia)
    assert np.array_equal(outs[1].cpu().numpy(), ib)
    assert np.array_equal(outs[2].cpu().numpy()[:, :W // 2], ic[:, :W // 2])


def _affine_ext(scene):
    """The extension with non-rigid maps: every instance scaled non-uniformly
    about its centre, every other one mirrored (negative determinant)."""
    x = _ext(scene)
    inst = _instances(x)
    for j, it in enumerate(inst):
        sx, sy, sz = 1.3, 0.8, (-1.1 if j % 2 else 1.1)
        for r in range(3):
            it.xform[4 * r + 0] *= sx
            it.xform[4 * r + 1] *= sy
            it.xform[4 * r + 2] *= sz
    x.instances = ctypes.addressof(inst)
    return x, inst


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_non_rigid_instances_match_oracle(device, inst_scene, form):
    """Scaled and mirrored instances: t is shared by both spaces, normals go
    through the inverse transpose, facing survives a mirror -- against the
    oracle, which flattens the same maps in double."""
    x, keep = _affine_ext(inst_scene)
    ds = sb.DeviceScene(inst_scene, form, ext=x)
    img, _ = ds.render_host(W, H, AA)
    rays = _torus_rays(inst_scene, 10000, seed=8)
    obj, mat, t = ds.trace(rays)
    ds.close()
    o = Oracle()
    h = o.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    ref = o.render(h, W, H, AA)
    h.close()
    err = image_error(img, ref)
    assert err["mean_abs"] <= 1e-3 and err["frac_px_over_1e-2"] <= 0.01, err
    o64 = Oracle(fp64=True)
    h = o64.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(x))
    cat, prim, t64 = o64.trace(h, np.c_[rays[:, 0:3], rays[:, 4:7]].astype(np.float64))
    h.close()
    want = np.where(cat == 0, prim, -(prim + 1))
    same = (cat >= 0) & (obj == want)
    both = (cat >= 0) & (obj != MISS)
    assert same.sum() >= 0.99 * both.sum()
    sel = same & (obj < -inst_scene.view.num_triangles)
    assert sel.sum() > 1000
    rel = np.abs(t[sel].astype(np.float64) - t64[sel]) / np.abs(t64[sel])
    assert np.quantile(rel, 0.99) <= 1e-5, np.quantile(rel, 0.99)
    del keep


def test_instance_arrays_build_the_generators_extension(inst_scene):
    """contract.InstanceArrays (numpy-owned meshes, maps and materials) gives
    the oracle the same scene as the generator's own extension."""
    x = _ext(inst_scene)
    inst = _instances(x)
    meshes = (C.SheenMesh * x.num_meshes).from_address(x.meshes)
    tris = np.frombuffer(ctypes.string_at(x.mesh_triangles, C.TRIANGLE.itemsize * x.num_mesh_triangles),
                         C.TRIANGLE).copy()
    arrays = C.InstanceArrays(
        mesh_triangles=tris,
        meshes=np.array([[m.tri_offset, m.tri_count] for m in meshes], np.int32),
        xforms=np.array([list(i.xform) for i in inst], np.float32).reshape(-1, 3, 4),
        inst_mesh=np.array([i.mesh for i in inst], np.int32),
        inst_material=np.array([i.material_id for i in inst], np.int32))
    mine = arrays.view()
    o = Oracle()
    imgs = []
    for ext in (x, mine):
        h = o.scene(inst_scene.view_ptr, ext_ptr=ctypes.addressof(ext))
        imgs.append(o.render(h, 48, 27, 1))
        h.close()
    assert np.array_equal(imgs[0], imgs[1])
