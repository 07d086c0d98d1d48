"""Binary scene contract on the Python side.

numpy structured dtypes for every POD array of a Sheen scene and a ctypes
``SheenScene`` with the exact layout of ``include/sheen_c_api.h`` (352 bytes,
field offsets of the reference's sheen_c_api.h:18-87).  The reference's
ctypes contract (addon_sheen/sheen_render/c_api_contract.py) is kept as the
naming model, but its two size defects are not reproduced: HeightField is 64
bytes here (the reference's ctypes class is 72, c_api_contract.py:144-160)
and CSGNode is 32 (the reference's ctypes class is 20).  The C layout is the
authority; tests/test_abi.py checks these dtypes against the compiled library.

``SceneArrays`` keeps the numpy arrays alive and hands out a ``SheenScene``
whose pointers point into them.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

F3 = ("<f4", (3,))
F2 = ("<f4", (2,))


def _dt(fields, itemsize):
    names, formats, offsets = [], [], []
    for name, fmt, off in fields:
        names.append(name)
        formats.append(fmt)
        offsets.append(off)
    return np.dtype({"names": names, "formats": formats, "offsets": offsets,
                     "itemsize": itemsize})


CAMERA = _dt([("position", F3, 0), ("right", F3, 12), ("up", F3, 24), ("forward", F3, 36),
              ("focal_length", "<f4", 48), ("sensor_width", "<f4", 52),
              ("shift_x", "<f4", 56), ("shift_y", "<f4", 60)], 64)

MATERIAL = _dt([("diffuse_color", F3, 0), ("specular", "<f4", 12), ("shininess", "<f4", 16),
                ("ambient", "<f4", 20), ("texture_id", "<i4", 24), ("_pad_tex", "<i4", 28),
                ("anisotropy", "<f4", 32), ("hair_shift", "<f4", 36), ("hair_spec_r", "<f4", 40),
                ("hair_exp_r", "<f4", 44), ("hair_spec_t", "<f4", 48), ("hair_exp_t", "<f4", 52),
                ("hair_backlight", "<f4", 56), ("reflect", "<f4", 60), ("transmission", "<f4", 64),
                ("ior", "<f4", 68), ("emission_color", F3, 72), ("emission", "<f4", 84),
                ("mask_id", "<i4", 88), ("normal_id", "<i4", 92), ("normal_strength", "<f4", 96)], 112)

TRIANGLE = _dt([("v0", F3, 0), ("v1", F3, 12), ("v2", F3, 24), ("n0", F3, 36), ("n1", F3, 48),
                ("n2", F3, 60), ("uv0", F2, 72), ("uv1", F2, 80), ("uv2", F2, 88),
                ("material_id", "<i4", 96)], 112)

OBJECT = _dt([("type", "<i4", 0), ("material_id", "<i4", 4), ("param1", F3, 8),
              ("param2", "<f4", 20)], 48)

LIGHT = _dt([("direction", F3, 0), ("position", F3, 12), ("u_axis", F3, 24), ("v_axis", F3, 36),
             ("color", F3, 48), ("intensity", "<f4", 60), ("radius", "<f4", 64), ("angle", "<f4", 68),
             ("blend", "<f4", 72), ("beam", "<f4", 76), ("type", "<i4", 80), ("flags", "<i4", 84),
             ("texture_id", "<i4", 88)], 96)

MEDIUM = _dt([("center", F3, 0), ("half", F3, 12), ("sigma_s", F3, 24), ("sigma_t", "<f4", 36),
              ("samples", "<i4", 40)], 48)

PLANE = _dt([("normal", F3, 0), ("d", "<f4", 12), ("material_id", "<i4", 16)], 32)

SWEEP_POINT = _dt([("position", F3, 0), ("radius", "<f4", 12)], 16)
SWEEP_STRAND = _dt([("point_offset", "<i4", 0), ("point_count", "<i4", 4),
                    ("material_id", "<i4", 8)], 16)

HEIGHTFIELD = _dt([("center", F3, 0), ("size_x", "<f4", 12), ("size_z", "<f4", 16),
                   ("height", "<f4", 20), ("freq", "<f4", 24), ("octaves", "<i4", 28),
                   ("seed", "<i4", 32), ("material_id", "<i4", 36), ("image", "<u8", 40),
                   ("img_w", "<i4", 48), ("img_h", "<i4", 52)], 64)

LATHE_POINT = _dt([("y", "<f4", 0), ("radius", "<f4", 4)], 16)
LATHE = _dt([("center", F3, 0), ("point_offset", "<i4", 12), ("point_count", "<i4", 16),
             ("material_id", "<i4", 20)], 32)

PRISM_POINT = _dt([("x", "<f4", 0), ("z", "<f4", 4)], 16)
PRISM = _dt([("center", F3, 0), ("y_min", "<f4", 12), ("y_max", "<f4", 16), ("sweep", "<f4", 20),
             ("point_offset", "<i4", 24), ("point_count", "<i4", 28), ("material_id", "<i4", 32)], 48)

CSG_NODE = _dt([("op", "<i4", 0), ("leaf_kind", "<i4", 4), ("leaf_index", "<i4", 8),
                ("left", "<i4", 12), ("right", "<i4", 16)], 32)

SUPERELLIPSOID = _dt([("center", F3, 0), ("a", "<f4", 12), ("b", "<f4", 16), ("c", "<f4", 20),
                      ("n", "<f4", 24), ("material_id", "<i4", 28)], 48)


class _F3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class CameraData(ctypes.Structure):
    _fields_ = [("position", _F3), ("right", _F3), ("up", _F3), ("forward", _F3),
                ("focal_length", ctypes.c_float), ("sensor_width", ctypes.c_float),
                ("shift_x", ctypes.c_float), ("shift_y", ctypes.c_float)]


_P = ctypes.c_void_p
_I = ctypes.c_int


class SheenScene(ctypes.Structure):
    """ctypes view of ``SheenScene`` (sheen_c_api.h:18-87).  Pointer fields
    are untyped here; ``SceneArrays.view()`` fills them."""
    _fields_ = [
        ("camera", CameraData),
        ("objects", _P), ("num_objects", _I),
        ("sweep_points", _P), ("num_sweep_points", _I),
        ("sweep_strands", _P), ("num_sweep_strands", _I),
        ("triangles", _P), ("num_triangles", _I),
        ("heightfields", _P), ("num_heightfields", _I),
        ("superellipsoids", _P), ("num_superellipsoids", _I),
        ("lathe_points", _P), ("num_lathe_points", _I),
        ("lathes", _P), ("num_lathes", _I),
        ("prism_points", _P), ("num_prism_points", _I),
        ("prisms", _P), ("num_prisms", _I),
        ("csg_nodes", _P), ("csg_root", _I), ("num_csg_nodes", _I),
        ("planes", _P), ("num_planes", _I),
        ("materials", _P), ("num_materials", _I),
        ("texture_pixels", _P), ("texture_widths", _P), ("texture_heights", _P),
        ("num_textures", _I),
        ("lights", _P), ("num_lights", _I),
        ("photons", _I), ("photon_cell", ctypes.c_float), ("caustics", ctypes.c_float),
        ("media", _P), ("num_media", _I),
        # ctypes aligns CameraData to 4 bytes, the C struct to 16, which rounds
        # the C SheenScene up to 352 bytes; the explicit tail matches that.
        ("_tail", ctypes.c_byte * 12),
    ]


assert ctypes.sizeof(SheenScene) == 352
assert SheenScene.photons.offset == 316 and SheenScene.media.offset == 328


class SheenSceneExt(ctypes.Structure):
    """ctypes view of this library's ``SheenSceneExt`` (scene extensions, no
    counterpart in the reference's contract).  Pointer fields are untyped."""
    _fields_ = [
        ("lathe_bezier", _P), ("prism_bezier", _P), ("bezier_ctrl", _P), ("num_bezier_ctrl", _I),
        ("se_n2", _P),
        ("hf_grid", _P), ("hf_heights", _P), ("num_hf_heights", _I),
        ("csg_roots", _P), ("num_csg_roots", _I),
        ("csg_boxes", _P), ("num_csg_boxes", _I),
        ("csg_cones", _P), ("num_csg_cones", _I),
        ("max_depth", _I),
        ("mesh_triangles", _P), ("num_mesh_triangles", _I),
        ("meshes", _P), ("num_meshes", _I),
        ("instances", _P), ("num_instances", _I),
    ]


class SheenInstance(ctypes.Structure):
    """ctypes view of ``SheenInstance``: a mesh placed by a row-major 3x4
    object-to-world map."""
    _fields_ = [("xform", ctypes.c_float * 12), ("mesh", _I), ("material_id", _I)]


class SheenMesh(ctypes.Structure):
    _fields_ = [("tri_offset", _I), ("tri_count", _I)]


def _ptr(a):
    return a.ctypes.data if a is not None and len(a) else None


ARRAY_FIELDS = [
    ("objects", OBJECT), ("sweep_points", SWEEP_POINT), ("sweep_strands", SWEEP_STRAND),
    ("triangles", TRIANGLE), ("heightfields", HEIGHTFIELD), ("superellipsoids", SUPERELLIPSOID),
    ("lathe_points", LATHE_POINT), ("lathes", LATHE), ("prism_points", PRISM_POINT),
    ("prisms", PRISM), ("csg_nodes", CSG_NODE), ("planes", PLANE), ("materials", MATERIAL),
    ("lights", LIGHT), ("media", MEDIUM),
]


@dataclass
class SceneArrays:
    """Owns the numpy arrays of one scene and builds the C view."""
    camera: np.ndarray = field(default_factory=lambda: np.zeros((), CAMERA))
    objects: np.ndarray = field(default_factory=lambda: np.zeros(0, OBJECT))
    sweep_points: np.ndarray = field(default_factory=lambda: np.zeros(0, SWEEP_POINT))
    sweep_strands: np.ndarray = field(default_factory=lambda: np.zeros(0, SWEEP_STRAND))
    triangles: np.ndarray = field(default_factory=lambda: np.zeros(0, TRIANGLE))
    heightfields: np.ndarray = field(default_factory=lambda: np.zeros(0, HEIGHTFIELD))
    superellipsoids: np.ndarray = field(default_factory=lambda: np.zeros(0, SUPERELLIPSOID))
    lathe_points: np.ndarray = field(default_factory=lambda: np.zeros(0, LATHE_POINT))
    lathes: np.ndarray = field(default_factory=lambda: np.zeros(0, LATHE))
    prism_points: np.ndarray = field(default_factory=lambda: np.zeros(0, PRISM_POINT))
    prisms: np.ndarray = field(default_factory=lambda: np.zeros(0, PRISM))
    csg_nodes: np.ndarray = field(default_factory=lambda: np.zeros(0, CSG_NODE))
    csg_root: int = -1
    planes: np.ndarray = field(default_factory=lambda: np.zeros(0, PLANE))
    materials: np.ndarray = field(default_factory=lambda: np.zeros(0, MATERIAL))
    lights: np.ndarray = field(default_factory=lambda: np.zeros(0, LIGHT))
    media: np.ndarray = field(default_factory=lambda: np.zeros(0, MEDIUM))
    textures: list = field(default_factory=list)   # list of (h, w, 3) uint8 arrays
    photons: int = 0
    photon_cell: float = 0.25
    caustics: float = 0.0

    def view(self) -> SheenScene:
        """C view; valid while this object (and its arrays) is alive."""
        s = SheenScene()
        ctypes.memmove(ctypes.addressof(s.camera), self.camera.ctypes.data, 64)
        for name, dt in ARRAY_FIELDS:
            arr = getattr(self, name)
            assert arr.dtype == dt, name
            arr = np.ascontiguousarray(arr)
            setattr(self, name, arr)
            setattr(s, name, _ptr(arr))
            setattr(s, "num_" + name, len(arr))
        s.csg_root = int(self.csg_root)
        s.num_csg_nodes = len(self.csg_nodes)
        n = len(self.textures)
        self._tex = [np.ascontiguousarray(t, dtype=np.uint8) for t in self.textures]
        self._tex_ptrs = (ctypes.c_void_p * max(n, 1))(*[t.ctypes.data for t in self._tex])
        self._tex_w = (ctypes.c_int * max(n, 1))(*[t.shape[1] for t in self._tex])
        self._tex_h = (ctypes.c_int * max(n, 1))(*[t.shape[0] for t in self._tex])
        if n:
            s.texture_pixels = ctypes.cast(self._tex_ptrs, ctypes.c_void_p)
            s.texture_widths = ctypes.cast(self._tex_w, ctypes.c_void_p)
            s.texture_heights = ctypes.cast(self._tex_h, ctypes.c_void_p)
        s.num_textures = n
        s.photons = int(self.photons)
        s.photon_cell = float(self.photon_cell)
        s.caustics = float(self.caustics)
        self._view = s
        return s


def default_material(color=(0.8, 0.8, 0.8), spec=0.0, shin=32.0, amb=0.1):
    """One material record with the defaults of Scene::add_material (scene.h:303-330)."""
    m = np.zeros(1, MATERIAL)
    m["diffuse_color"] = color
    m["specular"] = spec
    m["shininess"] = shin
    m["ambient"] = amb
    m["hair_shift"] = 0.1
    m["texture_id"] = -1
    m["mask_id"] = -1
    m["normal_id"] = -1
    m["ior"] = 1.45
    m["normal_strength"] = 1.0
    return m


def make_light(kind, **kw):
    """One light record with the defaults of Scene::make_light (scene.h:391-408)."""
    l = np.zeros(1, LIGHT)
    l["direction"] = (0.0, 0.0, -1.0)
    l["color"] = (1.0, 1.0, 1.0)
    l["intensity"] = 1.0
    l["flags"] = 1
    l["texture_id"] = -1
    l["type"] = kind
    for k, v in kw.items():
        l[k] = v
    return l


@dataclass
class InstanceArrays:
    """Owns the arrays of an instancing / recursion extension and builds the
    C ``SheenSceneExt`` (the other extension fields left empty).

    mesh_triangles: object-space triangles (TRIANGLE dtype) of every mesh;
    meshes: (n, 2) int32 rows of (first triangle, triangle count);
    xforms: (k, 3, 4) float32 object-to-world maps; inst_mesh / inst_material:
    per-instance mesh index and material id; max_depth: reflect + refract
    recursion (0: the reference's depth-1 rules)."""
    mesh_triangles: np.ndarray = field(default_factory=lambda: np.zeros(0, TRIANGLE))
    meshes: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    xforms: np.ndarray = field(default_factory=lambda: np.zeros((0, 3, 4), np.float32))
    inst_mesh: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    inst_material: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    max_depth: int = 0

    def view(self) -> SheenSceneExt:
        """C view; valid while this object (and its arrays) is alive."""
        k = len(self.xforms)
        assert len(self.inst_mesh) == k and len(self.inst_material) == k
        self._tris = np.ascontiguousarray(self.mesh_triangles, dtype=TRIANGLE)
        self._meshes = (SheenMesh * max(len(self.meshes), 1))(
            *[SheenMesh(int(a), int(b)) for a, b in np.asarray(self.meshes, np.int32).reshape(-1, 2)])
        inst = (SheenInstance * max(k, 1))()
        xf = np.asarray(self.xforms, np.float32).reshape(k, 12)
        for j in range(k):
            for q in range(12):
                inst[j].xform[q] = float(xf[j, q])
            inst[j].mesh = int(self.inst_mesh[j])
            inst[j].material_id = int(self.inst_material[j])
        self._inst = inst
        x = SheenSceneExt()
        x.mesh_triangles = _ptr(self._tris)
        x.num_mesh_triangles = len(self._tris)
        x.meshes = ctypes.addressof(self._meshes) if len(self.meshes) else None
        x.num_meshes = len(self.meshes)
        x.instances = ctypes.addressof(inst) if k else None
        x.num_instances = k
        x.max_depth = int(self.max_depth)
        return x
