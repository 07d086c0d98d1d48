"""Generates tests/golden/contract_scene.npz: a scene built with the
reference's own ctypes contract (addon_sheen/sheen_render/c_api_contract.py,
the structures the Blender add-on passes to sheen_render_scene,
engine.py:88-147), recorded as raw bytes so that tests on machines without
the reference tree can hand this library exactly what the add-on would.

Run where the reference tree is present:
    SHEEN_REFERENCE=/path/to/reference python tests/golden/make_contract_fixture.py

Contents:
  scene_bytes       the ctypes SheenScene as the contract lays it out
  ptr_<field>       byte offset of each pointer field in scene_bytes
  arr_<field>       the bytes each pointer field points at
  sizeof_<Class>    ctypes sizes of the contract's structures (the
                    HeightField entry is the contract's 72 bytes, against 64
                    in C: with more than one heightfield the add-on's array
                    is misread, so the scene holds exactly one)
"""
import ctypes
import os
import sys

import numpy as np

REF = os.environ.get("SHEEN_REFERENCE", "/root/reference")
sys.path.insert(0, os.path.join(REF, "addon_sheen", "sheen_render"))
import c_api_contract as C  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "contract_scene.npz")


def f3(x, y, z):
    return C.Float3(x, y, z)


def build():
    keep = {}
    cam = C.CameraData()
    cam.position = f3(0.0, 3.0, -12.0)
    fwd = np.array([0.0, -3.0, 12.0]) / np.linalg.norm([0.0, -3.0, 12.0])
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    cam.forward = f3(*fwd)
    cam.right = f3(*right)
    cam.up = f3(*up)
    cam.focal_length = 35.0
    cam.sensor_width = 36.0

    mats = (C.Material * 3)()
    for i, (rgb, refl) in enumerate([((0.8, 0.3, 0.2), 0.0), ((0.3, 0.7, 0.4), 0.3), ((0.55, 0.55, 0.5), 0.0)]):
        m = mats[i]
        m.diffuse_color = f3(*rgb)
        m.specular = 0.4
        m.shininess = 40.0
        m.ambient = 0.08
        m.texture_id = -1
        m.mask_id = -1
        m.normal_id = -1
        m.reflect = refl
        m.ior = 1.0
    objs = (C.Object * 4)()
    for i, (c, r) in enumerate([((-2.5, 1.0, 0.0), 1.0), ((0.0, 1.4, 1.5), 1.4), ((2.6, 0.8, -0.5), 0.8),
                                ((1.0, 0.5, -3.0), 0.5)]):
        objs[i].type = 0
        objs[i].material_id = i % 2
        objs[i].param1 = f3(*c)
        objs[i].param2 = r
    planes = (C.Plane * 1)()
    planes[0].normal = f3(0.0, 1.0, 0.0)
    planes[0].d = 0.0
    planes[0].material_id = 2
    hfs = (C.HeightField * 1)()
    hf = hfs[0]
    hf.center = f3(0.0, 0.0, 6.0)
    hf.size_x = 14.0
    hf.size_z = 6.0
    hf.height = 1.5
    hf.freq = 5.0
    hf.octaves = 5
    hf.seed = 11
    hf.material_id = 2
    lights = (C.Light * 1)()
    L = lights[0]
    L.position = f3(6.0, 10.0, -8.0)
    L.color = f3(1.0, 1.0, 1.0)
    L.intensity = 12.566 * (36 + 100 + 64)
    L.type = 1
    L.texture_id = -1
    sc = C.SheenScene()
    sc.camera = cam
    sc.objects, sc.num_objects = objs, 4
    sc.planes, sc.num_planes = planes, 1
    sc.heightfields, sc.num_heightfields = hfs, 1
    sc.materials, sc.num_materials = mats, 3
    sc.lights, sc.num_lights = lights, 1
    sc.csg_root = -1
    keep.update(objects=objs, planes=planes, heightfields=hfs, materials=mats, lights=lights)
    return sc, keep


def main():
    sc, keep = build()
    out = {"scene_bytes": np.frombuffer(ctypes.string_at(ctypes.addressof(sc), ctypes.sizeof(sc)), np.uint8)}
    for name, arr in keep.items():
        out["ptr_" + name] = np.int64(getattr(C.SheenScene, name).offset)
        out["arr_" + name] = np.frombuffer(ctypes.string_at(ctypes.addressof(arr), ctypes.sizeof(arr)), np.uint8)
    for cls in ("SheenScene", "HeightField", "Object", "Material", "Light", "Plane", "CameraData"):
        out["sizeof_" + cls] = np.int64(ctypes.sizeof(getattr(C, cls)))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, {k: int(v) for k, v in out.items() if k.startswith("sizeof_")})


if __name__ == "__main__":
    main()
