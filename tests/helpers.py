"""Scene loading shared by the tests."""
import os

import numpy as np

import sheen_b200 as sb

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_case(c):
    """OwnedScene of a case of golden/cases.py."""
    if "gen" in c:
        cfg, seed, detail, photons = c["gen"]
        return sb.generate_scene(cfg, seed, detail, photons)
    cwd = os.getcwd()
    os.chdir(GOLDEN)
    try:
        return sb.load_scene_file(c["file"])
    finally:
        os.chdir(cwd)


def golden(c):
    return np.load(os.path.join(GOLDEN, c["name"] + ".npz"))


def contract_scene():
    """The scene of golden/contract_scene.npz (built with the reference's
    ctypes contract, c_api_contract.py) rebuilt in memory: a 352-byte buffer
    holding the contract's SheenScene bytes with its pointer fields aimed at
    fresh copies of the recorded arrays.  Returns (buffer, keep-alive list,
    fixture)."""
    import ctypes
    f = np.load(os.path.join(GOLDEN, "contract_scene.npz"))
    buf = (ctypes.c_ubyte * 352)()          # the C struct's size (the contract's 344 bytes + the C tail)
    sb_ = f["scene_bytes"]
    ctypes.memmove(buf, sb_.ctypes.data, len(sb_))
    keep = []
    for k in f.files:
        if not k.startswith("ptr_"):
            continue
        name = k[4:]
        arr = np.array(f["arr_" + name], dtype=np.uint8, copy=True)
        keep.append(arr)
        ctypes.c_void_p.from_buffer(buf, int(f[k])).value = arr.ctypes.data
    return buf, keep, f
