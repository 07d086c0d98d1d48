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
