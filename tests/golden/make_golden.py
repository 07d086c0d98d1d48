"""Regenerates the golden fixtures in this directory.

For every case of cases.py the reference's own per-pixel code, compiled for
the host (oracle/_ref/libsheen_ref_host.so, built by `make -C oracle ref`
from the reference sources), renders the RGBA image and the primary-ray
hits; they are stored as <name>.npz.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import sheen_b200 as sb  # noqa: E402
from cases import CASES  # noqa: E402
from oracle_bindings import RefHost  # noqa: E402


def load_case(c):
    if "gen" in c:
        cfg, seed, detail, photons = c["gen"]
        return sb.generate_scene(cfg, seed, detail, photons)
    cwd = os.getcwd()
    os.chdir(HERE)
    try:
        return sb.load_scene_file(c["file"])
    finally:
        os.chdir(cwd)


def main():
    ref = RefHost()
    for c in CASES:
        s = load_case(c)
        h = ref.scene(s.view_ptr)
        img = ref.render(h, c["W"], c["H"], c["aa"])
        obj, mat, t = ref.primary_hits(h, c["W"], c["H"], c["aa"])
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), rgba=img, obj=obj, mat=mat, t=t)
        print(c["name"], img[..., :3].mean())


if __name__ == "__main__":
    main()
