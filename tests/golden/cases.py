"""Parity cases shared by the golden-fixture generator and the tests.

Each case names a scene (a synthetic workload generator with its seed and
detail, or a .sheen file in this directory) and a small render size that
the CPU checkers finish in seconds.
"""
CASES = [
    dict(name="spheres_1spp", gen=(0, 1, 0, 0), W=64, H=48, aa=1),
    dict(name="spheres_4spp", gen=(0, 2, 0, 0), W=48, H=36, aa=4),
    dict(name="spheres_9spp", gen=(0, 3, 0, 0), W=32, H=24, aa=9),
    dict(name="mesh_l3", gen=(1, 1, 3, 0), W=64, H=36, aa=1),
    dict(name="analytic", gen=(2, 1, 0, 0), W=48, H=27, aa=1),
    dict(name="caustics_20k", gen=(3, 1, 0, 20000), W=64, H=36, aa=1),
    dict(name="features_a", file="features_a.sheen", W=96, H=72, aa=1),
    dict(name="features_b", file="features_b.sheen", W=80, H=60, aa=4),
]
