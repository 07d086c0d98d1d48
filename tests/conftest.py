import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

# the reference source tree (loader and layout tests read it when present)
REFERENCE = os.environ.get("SHEEN_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "small_frames: runs with the library's default small-frame megakernel rule")


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="session")
def reference_tree():
    if not os.path.isdir(REFERENCE):
        pytest.skip("reference source tree not present on this machine")
    return REFERENCE


@pytest.fixture(autouse=True)
def _queue_pipeline(request):
    """GPU tests exercise the wavefront form's queue pipeline at every frame
    size: the small-frame switch to the megakernel (wave.mega_samples) is
    turned off for them, and tests marked small_frames run with the
    library's default rule."""
    if request.node.get_closest_marker("gpu") is None or request.node.get_closest_marker("small_frames"):
        yield
        return
    import sheen_b200 as sb
    old = sb.tune_get("wave.mega_samples")
    sb.tune_set("wave.mega_samples", 0)
    try:
        yield
    finally:
        sb.tune_set("wave.mega_samples", old)
