"""Shared test setup: import paths, the `gpu` marker, built artefacts."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def lib():
    import aperture_b200
    return aperture_b200.load_library()


@pytest.fixture(scope="session")
def box_objects():
    import scenes
    return scenes.box_scene()


@pytest.fixture(scope="session")
def small_spheres_objects():
    import scenes
    return scenes.spheres_scene(n_spheres=120, n_lights=8, box=20.0)


@pytest.fixture(scope="session")
def config2_objects():
    """Config 2 at full size: 800 icospheres x 1280 triangles, ground quad,
    16 emissive spheres (scenes.spheres_scene() defaults)."""
    import scenes
    return scenes.spheres_scene()
