import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through libits.so")


@pytest.fixture(scope="session")
def ctx():
    from its_b200 import Context
    c = Context(0)
    yield c
    c.close()


def prepared_mesh(name, **kw):
    """Mesh normalised to the unit cube with the reference's cubic box (BaseModel ctor order)."""
    import oracle
    from its_b200 import meshes
    if name in ("small", "c0", "c1", "c2"):
        V, F = meshes.config_mesh(name)
    elif name == "torus":
        V, F = meshes.torus_mesh(**kw)
    elif name == "knot":
        V, F = meshes.torus_knot_tube(**kw)
    elif name == "superquadric":
        V, F = meshes.superquadric_mesh(**kw)
    elif name == "sphere":
        V, F = meshes.sphere_mesh(**kw)
    else:
        raise KeyError(name)
    V = oracle.model_to_unit_cube(V)
    o, e, w = oracle.uniform_bbox(V)
    return V, F, o, w
