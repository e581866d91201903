import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device; runs the product kernels")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build (or reuse) the in-tree native libraries once per session."""
    from libuipc_b200 import build

    build.build_scene()
    from oracle import build_oracle

    build_oracle.build_oracle_lib()
    if not os.path.exists(os.path.join(ROOT, "libuipc_b200", "_lib", "libb200solve.so")):
        build.build_solve()
    yield


@pytest.fixture(scope="session")
def cube10():
    from libuipc_b200 import scene

    return scene.cube_on_ground(10, seed=0)


@pytest.fixture(scope="session")
def cube5():
    from libuipc_b200 import scene

    return scene.cube_on_ground(5, seed=3)


@pytest.fixture(scope="session")
def stack_small():
    from libuipc_b200 import scene

    return scene.stacked_cubes(8, 3, seed=1)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch.device("cuda:0")


@pytest.fixture()
def solver(cuda):
    from libuipc_b200.linear_system import Solver

    s = Solver(0)
    yield s
    s.close()


def to_dev(a, dev, dtype=None):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(dev)
