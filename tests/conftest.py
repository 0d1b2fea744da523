import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

__graft_entry__.package()
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


@pytest.fixture(scope="session")
def prepare():
    from film_juicer_b200 import prepare as p

    return p


@pytest.fixture(scope="session")
def recipes(prepare):
    return {name: prepare.PreparedRecipe.load(os.path.join(GOLDEN, f"recipe_{name}.npz"))
            for name in ("direct", "print")}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc

    orc.load()
    return orc


@pytest.fixture(scope="session")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
