import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = ["cornell", "zoo", "env", "hf", "cornell_pt", "env_pt", "cornell_ls", "hf_ls", "phong", "phong_pt",
            "phong_ls", "srgb", "lens", "lens_ls"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build(with_reference=False)
    return oracle


@pytest.fixture(scope="session")
def wr_lib():
    import wurstrenderer_b200 as wr
    from wurstrenderer_b200 import build
    build.build()
    return wr


def golden_scene(name):
    import json
    with open(os.path.join(GOLDEN, name + "_meta.json")) as f:
        meta = json.load(f)
    return os.path.join(GOLDEN, meta["scene"]), meta
