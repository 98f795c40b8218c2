import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "last: runs after every other test of the session")


def pytest_collection_modifyitems(session, config, items):
    """Tests marked `last` run at the end (in their collected order), so that under -x a
    failure there stops nothing else."""
    items[:] = [i for i in items if not i.get_closest_marker("last")] + \
        [i for i in items if i.get_closest_marker("last")]


@pytest.fixture(scope="session")
def hb():
    import __graft_entry__ as ge
    mod = ge.load_package()
    from hevc_b200 import build
    build.build_synth()
    return mod


@pytest.fixture(scope="session")
def port(hb):
    import oracle
    if not os.path.exists(oracle.PORT_SO):
        oracle.build(with_ref=False)
    return oracle.port()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(HERE, "golden", "digests.json")) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session")
def gpu_ctx(hb):
    from hevc_b200 import build
    build.build_gpu()
    ctx = hb.Context(0)
    yield ctx
    ctx.close()
