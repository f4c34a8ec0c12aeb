import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def golden():
    """The 32 rANS streams harvested from the reference's container fixtures."""
    import json

    here = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(here, "fixture_streams.json")) as f:
        index = json.load(f)["streams"]
    with open(os.path.join(here, "fixture_streams.bin"), "rb") as f:
        blob = f.read()
    return [(e, blob[e["offset"]:e["offset"] + e["length"]]) for e in index]
