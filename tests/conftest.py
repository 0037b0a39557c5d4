import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    """The checker: the reference build when present, else the C restatement."""
    import oracle_lib as O
    return O


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(HERE, "golden", "splice_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ext_golden():
    import json
    with open(os.path.join(HERE, "golden", "ext_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def hmm_golden():
    import json
    with open(os.path.join(HERE, "golden", "hmm_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def gapless_golden():
    """Scores of the reference's gapless kernel with the generator that regenerates its inputs."""
    import json
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_gapless_golden as G
    with open(os.path.join(HERE, "golden", "gapless_golden.json")) as f:
        return json.load(f), G
