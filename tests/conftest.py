import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def junit():
    import json
    return json.loads((ROOT / "tests" / "golden" / "reference_junit.json").read_text())


@pytest.fixture(scope="session")
def refshim_fx():
    import numpy as np
    return dict(np.load(ROOT / "tests" / "golden" / "global_refshim.npz"))


@pytest.fixture(scope="session")
def shape_fx():
    import numpy as np
    return dict(np.load(ROOT / "tests" / "golden" / "shape_refshim.npz"))


@pytest.fixture(scope="session")
def volume_fx():
    import numpy as np
    return dict(np.load(ROOT / "tests" / "golden" / "volume_refshim.npz"))


def volume_cases(fx):
    """(name, bw, bh, bd) of the cases in volume_refshim.npz."""
    for n in sorted({k.split("/")[0] for k in fx}):
        bw, bh, bd = (int(v) for v in n.rsplit("_", 1)[1].split("x"))
        yield n, bw, bh, bd


@pytest.fixture(scope="session")
def relevance_fx():
    import numpy as np
    return dict(np.load(ROOT / "tests" / "golden" / "relevance_refshim.npz"))
