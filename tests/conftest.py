import os
import sys
import warnings
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
warnings.filterwarnings("ignore", category=DeprecationWarning)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libpmb200.so")
    config.addinivalue_line("markers", "slow: long-running case")


GOLDEN = ROOT / "tests" / "golden"


@pytest.fixture(scope="session")
def golden():
    import json
    import numpy as np

    def load(name):
        z = np.load(GOLDEN / f"{name}.npz")
        d = {k: z[k] for k in z.files if k != "meta"}
        d["meta"] = json.loads(str(z["meta"]))
        return d
    return load
