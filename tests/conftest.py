import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the sm_100a library")
    config.addinivalue_line("markers", "slow: long-running CPU case")


def pytest_sessionfinish(session, exitstatus):
    """Write the parity comparisons recorded by tests/test_gpu_parity.py's
    assert_state_close (errors, oracle twin floors, tolerances) as JSON lines
    to $KYN_PARITY_REPORT, when that is set."""
    path = os.environ.get("KYN_PARITY_REPORT")
    mod = sys.modules.get("tests.test_gpu_parity")
    if not path or mod is None or not getattr(mod, "REPORT", None):
        return
    with open(path, "w") as f:
        for r in mod.REPORT:
            f.write(json.dumps(r) + "\n")
