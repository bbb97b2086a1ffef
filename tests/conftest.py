import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)

_REPORT = []


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU runs")


@pytest.fixture
def parity_report(request):
    """record(quantity, measured, tolerance): the measured parity figures of a test; with
    LSD_PARITY_REPORT=<path> set they are written there as JSON when the session ends."""
    def record(quantity, measured, tolerance=None):
        _REPORT.append({"test": request.node.nodeid, "quantity": quantity, "measured": float(measured),
                        "tolerance": tolerance})
    return record


def pytest_sessionfinish(session, exitstatus):
    path = os.environ.get("LSD_PARITY_REPORT")
    if path and _REPORT:
        with open(path, "w") as fh:
            json.dump(_REPORT, fh, indent=1)
