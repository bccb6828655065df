import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test (tens of seconds)")


# summary lines that tests add (report_line fixture); printed after the run
# whatever the capture mode, so the measured errors are on record without -s
_SUMMARY = []


@pytest.fixture
def report_line():
    return _SUMMARY.append


def pytest_terminal_summary(terminalreporter):
    if _SUMMARY:
        terminalreporter.section("measured errors")
        for line in _SUMMARY:
            terminalreporter.write_line(line)


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
