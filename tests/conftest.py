import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "simint-generator_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(session, config, items):
    """The comparisons against the reference's generated library (the
    longest GPU tests, each in a child process) run after every other test,
    so that a stop-at-first-failure run has covered the rest first."""
    last = [it for it in items if os.path.basename(str(it.fspath)) == "test_gpu_reference.py"]
    if last:
        keep = [it for it in items if os.path.basename(str(it.fspath)) != "test_gpu_reference.py"]
        items[:] = keep + last
