import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "daggerfft.jl_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libdfft")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly (no fallback) when no GPU is visible; the CPU
    # suite selects them out with -m "not gpu".
    pass
