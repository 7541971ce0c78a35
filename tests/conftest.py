import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "multiphase-sph-solver_b200"), os.path.join(REPO, "tests"),
          os.path.join(REPO, "tests", "golden"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libsphgpu.so")
    config.addinivalue_line("markers", "reference: needs oracle/_ref/libsphref.so built from the reference")
