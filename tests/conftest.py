import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference project's checkout (JackDanger/gzippy), when one is mounted:
# GZIPPY_REFERENCE names its root (default: a "reference" directory beside
# this repository); tests that read its fixtures skip without it.
REFERENCE_ROOT = os.environ.get("GZIPPY_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
REFERENCE_BLOCKS = os.path.join(REFERENCE_ROOT, "corpus", "silesia_blocks")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger inputs")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
