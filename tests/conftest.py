"""Shared test setup: import paths, the gpu marker, library builds."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("", "block-daglu_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


# The autotuner's cache goes to a per-run temporary file, not $HOME.
if "BDLU_TUNE_CACHE" not in os.environ:
    import tempfile
    os.environ["BDLU_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="bdlu-tune-"), "tune.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running parity case")


def _ensure_built():
    import build as bdlu_build  # block-daglu_b200/build.py
    bdlu_build.build()
    import oracle
    oracle.load()


_ensure_built()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_device():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return 0
