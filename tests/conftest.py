"""Test configuration.

Markers:
  gpu  -- needs a B200 (calls into libmublis' device path).  The rest of the
          suite (oracle pins, golden vectors, host logic, ABI surface) runs on
          any CPU host.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: requires a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def lib():
    import mublis_b200 as mb
    return mb.load()


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import oracle as orc
    path = orc.ref_lib_path("avx2")
    if not path.is_file():
        pytest.skip(f"reference build {path} not present")
    return orc.reference("avx2")
