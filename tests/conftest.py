"""Shared test setup.

Markers: `gpu` tests need a CUDA device (B200) and call the native library
through its C ABI; everything else runs on the CPU.  The CPU oracle library
(oracle/libvnlb_oracle.so) is built on demand with make."""
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "vapoursynth-vnlb_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the native library")
    if not (ROOT / "oracle" / "libvnlb_oracle.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np

    data = np.load(ROOT / "tests" / "golden" / "ref_outputs.npz")
    meta = json.loads(str(data["meta"]))
    return data, meta


def pytest_collection_modifyitems(config, items):
    # run files whose names sort last (test_zz_*) after everything else
    items.sort(key=lambda item: 1 if Path(str(item.fspath)).name.startswith("test_zz_") else 0)
