import json
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
for p in (ROOT / "yao-rs_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the CUDA library)")
    # build the library and the oracle if they are missing (nvcc/gcc present here and on GPU hosts)
    lib = ROOT / "yao-rs_b200" / "yao_rs" / "libyao_gpu.so"
    if not lib.exists():
        sys.path.insert(0, str(ROOT / "yao-rs_b200"))
        import build as _b  # noqa: E402
        _b.build()
    import oracle as _o  # noqa: E402
    if not _o.LIB.exists():
        _o.build()


def load_golden(name):
    return json.loads((GOLDEN / f"{name}.json").read_text())


@pytest.fixture(scope="session")
def golden():
    return load_golden
