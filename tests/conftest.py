import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "bigdft-suite_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

# the reference source tree, for the tests that re-derive pins from it; unset:
# those tests skip and the committed fixtures stand
_ref = os.environ.get("WVLH_REFERENCE_ROOT")
REFERENCE = Path(_ref) if _ref else Path("/nonexistent-reference-tree")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def wctx(torch_cuda):
    from wvlh.batch import Context
    ctx = Context(0)
    yield ctx
    ctx.close()
