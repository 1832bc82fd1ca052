import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "nanovdb-editor_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as oracle_py

    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def vox_ctx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from nanovdb_editor.vox import VoxContext

    ctx = VoxContext(0)
    yield ctx
    ctx.close()
