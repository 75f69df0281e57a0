"""Shared test set-up: the `gpu` marker, import paths and the oracle build."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _build_missing():
    """Builds what the tests load when it is missing: the C oracle, libaxr.so
    (nvcc cross-compiles without a GPU) and, where the reference checkout is
    present, its kernels for the CPU (oracle/_ref)."""
    import shutil
    import oracle as O
    O.build_oracle()
    try:
        from axi_visualizer_b200 import build as B
        if B.needs_build() and (os.path.exists(B.NVCC) or shutil.which(B.NVCC)):
            B.build()
    except Exception as e:          # a broken build shows up in the tests that load the library
        print(f"conftest: libaxr.so not built: {e}")
    if not O.ref_available():
        try:
            import build_ref
            build_ref.build()
        except Exception as e:
            print(f"conftest: reference kernels not built: {e}")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libaxr.so")
    _build_missing()


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    import oracle as O
    O.build_oracle()
    yield
