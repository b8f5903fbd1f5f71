import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libgemini_b200.so")


# The sub-steps outside the fused hot path (compression, source/loss rates and solves, the
# full step composed of them) run after the hot-path tests, so that under -x a failure there
# stops the run only once the hot path's own results are in.  test_zz_no_alloc stays last.
LATE_MODULES = ("test_gpu_clock", "test_gpu_compression", "test_gpu_sources", "test_gpu_rates", "test_gpu_fullstep",
                "test_zz_no_alloc")


def pytest_collection_modifyitems(config, items):
    def rank(it):
        name = it.module.__name__.rsplit(".", 1)[-1] if it.module else ""
        return LATE_MODULES.index(name) + 1 if name in LATE_MODULES else 0

    items.sort(key=rank)
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
