import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libcelgpu.so")


@pytest.fixture(scope="session")
def ref_poisson():
    """Known-answer fixtures produced by the reference's own C generator."""
    out = {}
    for f in sorted(os.listdir(GOLDEN)):
        if f.startswith("ref_poisson7_") and f.endswith(".npz"):
            d = np.load(os.path.join(GOLDEN, f))
            out[f[len("ref_poisson7_"):-4]] = {k: d[k] for k in d.files}
    return out


@pytest.fixture(scope="session")
def gpu():
    """(celgpu module, Handle on torch's current stream, torch) for GPU tests."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cel_v3_b200 import celgpu
    torch.cuda.init()
    h = celgpu.Handle(0, torch.cuda.current_stream().cuda_stream)
    yield celgpu, h, torch
    torch.cuda.synchronize()
    h.close()
