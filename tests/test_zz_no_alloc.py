"""The allocation-free dot product (celg_dot_noalloc).

Callers whose device memory is owned by someone else (their own pool, or a
framework's caching allocator that has already committed the GPU) cannot let
the library allocate.  celg_dot_noalloc serves them: no handle, no
cudaMalloc, its reduction scratch in a fixed device array of the library.
These checks call it through the C ABI and compare it with the handle-based
celg_dot on two calls in a row (the second call must not see the first
call's scratch): the results must be identical, since both use the same
fixed reduction order.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_dot_matches_handle_dot_twice(gpu):
    celgpu, h, torch = gpu
    rng = np.random.default_rng(2026)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for n in (300_001, 4_097):  # two calls in a row, different sizes
        a = torch.from_numpy(rng.standard_normal(n)).cuda()
        b = torch.from_numpy(rng.standard_normal(n)).cuda()
        st = celgpu.dot_noalloc(n, a.data_ptr(), b.data_ptr(), out.data_ptr(), stream)
        assert st == celgpu.OK
        got = float(out.cpu()[0])
        ref = h.dot(n, a.data_ptr(), b.data_ptr())
        assert got == ref                                  # same order: bit-identical
        assert abs(got - float(torch.dot(a, b))) <= 1e-12 * float(torch.dot(a.abs(), b.abs()))


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    celgpu, h, torch = gpu
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    a = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = celgpu.lib.celg_dot_noalloc(celgpu.NOALLOC_MAX_ROWS + 1, ctypes.c_void_p(a.data_ptr()),
                                     ctypes.c_void_p(a.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), None)
    assert st == celgpu.ERR_ARG
