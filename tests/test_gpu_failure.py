"""Failure detection on the GPU without faulting it: a bounded device wait
that can never be satisfied ends with CELG_ERR_TIMEOUT after its limit, the
host reads the status, and the same handle then solves normally."""
import time

import numpy as np
import pytest

from cel_v3_b200 import synth

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(gpu):
    celgpu, h, torch = gpu
    t0 = time.perf_counter()
    status = h.check_bounded_wait(200)
    dt = time.perf_counter() - t0
    assert status == celgpu.ERR_TIMEOUT
    assert 0.15 < dt < 5.0
    rp, ci, v = synth.poisson7(12)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    b = torch.ones(rp.size - 1, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    info = h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), eps_rel=1e-8)
    assert info.status == celgpu.OK and info.verified_relres <= 1.5e-8
    m.destroy()


def test_invalid_arguments_return_status_not_abort(gpu):
    celgpu, h, torch = gpu
    with pytest.raises(celgpu.CelgError) as e:
        h.check_bounded_wait(0)
    assert e.value.status == celgpu.ERR_ARG
    rp, ci, v = synth.poisson7(4)
    m = h.matrix_from_csr(rp, ci, v)            # no Jacobi yet
    b = torch.ones(rp.size - 1, dtype=torch.float64, device="cuda")
    with pytest.raises(celgpu.CelgError) as e:
        h.pcg_jacobi(m, b.data_ptr(), b.data_ptr())
    assert e.value.status == celgpu.ERR_STATE
    with pytest.raises(celgpu.CelgError) as e:
        h.spmv(m, b.data_ptr(), b.data_ptr(), fmt=celgpu.FMT_JAD)   # JAD not built
    assert e.value.status == celgpu.ERR_STATE
    m.destroy()
