"""GPU parity against the oracle at the full sizes of the benchmark
configurations (the other parity tests run at 32^3 and below).

  * 256^3 Poisson (16,777,216 rows, 117,047,296 non-zeros): the CSR and JAD
    SpMV bit for bit against the oracle's row sums, the JAD permutation bit
    for bit against the reference's stable descending-length sort, and the
    plain FP64 Jacobi-PCG to rel-res 1e-8 -- bit for bit against the oracle
    in the GPU's reduction order, and within 1e-10 relative (solution and
    residual history, same iteration count +-1) against the reference's own
    order with one OpenMP worker per host core but one
    (src/fcgalg/cel_cgalg_module.f90:205-304, reductions as
    src/fop/cel_fop_vec_distr_module.f90:724-775 with the worker chunks of
    src/fbase/cel_omp_shared_work_module.f90:183-232).
  * the largest system (95^3) of the 64-system seed-4 batch, solved inside
    the whole batched launch, against the oracle's solve of that system.
  * two columns of the 128^3 x 32 multi-right-hand-side solve against the
    oracle's single-vector solves of those columns.
"""
import os

import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R

pytestmark = pytest.mark.gpu

WORKERS = max(1, (os.cpu_count() or 2) - 1)  # the reference's idle master + workers


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def close_to_reference_order(info, x, io, xo, tol=1e-10):
    """Parity of a PCG solve with the reference's reduction order: iteration
    count within one, history and solution within tol relative."""
    assert abs(io["iter_done"] - info.iter_done) <= 1
    k = min(len(io["history"]), len(info.history))
    hist = np.abs(info.history[:k] - io["history"][:k]) / io["history"][:k]
    assert hist.max() < tol, hist.max()
    assert np.abs(x - xo).max() <= tol * np.abs(xo).max()


@pytest.fixture(scope="module")
def poisson256(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, xt = synth.plain(256, 1)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    yield rp, ci, v, xt, m
    m.destroy()
    torch.cuda.empty_cache()


def test_spmv_and_jad_256_bitexact(gpu, poisson256):
    celgpu, h, torch = gpu
    rp, ci, v, xt, m = poisson256
    n = rp.size - 1
    assert n == 16_777_216 and int(rp[-1]) == 117_047_296
    y_ref = R.spmv_csr(rp, ci, v, xt, nworkers=WORKERS)
    xd = dev(torch, xt)
    y = torch.empty_like(xd)
    h.spmv(m, xd.data_ptr(), y.data_ptr())
    assert np.array_equal(y.cpu().numpy(), y_ref)
    perm = m.to_jad()
    perm_ref, mmax = R.jad_perm(rp)
    assert mmax == 7
    assert np.array_equal(perm, perm_ref)
    y.zero_()
    h.spmv(m, xd.data_ptr(), y.data_ptr(), fmt=celgpu.FMT_JAD)
    assert np.array_equal(y.cpu().numpy(), y_ref)      # diagonal order = stored order per row


def test_pcg_256_tree_bitexact_and_reference_order(gpu, poisson256):
    celgpu, h, torch = gpu
    rp, ci, v, xt, m = poisson256
    n = rp.size - 1
    b = R.spmv_csr(rp, ci, v, xt, nworkers=WORKERS)
    bd, xd = dev(torch, b), torch.zeros(n, dtype=torch.float64, device="cuda")
    info = h.pcg_jacobi(m, bd.data_ptr(), xd.data_ptr(), history=True, eps_rel=1e-8,
                        iter_max=5000, x0_mode=celgpu.X0_ZERO)
    assert info.status == celgpu.OK and info.verified_relres <= 1e-8
    x = xd.cpu().numpy()
    A, J = R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v))
    xo, io = R.pcg_jacobi(A, J, b, eps_rel=1e-8, iter_max=5000, red=R.RED_TREE, nworkers=WORKERS)
    assert info.iter_done == io["iter_done"] == 597
    assert np.array_equal(info.history, io["history"])
    assert np.array_equal(x, xo)
    xs, is_ = R.pcg_jacobi(A, J, b, eps_rel=1e-8, iter_max=5000, red=R.RED_SEQ, nworkers=WORKERS)
    close_to_reference_order(info, x, is_, xs)


def test_batch_largest_system_vs_oracle(gpu):
    celgpu, h, torch = gpu
    probs = synth.batch_problems()
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for _, rp, ci, v, _ in probs]
    bs = [dev(torch, b) for *_, b in probs]
    xs = [torch.zeros_like(b) for b in bs]
    try:
        infos = h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs],
                              eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO)
        assert all(i.status == celgpu.OK for i in infos)
        big = int(np.argmax([s for s, *_ in probs]))
        side, rp, ci, v, b = probs[big]
        assert side == 95
        A, J = R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v))
        xo, io = R.pcg_jacobi(A, J, b, eps_rel=1e-8, iter_max=5000, red=R.RED_TREE,
                              nworkers=WORKERS)
        x = xs[big].cpu().numpy()
        assert infos[big].iter_done == io["iter_done"]
        assert np.array_equal(x, xo)
        xsq, is_ = R.pcg_jacobi(A, J, b, eps_rel=1e-8, iter_max=5000, red=R.RED_SEQ,
                                nworkers=WORKERS)
        assert abs(is_["iter_done"] - infos[big].iter_done) <= 1
        assert np.abs(x - xsq).max() <= 1e-10 * np.abs(xsq).max()
    finally:
        for mm in mats:
            mm.destroy()


def test_multirhs_128_k32_columns_vs_oracle(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, B = synth.multirhs_problem()
    n, k = B.shape
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd = dev(torch, B)
    Xd = torch.zeros_like(Bd)
    try:
        infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-8, iter_max=5000,
                               x0_mode=celgpu.X0_ZERO)
        assert all(i.status == celgpu.OK and i.verified_relres <= 1e-8 for i in infos)
        X = Xd.cpu().numpy()
        A, J = R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v))
        for c in (0, k - 1):
            xs, is_ = R.pcg_jacobi(A, J, np.ascontiguousarray(B[:, c]), eps_rel=1e-8,
                                   iter_max=5000, red=R.RED_SEQ, nworkers=WORKERS)
            assert abs(is_["iter_done"] - infos[c].iter_done) <= 1
            assert np.abs(X[:, c] - xs).max() <= 1e-10 * np.abs(xs).max()
    finally:
        m.destroy()
