"""Block-Jacobi preconditioner: the oracle's block inverse (CPU), the device
set-up and apply bit for bit against it, and block-Jacobi PCG bit for bit
against a composition of oracle pieces in the device's reduction order."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R
from tests.helpers import random_csr, spd_from_pattern

BLOCKS = [1, 2, 4, 8, 16, 32]


def dense(rp, ci, v):
    n = rp.size - 1
    A = np.zeros((n, n))
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            A[i, ci[k]] = v[k]
    return A


@pytest.mark.parametrize("bs", BLOCKS + [3, 5])
def test_oracle_block_inverse_inverts_the_blocks(bs):
    rp, ci, v = synth.poisson7(6, 5, 4)
    inv, ok = R.block_jacobi_inv(rp, ci, v, bs)
    assert ok
    A = dense(rp, ci, v)
    n = A.shape[0]
    for b0 in range(0, n, bs):
        nb = min(bs, n - b0)
        D = A[b0:b0 + nb, b0:b0 + nb]
        assert np.abs(inv[b0:b0 + nb, :nb] @ D - np.eye(nb)).max() < 1e-13
        assert not inv[b0:b0 + nb, nb:].any()
    r = np.random.default_rng(0).standard_normal(n)
    z = R.block_jacobi_apply(inv, r)
    zr = np.concatenate([np.linalg.solve(A[b0:b0 + bs, b0:b0 + bs], r[b0:b0 + bs])
                         for b0 in range(0, n, bs)])
    assert np.abs(z - zr).max() <= 1e-13 * np.abs(zr).max()


def test_oracle_block_extraction_stops_at_the_first_column_right_of_the_block():
    # row 0 stores (0, 5) before (0, 1): the scan ends at column 5, so the
    # in-block entry (0, 1) after it is not part of the block
    rp = np.array([0, 3, 5], np.int32)
    ci = np.array([0, 5, 1, 0, 1], np.int32)
    v = np.array([4.0, 9.0, -1.0, -1.0, 4.0])
    n = 2
    inv, ok = R.block_jacobi_inv(rp, ci, v, 2)
    assert ok
    D = np.array([[4.0, 0.0], [-1.0, 4.0]])
    assert np.allclose(inv @ D, np.eye(2), atol=1e-15)


def test_oracle_zero_pivot_is_reported():
    rp, ci, v = synth.poisson7(4, 3, 2)
    v = v.copy()
    v[rp[0]:rp[1]][ci[rp[0]:rp[1]] == 0] = 0.0   # zero diagonal in the first block
    _, ok = R.block_jacobi_inv(rp, ci, v, 2)
    assert not ok


def mirror_pcg(rp, ci, v, inv, b, eps_rel, iter_max):
    dot = lambda a, c: R.dot(np.ascontiguousarray(a), np.ascontiguousarray(c), red=R.RED_TREE)
    spmv = lambda x: R.spmv_csr(rp, ci, v, x)
    n = b.size
    x = np.zeros(n)
    r = b - (0.0 + spmv(x))
    z = R.block_jacobi_apply(inv, r)
    p = z.copy()
    eps = eps_rel * np.sqrt(dot(b, b))
    alpha, norm = dot(r, z), np.sqrt(dot(r, r))
    hist, it = [norm], 0
    go = lambda: it < iter_max and abs(alpha) > R.REAL_SMALL and norm > eps
    while go():
        vv = 0.0 + spmv(p)
        sg = alpha / dot(vv, p)
        x = x + sg * p
        r = r + (-sg) * vv
        z = R.block_jacobi_apply(inv, r)
        rz, rr = dot(r, z), dot(r, r)
        beta = rz / alpha
        alpha, norm = rz, np.sqrt(rr)
        it += 1
        hist.append(norm)
        if go():
            p = beta * p + z
    return x, it, np.array(hist)


def problems():
    rng = np.random.default_rng(21)
    _, (kx, ky, kz) = synth.lognormal_faces(rng, 13, 11, 9)
    yield "diffusion", synth.diffusion7(13, 11, 9, kx, ky, kz), rng.uniform(-1, 1, 13 * 11 * 9)
    rp, ci, v = spd_from_pattern(*random_csr(2500, rng, max_len=8, empty_frac=0.0))
    yield "random", (rp, ci, v), rng.uniform(-1, 1, 2500)


@pytest.mark.gpu
@pytest.mark.parametrize("bs", BLOCKS)
def test_gpu_block_inverse_and_apply_bitexact(gpu, bs):
    celgpu, h, torch = gpu
    for name, (rp, ci, v), b in problems():
        m = h.matrix_from_csr(rp, ci, v).block_jacobi(bs)
        inv, ok = R.block_jacobi_inv(rp, ci, v, bs)
        assert ok and np.array_equal(m.get_block_jacobi(), inv), name
        r = np.random.default_rng(bs).standard_normal(rp.size - 1)
        rd, zd = torch.from_numpy(r).cuda(), torch.zeros(rp.size - 1, dtype=torch.float64, device="cuda")
        h.block_jacobi_apply(m, rd.data_ptr(), zd.data_ptr())
        assert np.array_equal(zd.cpu().numpy(), R.block_jacobi_apply(inv, r)), name
        m.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("bs", [1, 4, 8, 32])
def test_gpu_block_jacobi_pcg_bitexact(gpu, bs):
    celgpu, h, torch = gpu
    for name, (rp, ci, v), b in problems():
        m = h.matrix_from_csr(rp, ci, v).jacobi().block_jacobi(bs)
        bd = torch.from_numpy(b).cuda()
        xd = torch.zeros_like(bd)
        info = h.pcg_jacobi(m, bd.data_ptr(), xd.data_ptr(), history=True, eps_rel=1e-10,
                            iter_max=3000, precond=celgpu.PRECOND_BLOCK_JACOBI)
        inv, _ = R.block_jacobi_inv(rp, ci, v, bs)
        xo, ito, ho = mirror_pcg(rp, ci, v, inv, b, 1e-10, 3000)
        assert info.status == celgpu.OK, name
        assert info.iter_done == ito, name
        assert np.array_equal(info.history, ho), name
        assert np.array_equal(xd.cpu().numpy(), xo), name
        assert info.verified_relres <= 1e-8
        m.destroy()


@pytest.mark.gpu
def test_gpu_block_jacobi_rejections(gpu):
    celgpu, h, torch = gpu
    rp, ci, v = synth.poisson7(6)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    with pytest.raises(celgpu.CelgError):
        m.block_jacobi(3)                      # not a divisor of the warp width
    b = torch.ones(rp.size - 1, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    with pytest.raises(celgpu.CelgError):      # no block inverse built yet
        h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), precond=celgpu.PRECOND_BLOCK_JACOBI)
    m.block_jacobi(4)
    with pytest.raises(celgpu.CelgError):      # FP32 forms keep point Jacobi
        h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), precond=celgpu.PRECOND_BLOCK_JACOBI,
                     precision=celgpu.PREC_FP32_RU)
    m.destroy()
