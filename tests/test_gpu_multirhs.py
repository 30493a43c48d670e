"""Multi-right-hand-side Jacobi-PCG (celg_pcg_multirhs): bit-exact against a
composition of oracle pieces with the documented per-column reduction order
(warp-sequential tiles), and within 1e-10 of single-vector solves."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def dot_cols(A, B):
    """Per column: warp w of a 1024-row tile sums rows q*256 + w*32 + r in
    (q, r) order from 0.0, tile partial = warp 0 + ... + warp 7, tiles reduced
    in the single-vector order."""
    n, k = A.shape
    nt = (n + 1023) // 1024
    P = np.zeros((nt * 1024, k))
    P[:n] = A * B
    P = P.reshape(nt, 4, 8, 32, k)
    acc = np.zeros((nt, 8, k))
    for q in range(4):
        for r in range(32):
            acc = acc + P[:, q, :, r, :]
    tot = acc[:, 0, :]
    for w in range(1, 8):
        tot = tot + acc[:, w, :]
    return np.array([R.reduce256(tot[:, c]) for c in range(k)])


def mirror(rp, ci, v, B, eps_rel, iter_max):
    n, k = B.shape
    J = R.jacobi(R.diag(rp, ci, v))[:, None]
    spmm = lambda X: np.stack([R.spmv_csr(rp, ci, v, X[:, c]) for c in range(k)], 1)
    X = np.zeros((n, k))
    bn = np.sqrt(dot_cols(B, B))
    eps = eps_rel * bn
    Rr = B - (0.0 + spmm(X))
    Z = Rr * J
    P = Z.copy()
    alpha = dot_cols(Rr, Z)
    norm = np.sqrt(dot_cols(Rr, Rr))
    it = np.zeros(k, int)
    go = lambda c: it[c] < iter_max and abs(alpha[c]) > R.REAL_SMALL and norm[c] > eps[c]
    active = np.array([go(c) for c in range(k)])
    while active.any():
        V = spmm(P)
        pv = dot_cols(V, P)
        sigma = np.zeros(k)
        for c in np.flatnonzero(active):
            sigma[c] = alpha[c] / pv[c]
            X[:, c] = X[:, c] + sigma[c] * P[:, c]
            Rr[:, c] = Rr[:, c] + (-sigma[c]) * V[:, c]
        Z = Rr * J
        rz, rr = dot_cols(Rr, Z), dot_cols(Rr, Rr)
        beta = np.zeros(k)
        for c in np.flatnonzero(active):
            beta[c] = rz[c] / alpha[c]
            alpha[c] = rz[c]
            norm[c] = np.sqrt(rr[c])
            it[c] += 1
            active[c] = go(c)
        for c in np.flatnonzero(active):
            P[:, c] = beta[c] * P[:, c] + Rr[:, c] * J[:, 0]
    return X, it, norm


@pytest.mark.parametrize("case", ["poisson12_k5", "diffusion_k32"])
def test_multirhs_bitexact_and_close_to_single(gpu, case):
    celgpu, h, torch = gpu
    rng = np.random.default_rng(5)
    if case == "poisson12_k5":
        rp, ci, v = synth.poisson7(12)
        k = 5
    else:
        _, (kx, ky, kz) = synth.lognormal_faces(rng, 9, 10, 11)
        rp, ci, v = synth.diffusion7(9, 10, 11, kx, ky, kz)
        k = 32
    n = rp.size - 1
    B = rng.uniform(-1.0, 1.0, (n, k))
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-10, iter_max=2000)
    Xo, ito, normo = mirror(rp, ci, v, B, 1e-10, 2000)
    X = Xd.cpu().numpy()
    assert np.array_equal(X, Xo)
    assert [i.iter_done for i in infos] == list(ito)
    # the loop may also end on the reference's absolute |r.z| guard
    # (cel_cgalg_module.f90:248) once ||r|| is tiny: the true residual stays small
    assert all(i.status == celgpu.OK and i.verified_relres <= 1e-8 for i in infos)
    for c in range(k):
        xs = dev(torch, np.zeros(n))
        one = h.pcg_jacobi(m, dev(torch, B[:, c]).data_ptr(), xs.data_ptr(), eps_rel=1e-10, iter_max=2000)
        assert abs(one.iter_done - infos[c].iter_done) <= 1
        assert np.abs(xs.cpu().numpy() - X[:, c]).max() <= 1e-9 * np.abs(X[:, c]).max()
    m.destroy()


@pytest.mark.parametrize("cfg", range(8))
def test_every_spmm_variant_is_bitexact(gpu, cfg, monkeypatch):
    """Each launch variant the autotuner can pick (forced with
    CELG_SPMM_CFG) gives the mirror's bits, including rows longer than the
    gather chunk."""
    celgpu, h, torch = gpu
    monkeypatch.setenv("CELG_SPMM_CFG", str(cfg))
    rng = np.random.default_rng(9)
    from tests.helpers import random_csr, spd_from_pattern
    rp, ci, v = spd_from_pattern(*random_csr(3000, rng, max_len=9, empty_frac=0.0, long_rows=3,
                                             long_len=40))
    n, k = rp.size - 1, 7
    B = rng.uniform(-1.0, 1.0, (n, k))
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-10, iter_max=300)
    Xo, ito, _ = mirror(rp, ci, v, B, 1e-10, 300)
    m.destroy()
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == list(ito)
