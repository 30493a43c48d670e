"""Multi-right-hand-side Jacobi-PCG (celg_pcg_multirhs): bit-exact against a
composition of oracle pieces with the documented per-column reduction order
(warp-sequential tiles), and within 1e-10 of single-vector solves."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R
from tests.helpers import ir_step_tolerance

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


@pytest.mark.parametrize("cfg", range(15))
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


@pytest.mark.parametrize("iter_max", [1, 6])
def test_multirhs_iteration_cap_bitexact(gpu, iter_max):
    """Columns stopped by the iteration cap still get the last x update
    (which the direction sweep applies after the update sweep stopped
    them): X equals the mirror bit for bit, columns of different speed
    included."""
    celgpu, h, torch = gpu
    rp, ci, v = synth.poisson7(11, 10, 9)
    n, k = rp.size - 1, 8
    B = np.random.default_rng(17).uniform(-1.0, 1.0, (n, k))
    B[:, 2] = 0.0                            # stops at once (alpha = 0)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-12, iter_max=iter_max)
    Xo, ito, _ = mirror(rp, ci, v, B, 1e-12, iter_max)
    m.destroy()
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == list(ito)


def mirror_ir(rp, ci, v, B, eps_rel, inner_eps, inner_max, outer_max):
    """FP64 refinement of every column around an FP32 multi-column PCG,
    composed from oracle pieces in the multi-column reduction order."""
    f32, f64 = np.float32, np.float64
    n, k = B.shape
    J = R.jacobi(R.diag(rp, ci, v))
    J32 = J.astype(f32)
    v32 = v.astype(f32)
    spmm64 = lambda X: np.stack([R.spmv_csr(rp, ci, v, X[:, c]) for c in range(k)], 1)
    spmm32 = lambda X: np.stack([R.spmv_csr_f32(rp, ci, v32, X[:, c]) for c in range(k)], 1)
    D = lambda a: a.astype(f64)

    def inner(B32, part, taus):
        X = np.zeros((n, k), f32)
        bn = np.sqrt(dot_cols(D(B32), D(B32)))
        eps = taus * bn
        Rr = (D(B32) - D(f32(0) + spmm32(X))).astype(f32)
        Z = D(Rr) * D(J32)[:, None]
        P = Z.astype(f32)
        alpha, norm = dot_cols(D(Rr), Z), np.sqrt(dot_cols(D(Rr), D(Rr)))
        it = np.zeros(k, int)
        go = lambda c: it[c] < inner_max and abs(alpha[c]) > R.REAL_SMALL and norm[c] > eps[c]
        active = np.array([bool(part[c]) and go(c) for c in range(k)])
        while active.any():
            V = (f32(0) + spmm32(P)).astype(f32)
            pv = dot_cols(D(V), D(P))
            for c in np.flatnonzero(active):
                sg = alpha[c] / pv[c]
                X[:, c] = (D(X[:, c]) + sg * D(P[:, c])).astype(f32)
                Rr[:, c] = (D(Rr[:, c]) + (-sg) * D(V[:, c])).astype(f32)
            Z = D(Rr) * D(J32)[:, None]
            rz, rr = dot_cols(D(Rr), Z), dot_cols(D(Rr), D(Rr))
            beta = np.zeros(k)
            for c in np.flatnonzero(active):
                beta[c] = rz[c] / alpha[c]
                alpha[c], norm[c] = rz[c], np.sqrt(rr[c])
                it[c] += 1
                active[c] = go(c)
            for c in np.flatnonzero(active):
                P[:, c] = (beta[c] * D(P[:, c]) + D(Rr[:, c]) * D(J32)).astype(f32)
        return X, it

    X = np.zeros((n, k))
    tol = eps_rel * np.sqrt(dot_cols(B, B))
    done = np.zeros(k, bool)
    outer = np.zeros(k, int)
    inner_total = np.zeros(k, int)
    rn = np.zeros(k)
    for _ in range(outer_max + 1):
        Rr = B - (0.0 + spmm64(X))
        rn_all = np.sqrt(dot_cols(Rr, Rr))
        part = np.zeros(k, bool)
        for c in range(k):
            if done[c]:
                continue
            rn[c] = rn_all[c]
            if rn[c] <= tol[c] or outer[c] >= outer_max:
                done[c] = True
            else:
                part[c] = True
        if not part.any():
            break
        B32 = np.zeros((n, k), f32)
        taus = np.full(k, inner_eps)
        for c in np.flatnonzero(part):
            B32[:, c] = (Rr[:, c] * (1.0 / rn[c])).astype(f32)
            taus[c] = ir_step_tolerance(rn[c], tol[c], inner_eps)
        Dd, its = inner(B32, part, taus)
        for c in np.flatnonzero(part):
            inner_total[c] += its[c]
            outer[c] += 1
            X[:, c] = X[:, c] + rn[c] * D(Dd[:, c])
    return X, outer, inner_total, rn


@pytest.mark.parametrize("mode", ["graph", "host_loop"])
@pytest.mark.parametrize("k", [6, 8])
def test_multirhs_fp32_refinement_bitexact(gpu, mode, k, monkeypatch):
    """k = 8 runs the inner SpMM with 16-byte gathers of four FP32 columns,
    k = 6 the register-pipeline SpMM."""
    celgpu, h, torch = gpu
    if mode == "host_loop":
        monkeypatch.setenv("CELG_GRAPH", "0")
    rng = np.random.default_rng(15)
    _, (kx, ky, kz) = synth.lognormal_faces(rng, 9, 8, 10, 0.5)
    rp, ci, v = synth.diffusion7(9, 8, 10, kx, ky, kz)
    n = rp.size - 1
    B = rng.uniform(-1.0, 1.0, (n, k))
    B[:, 3] *= 1e-3                         # columns of different scale
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    kw = dict(eps_rel=1e-10, iter_max=3000, precision=celgpu.PREC_FP32_IR, inner_eps_rel=1e-4,
              inner_iter_max=800, outer_max=20)
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), **kw)
    Xo, outer, inner_total, rn = mirror_ir(rp, ci, v, B, 1e-10, 1e-4, 800, 20)
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == list(outer)
    assert [i.arnoldi_steps for i in infos] == list(inner_total)
    assert [i.final_norm2 for i in infos] == list(rn)
    assert all(i.status == celgpu.OK and i.verified_relres <= 1e-10 for i in infos)
    m.destroy()


def mirror_ru(rp, ci, v, B, eps_rel, delta, iter_max):
    """FP32 PCG with FP64 reliable updates of every column: the recurrence of
    the single solve (ru_oracle in test_gpu_solvers.py) per column, composed
    from oracle pieces in the multi-column reduction order."""
    f32, f64 = np.float32, np.float64
    n, k = B.shape
    J32 = R.jacobi(R.diag(rp, ci, v)).astype(f32).astype(f64)
    v32 = v.astype(f32)
    dc = lambda a, b: dot_cols(a[:, None], b[:, None])[0]
    X = np.zeros((n, k))
    its, ups, norms = [], [], []
    for c in range(k):
        b = B[:, c]

        def residual(x):
            r64 = b - (0.0 + R.spmv_csr(rp, ci, v, x))
            r = r64.astype(f32)
            z = r.astype(f64) * J32
            return r, z, dc(r.astype(f64), z), np.sqrt(dc(r64, r64))

        x = np.zeros(n)
        eps = eps_rel * np.sqrt(dc(b, b))
        r, z, rz, norm64 = residual(x)
        p = z.astype(f32)
        d = np.zeros(n, f32)
        maxr, it, updates = norm64, 0, 1
        active = norm64 > eps and it < iter_max
        while active:
            w = (f32(0) + R.spmv_csr_f32(rp, ci, v32, p)).astype(f32)
            sigma = rz / dc(w.astype(f64), p.astype(f64))
            d = (d.astype(f64) + sigma * p.astype(f64)).astype(f32)
            r = r + f32(-sigma) * w                 # FP32 arithmetic, one rounding each
            z = r.astype(f64) * J32
            rz_new = dc(r.astype(f64), z)
            norm = np.sqrt(dc(r.astype(f64), r.astype(f64)))
            rz_prev, beta, rz = rz, rz_new / rz, rz_new
            it += 1
            if norm < delta * maxr or norm <= eps or it >= iter_max:
                x = x + d.astype(f64)
                d[:] = 0
                r, z, rzh, norm64 = residual(x)
                maxr = norm64
                beta, rz = rzh / rz_prev, rzh
                updates += 1
                active = norm64 > eps and it < iter_max
            else:
                active = it < iter_max and abs(rz) > 0
            if active:
                p = (beta * p.astype(f64) + z).astype(f32)
        X[:, c] = x + d.astype(f64)
        its.append(it)
        ups.append(updates)
        norms.append(norm64)
    return X, its, ups, norms


def ru_problem(k, seed=15):
    rng = np.random.default_rng(seed)
    _, (kx, ky, kz) = synth.lognormal_faces(rng, 9, 8, 10, 0.5)
    rp, ci, v = synth.diffusion7(9, 8, 10, kx, ky, kz)
    B = rng.uniform(-1.0, 1.0, (rp.size - 1, k))
    B[:, 3] *= 1e-3                         # columns of different scale
    return rp, ci, v, B


@pytest.mark.parametrize("mode", ["graph", "host_loop"])
@pytest.mark.parametrize("k", [6, 8])
def test_multirhs_fp32_reliable_update_bitexact(gpu, mode, k, monkeypatch):
    """Every column runs FP32 PCG with FP64 reliable updates: X, iteration and
    update counts and the last FP64 residual norms equal the mirror's.  k = 8
    runs the FP32 SpMM with 16-byte gathers, k = 6 the register pipeline."""
    celgpu, h, torch = gpu
    if mode == "host_loop":
        monkeypatch.setenv("CELG_GRAPH", "0")
    rp, ci, v, B = ru_problem(k)
    n = rp.size - 1
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-10, iter_max=3000,
                           precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2)
    Xo, its, ups, norms = mirror_ru(rp, ci, v, B, 1e-10, 1e-2, 3000)
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == its
    assert [i.arnoldi_steps for i in infos] == ups
    assert [i.final_norm2 for i in infos] == norms
    assert all(i.status == celgpu.OK and i.verified_relres <= 1e-10 for i in infos)
    # the same solutions as the FP64 multi-column solve, to the tolerance
    # (column 3, scaled by 1e-3, is left out: the FP64 loop's absolute guard
    # |r.z| > 1.1 eps_mach ends it before rel-res 1e-10)
    X64 = dev(torch, np.zeros((n, k)))
    h.pcg_multirhs(m, k, Bd.data_ptr(), X64.data_ptr(), eps_rel=1e-10, iter_max=3000)
    Xr, X6 = Xd.cpu().numpy(), X64.cpu().numpy()
    for c in range(k):
        if c != 3:
            assert np.abs(Xr[:, c] - X6[:, c]).max() <= 1e-6 * np.abs(X6[:, c]).max()
    m.destroy()


@pytest.mark.parametrize("iter_max", [1, 9])
def test_multirhs_fp32_reliable_update_iteration_cap(gpu, iter_max):
    """The iteration cap forces a reliable update; the pending d += sigma p is
    applied before x is flushed, and every column reports CELG_ERR_NOCONV."""
    celgpu, h, torch = gpu
    rp, ci, v, B = ru_problem(5, seed=16)
    n, k = B.shape
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-10, iter_max=iter_max,
                           precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2)
    Xo, its, ups, norms = mirror_ru(rp, ci, v, B, 1e-10, 1e-2, iter_max)
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == its == [iter_max] * k
    assert all(i.status == celgpu.ERR_NOCONV for i in infos)
    m.destroy()


@pytest.mark.parametrize("cfg32", range(5))
def test_every_fp32_spmm_shape_is_bitexact(gpu, cfg32, monkeypatch):
    """Each FP32 SpMM launch shape the tuner chooses from (forced with
    CELG_SPMM32_CFG) gives the mirror's bits in the reliable-update form."""
    celgpu, h, torch = gpu
    monkeypatch.setenv("CELG_SPMM32_CFG", str(cfg32))
    rp, ci, v, B = ru_problem(8, seed=17)
    n, k = B.shape
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-10, iter_max=3000,
                           precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2)
    assert h.tuned_config(celgpu.TUNE_SPMM)[1] == cfg32
    Xo, its, _, _ = mirror_ru(rp, ci, v, B, 1e-10, 1e-2, 3000)
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == its
    m.destroy()


def test_multirhs_fp32_reliable_update_unstructured(gpu):
    """An unstructured matrix with some long rows (no row patterns, no 1-byte
    offsets: the SpMMs read the int32 columns, long rows past the staging
    chunks): every column still equals the mirror bit for bit."""
    celgpu, h, torch = gpu
    from tests.helpers import random_csr, spd_from_pattern
    rng = np.random.default_rng(21)
    rp, ci, v = spd_from_pattern(*random_csr(3000, rng, max_len=9, empty_frac=0.0, long_rows=3,
                                             long_len=400))
    n, k = rp.size - 1, 8
    B = rng.uniform(-1.0, 1.0, (n, k))
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd, Xd = dev(torch, B), dev(torch, np.zeros((n, k)))
    infos = h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), eps_rel=1e-10, iter_max=3000,
                           precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2)
    assert m.column_form() == celgpu.COLS_INT32
    Xo, its, ups, norms = mirror_ru(rp, ci, v, B, 1e-10, 1e-2, 3000)
    assert np.array_equal(Xd.cpu().numpy(), Xo)
    assert [i.iter_done for i in infos] == its
    assert [i.arnoldi_steps for i in infos] == ups
    assert all(i.status == celgpu.OK and i.verified_relres <= 1e-10 for i in infos)
    m.destroy()
