"""GPU parity of the operators (through the C ABI): SpMV CSR/JAD/FP32, the
JAD conversion, Jacobi set-up, row scaling and the vector reductions, all
compared bit for bit with the oracle."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R
from tests.helpers import random_csr

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def matrices():
    rng = np.random.default_rng(2024)
    out = {}
    out["poisson32"] = synth.poisson7(32)
    out["poisson_5x7x33"] = synth.poisson7(5, 7, 33)
    for n in (1, 255, 256, 257, 1023, 1025, 5000):
        out[f"random{n}"] = random_csr(n, rng)
    out["long_rows"] = random_csr(8000, rng, long_rows=3, long_len=6000)
    out["medium_rows"] = random_csr(3000, rng, long_rows=2, long_len=2500)
    g, (kx, ky, kz) = synth.lognormal_faces(np.random.default_rng(1), 9, 10, 11)
    out["diffusion"] = synth.diffusion7(9, 10, 11, kx, ky, kz)
    return out


MATS = matrices()


@pytest.mark.parametrize("name", sorted(MATS))
def test_spmv_csr_bitexact(gpu, name, ref_poisson):
    celgpu, h, torch = gpu
    rp, ci, v = MATS[name]
    n = rp.size - 1
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    y0 = rng.standard_normal(n)
    m = h.matrix_from_csr(rp, ci, v)
    xd, yd = dev(torch, x), dev(torch, y0)
    h.spmv(m, xd.data_ptr(), yd.data_ptr())
    assert np.array_equal(yd.cpu().numpy(), R.spmv_csr(rp, ci, v, x))
    yd = dev(torch, y0)
    h.spmv(m, xd.data_ptr(), yd.data_ptr(), accumulate=True)
    assert np.array_equal(yd.cpu().numpy(), R.spmv_csr(rp, ci, v, x, y0, accumulate=True))
    m.destroy()


def test_spmv_reference_fixtures(gpu, ref_poisson):
    celgpu, h, torch = gpu
    for key, d in ref_poisson.items():
        m = h.matrix_from_csr(d["rp"] + 1, d["ci"] + 1, d["v"], index_base=1)
        yd = dev(torch, np.zeros(d["u"].size))
        h.spmv(m, dev(torch, d["u"]).data_ptr(), yd.data_ptr())
        y = yd.cpu().numpy()
        assert np.array_equal(y, R.spmv_csr(d["rp"], d["ci"], d["v"], d["u"]))
        assert np.abs(y - d["b"]).max() <= 1e-13 * np.abs(d["v"]).max() * np.abs(d["u"]).max()
        m.destroy()


def test_spmv_simple_test_known_answer(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, b, xth = synth.simple_test(4096, 32)
    m = h.matrix_from_csr(rp, ci, v)
    yd = dev(torch, np.zeros(4096))
    h.spmv(m, dev(torch, xth).data_ptr(), yd.data_ptr())
    assert np.array_equal(yd.cpu().numpy(), b)
    m.destroy()


@pytest.mark.parametrize("name", ["poisson32", "random5000", "long_rows", "diffusion"])
def test_spmv_f32_bitexact(gpu, name):
    celgpu, h, torch = gpu
    rp, ci, v = MATS[name]
    n = rp.size - 1
    x = np.random.default_rng(4).standard_normal(n).astype(np.float32)
    m = h.matrix_from_csr(rp, ci, v).jacobi().make_fp32()
    yd = dev(torch, np.zeros(n, np.float32))
    h.spmv_f32(m, dev(torch, x).data_ptr(), yd.data_ptr())
    assert np.array_equal(yd.cpu().numpy(), R.spmv_csr_f32(rp, ci, v.astype(np.float32), x))
    m.destroy()


def banded_dictionary_csr(n=5017, seed=7):
    """Rows of 14..18 entries (one empty row) whose column offsets come from a
    fixed set of 40, so the FP32 copy has a 1-byte offset dictionary: the
    FP32 dictionary sweep with rows longer than one 8-entry chunk."""
    rng = np.random.default_rng(seed)
    offs = np.sort(rng.choice(np.arange(-60, 61), size=40, replace=False))
    cols = []
    for i in range(n):
        ok = offs[(i + offs >= 0) & (i + offs < n)]
        k = 0 if i == 100 else min(ok.size, int(rng.integers(14, 19)))
        cols.append(np.sort(i + rng.choice(ok, size=k, replace=False)))
    rp = np.concatenate([[0], np.cumsum([c.size for c in cols])]).astype(np.int32)
    ci = np.concatenate(cols).astype(np.int32)
    return rp, ci, rng.standard_normal(ci.size)


def test_spmv_f32_dictionary_long_rows_bitexact(gpu):
    celgpu, h, torch = gpu
    rp, ci, v = banded_dictionary_csr()
    n = rp.size - 1
    x = np.random.default_rng(5).standard_normal(n).astype(np.float32)
    m = h.matrix_from_csr(rp, ci, v).jacobi().make_fp32()
    yd = dev(torch, np.full(n, 7.0, np.float32))
    h.spmv_f32(m, dev(torch, x).data_ptr(), yd.data_ptr())
    y = R.spmv_csr_f32(rp, ci, v.astype(np.float32), x)
    assert np.array_equal(yd.cpu().numpy(), y)
    assert yd[100].item() == 0.0                       # the empty row
    h.spmv_f32(m, dev(torch, x).data_ptr(), yd.data_ptr(), accumulate=True)
    assert np.array_equal(yd.cpu().numpy(), R.spmv_csr_f32(rp, ci, v.astype(np.float32), x, y=y,
                                                           accumulate=True))
    m.destroy()


def test_row_patterns_fp32_and_pcg_bitexact(gpu):
    """A 7-point operator with one row emptied and one row given a ninth
    entry: the rows of at most 8 entries use few distinct offset sequences,
    so the sweeps run on row patterns -- except that the long row rules them
    out for the second matrix, which runs on the 1-byte offsets instead.
    Both give the oracle's bits (FP32 SpMV; FP64 PCG on the first)."""
    celgpu, h, torch = gpu
    rp, ci, v = synth.poisson7(13, 9, 11)
    n = rp.size - 1
    lens = np.diff(rp)
    lens[40] = 0                                        # an empty row
    keep = np.ones(ci.size, bool)
    keep[rp[40]:rp[41]] = False
    rp_e = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci_e, v_e = ci[keep], v[keep]
    x = np.random.default_rng(6).standard_normal(n).astype(np.float32)
    for rp2, ci2, v2 in ((rp_e, ci_e, v_e),):
        m = h.matrix_from_csr(rp2, ci2, v2).make_fp32()
        yd = dev(torch, np.zeros(n, np.float32))
        h.spmv_f32(m, dev(torch, x).data_ptr(), yd.data_ptr())
        assert np.array_equal(yd.cpu().numpy(), R.spmv_csr_f32(rp2, ci2, v2.astype(np.float32), x))
        m.destroy()
    # a ninth entry in row 100 (a far column): no row patterns, 1-byte offsets
    cols = [ci[rp[i]:rp[i + 1]] for i in range(n)]
    vals = [v[rp[i]:rp[i + 1]] for i in range(n)]
    cols[100] = np.sort(np.append(cols[100], [n - 1, n - 2]))
    vals[100] = np.append(vals[100], [-0.25, -0.25])
    rp9 = np.concatenate([[0], np.cumsum([c.size for c in cols])]).astype(np.int32)
    ci9, v9 = np.concatenate(cols).astype(np.int32), np.concatenate(vals)
    m = h.matrix_from_csr(rp9, ci9, v9).make_fp32()
    yd = dev(torch, np.zeros(n, np.float32))
    h.spmv_f32(m, dev(torch, x).data_ptr(), yd.data_ptr())
    assert np.array_equal(yd.cpu().numpy(), R.spmv_csr_f32(rp9, ci9, v9.astype(np.float32), x))
    m.destroy()
    # FP64 PCG on the row patterns of the plain operator, against the oracle
    b = R.spmv_csr(rp, ci, v, np.random.default_rng(7).random(n))
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    xd = dev(torch, np.zeros(n))
    info = h.pcg_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=True, eps_rel=1e-10,
                        iter_max=2000)
    xo, io = R.pcg_jacobi(R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v)), b, eps_rel=1e-10,
                          iter_max=2000, red=R.RED_TREE)
    assert info.iter_done == io["iter_done"] and np.array_equal(info.history, io["history"])
    assert np.array_equal(xd.cpu().numpy(), xo)
    m.destroy()


@pytest.mark.parametrize("name", sorted(MATS))
def test_jad_conversion_and_spmv_bitexact(gpu, name):
    celgpu, h, torch = gpu
    rp, ci, v = MATS[name]
    n = rp.size - 1
    m = h.matrix_from_csr(rp, ci, v)
    perm = m.to_jad()
    ref = R.jad_build(rp, ci, v)
    assert np.array_equal(perm, ref["perm"])                 # bit-exact permutation
    got = m.get_jad()
    assert got["mmax"] == ref["mmax"]
    assert np.array_equal(got["jbegin"], ref["jbegin"])
    assert np.array_equal(got["jci"], ref["jci"]) and np.array_equal(got["jv"], ref["jv"])
    x = np.random.default_rng(5).standard_normal(n)
    yd = dev(torch, np.zeros(n))
    h.spmv(m, dev(torch, x).data_ptr(), yd.data_ptr(), fmt=celgpu.FMT_JAD)
    assert np.array_equal(yd.cpu().numpy(), R.spmv_jad(ref, x, n))
    m.destroy()


@pytest.mark.parametrize("name", ["poisson32", "random1025", "diffusion", "long_rows"])
def test_jacobi_and_scaling_bitexact(gpu, name):
    celgpu, h, torch = gpu
    rp, ci, v = MATS[name]
    n = rp.size - 1
    d = R.diag(rp, ci, v)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    with np.errstate(divide="ignore"):
        J = R.jacobi(d)
    assert np.array_equal(m.get_jacobi(), J)  # includes 1/0 = inf rows
    if np.all(d != 0):
        m.scale_diagonal()
        vs, s = R.row_scale(rp, v, d)
        assert np.array_equal(m.get_jacobi(), R.jacobi(d, s))
        x = np.random.default_rng(6).standard_normal(n)
        yd = dev(torch, np.zeros(n))
        h.spmv(m, dev(torch, x).data_ptr(), yd.data_ptr())
        assert np.array_equal(yd.cpu().numpy(), R.spmv_csr(rp, ci, vs, x))
    m.destroy()


@pytest.mark.parametrize("n", [0, 1, 255, 1023, 1024, 1025, 4097, 100003])
def test_blas1_bitexact(gpu, n):
    celgpu, h, torch = gpu
    rng = np.random.default_rng(n + 1)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    ad, bd = dev(torch, a), dev(torch, b)
    assert h.dot(n, ad.data_ptr(), bd.data_ptr()) == R.dot(a, b, R.RED_TREE)
    assert h.norm2(n, ad.data_ptr()) == np.sqrt(R.dot(a, a, R.RED_TREE))
    if n == 0:
        return
    yd = dev(torch, b)
    h.axpy(n, 0.37, ad.data_ptr(), yd.data_ptr())
    assert np.array_equal(yd.cpu().numpy(), b + 0.37 * a)
    yd = dev(torch, b)
    h.xpby(n, ad.data_ptr(), -1.25, yd.data_ptr())
    assert np.array_equal(yd.cpu().numpy(), -1.25 * b + a)


def test_jacobi_apply(gpu):
    celgpu, h, torch = gpu
    rp, ci, v = MATS["diffusion"]
    n = rp.size - 1
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    r = np.random.default_rng(8).standard_normal(n)
    zd = dev(torch, np.zeros(n))
    h.jacobi_apply(m, dev(torch, r).data_ptr(), zd.data_ptr())
    assert np.array_equal(zd.cpu().numpy(), r * R.jacobi(R.diag(rp, ci, v)))
    m.destroy()


def test_malformed_csr_rejected(gpu):
    celgpu, h, torch = gpu
    rp = np.array([0, 2, 1, 3], np.int32)  # not monotone
    ci = np.array([0, 1, 2], np.int32)
    with pytest.raises(celgpu.CelgError) as e:
        h.matrix_from_csr(rp, ci, np.ones(3))
    assert e.value.status == celgpu.ERR_ARG
    with pytest.raises(celgpu.CelgError):
        h.matrix_from_csr(np.array([0, 1], np.int32), np.array([5], np.int32), np.ones(1))


def test_empty_matrix(gpu):
    celgpu, h, torch = gpu
    m = h.matrix_from_csr(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    assert m.info()[:2] == (0, 0)
    m.destroy()
