"""Assembly path: the MatrixMarket reader (host code, runs without a GPU)
and COO -> CSR on the device (celg_mat_from_coo, ELM MatrixCompleted)."""
import numpy as np
import pytest

from oracle import celref as R


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return p


@pytest.fixture(scope="module")
def celgpu():
    from cel_v3_b200 import celgpu as C
    return C


def test_mm_coordinate_general(celgpu, tmp_path):
    p = write(tmp_path, "g.mtx", "%%MatrixMarket matrix coordinate real general\n% comment\n\n"
              "3 4 4\n1 1 2.5\n3 4 -1e-3\n2 2 7\n1 1 0.5\n")
    nr, nc, sy, r, c, v = celgpu.mm_read(p)
    assert (nr, nc, sy) == (3, 4, celgpu.MM_GENERAL)
    assert r.tolist() == [1, 3, 2, 1] and c.tolist() == [1, 4, 2, 1]
    assert v.tolist() == [2.5, -1e-3, 7.0, 0.5]


def test_mm_symmetric_as_stored_and_expanded(celgpu, tmp_path):
    p = write(tmp_path, "s.mtx", "%%MatrixMarket matrix coordinate real symmetric\n"
              "3 3 4\n1 1 4\n2 1 -1\n3 2 -2\n3 3 5\n")
    nr, nc, sy, r, c, v = celgpu.mm_read(p)
    assert sy == celgpu.MM_SYMMETRIC and r.size == 4          # the stored triangle only
    _, _, _, r, c, v = celgpu.mm_read(p, expand=True)
    assert list(zip(r.tolist(), c.tolist(), v.tolist())) == [
        (1, 1, 4.0), (2, 1, -1.0), (1, 2, -1.0), (3, 2, -2.0), (2, 3, -2.0), (3, 3, 5.0)]


def test_mm_pattern_integer_skew_and_array(celgpu, tmp_path):
    p = write(tmp_path, "p.mtx", "%%MatrixMarket matrix coordinate pattern general\n2 2 2\n1 2\n2 1\n")
    assert celgpu.mm_read(p)[5].tolist() == [1.0, 1.0]
    p = write(tmp_path, "i.mtx", "%%MatrixMarket matrix coordinate integer general\n2 2 1\n2 2 -3\n")
    assert celgpu.mm_read(p)[5].tolist() == [-3.0]
    p = write(tmp_path, "k.mtx", "%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 3\n")
    _, _, sy, r, c, v = celgpu.mm_read(p, expand=True)
    assert sy == celgpu.MM_SKEW and list(zip(r, c, v)) == [(2, 1, 3.0), (1, 2, -3.0)]
    # dense column-major; symmetric arrays store the lower triangle
    p = write(tmp_path, "a.mtx", "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    _, _, _, r, c, v = celgpu.mm_read(p)
    assert list(zip(r, c, v)) == [(1, 1, 1.0), (2, 1, 2.0), (1, 2, 3.0), (2, 2, 4.0)]
    p = write(tmp_path, "as.mtx", "%%MatrixMarket matrix array real symmetric\n2 2\n1\n2\n4\n")
    _, _, _, r, c, v = celgpu.mm_read(p)
    assert list(zip(r, c, v)) == [(1, 1, 1.0), (2, 1, 2.0), (2, 2, 4.0)]


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n",        # truncated
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",        # row out of range
    "not a matrix market file\n",
])
def test_mm_rejects(celgpu, tmp_path, text):
    p = write(tmp_path, "bad.mtx", text)
    with pytest.raises(celgpu.CelgError):
        celgpu.mm_read(p)


def coo_case(seed, n=700, nnz=5000):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n, nnz)
    cols = rng.integers(0, n, nnz)
    # duplicates (same key, different values) and explicit zeros
    rows[:50], cols[:50] = rows[50:100], cols[50:100]
    vals = rng.standard_normal(nnz)
    vals[100:120] = 0.0
    return n, rows, cols, vals


def csr_of(n, rows, cols, vals):
    order = np.lexsort((cols, rows))            # stable: equal keys keep input order
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp).astype(np.int32), cols[order].astype(np.int32), vals[order]


@pytest.mark.gpu
@pytest.mark.parametrize("base", [0, 1])
def test_coo_to_csr_keeps_order_of_equal_keys(gpu, base):
    celgpu, h, torch = gpu
    n, rows, cols, vals = coo_case(3)
    rp, ci, v = csr_of(n, rows, cols, vals)
    m = h.matrix_from_coo(n, rows + base, cols + base, vals, index_base=base)
    x = np.random.default_rng(4).standard_normal(n)
    xd, yd = torch.from_numpy(x).cuda(), torch.zeros(n, dtype=torch.float64, device="cuda")
    h.spmv(m, xd.data_ptr(), yd.data_ptr())
    # row sums in stored order: equal to the oracle only with the same entry order
    assert np.array_equal(yd.cpu().numpy(), R.spmv_csr(rp, ci, v, x))
    assert m.info()[:2] == (n, rows.size)
    m.destroy()
    with pytest.raises(celgpu.CelgError):
        h.matrix_from_coo(n, rows, np.where(cols == 5, n, cols), vals)   # column out of range


@pytest.mark.gpu
def test_matrix_market_to_pcg(gpu, tmp_path):
    """A symmetric MatrixMarket file, expanded and assembled on the device,
    solves like the CSR built directly."""
    celgpu, h, torch = gpu
    from cel_v3_b200 import synth
    rp, ci, v = synth.poisson7(7, 6, 5)
    n = rp.size - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    low = ci <= rows
    lines = [f"{r + 1} {c + 1} {float(val)!r}" for r, c, val in zip(rows[low], ci[low], v[low])]
    p = write(tmp_path, "poisson.mtx", "%%MatrixMarket matrix coordinate real symmetric\n"
              f"{n} {n} {len(lines)}\n" + "\n".join(lines) + "\n")
    nr, nc, sy, r, c, vv = celgpu.mm_read(p, expand=True)
    m = h.matrix_from_coo(nr, r, c, vv, index_base=1).jacobi()
    m2 = h.matrix_from_csr(rp, ci, v).jacobi()
    b = torch.from_numpy(np.random.default_rng(1).random(n)).cuda()
    x1, x2 = torch.zeros_like(b), torch.zeros_like(b)
    i1 = h.pcg_jacobi(m, b.data_ptr(), x1.data_ptr(), eps_rel=1e-10)
    i2 = h.pcg_jacobi(m2, b.data_ptr(), x2.data_ptr(), eps_rel=1e-10)
    assert i1.iter_done == i2.iter_done and torch.equal(x1, x2)
    m.destroy()
    m2.destroy()
