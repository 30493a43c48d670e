"""CPU tests of the oracle (oracle/libcelref.so): pinned against the
reference's own known answers and checked for the properties the GPU
parity tests rely on."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R
from tests.helpers import random_csr


# ---- work split (src/fbase/cel_omp_shared_work_module.f90:196-220) -----------

@pytest.mark.parametrize("length,W,expect", [
    (10, 2, [(0, 4), (4, 10)]),          # 4-aligned blocks, remainder to the last worker
    (3, 4, [(0, 0), (0, 0), (0, 0), (0, 3)]),
    (17, 3, [(0, 4), (4, 8), (8, 17)]),
    (16, 4, [(0, 4), (4, 8), (8, 12), (12, 16)]),
    (0, 2, [(0, 0), (0, 0)]),
])
def test_work_chunk_hand_values(length, W, expect):
    got = [R.work_chunk(length, W, w) for w in range(1, W + 1)]
    got = [(s, e) if e > s else (0, 0) for s, e in got]
    exp = [(s, e) if e > s else (0, 0) for s, e in expect]
    assert got == exp


@pytest.mark.parametrize("length", [1, 5, 63, 64, 1000, 12345])
@pytest.mark.parametrize("W", [1, 2, 3, 7])
def test_work_chunk_partitions(length, W):
    covered = []
    for w in range(1, W + 1):
        s, e = R.work_chunk(length, W, w)
        covered.extend(range(s, e))
    assert covered == list(range(length))


def test_seq_dot_is_worker_ordered_chunk_sum():
    rng = np.random.default_rng(11)
    a, b = rng.standard_normal(5003), rng.standard_normal(5003)
    for W in (1, 2, 5):
        tot = 0.0
        for w in range(1, W + 1):
            s, e = R.work_chunk(a.size, W, w)
            acc = 0.0
            for i in range(s, e):
                acc = acc + a[i] * b[i]
            tot = tot + acc
        assert R.dot(a, b, R.RED_SEQ, W) == tot


# ---- block-tree reduction --------------------------------------------------------

def test_tree_reduction_exact_on_integers():
    rng = np.random.default_rng(3)
    for n in (0, 1, 255, 256, 1023, 1024, 1025, 70001):
        a = rng.integers(-1000, 1000, n).astype(np.float64)
        b = rng.integers(-1000, 1000, n).astype(np.float64)
        assert R.dot(a, b, R.RED_TREE) == float(np.dot(a.astype(np.int64), b.astype(np.int64)))


def test_tree_matches_python_restatement():
    """Lane j sums j, j+256, ...; butterfly within 32 lanes; warps in order."""
    def fold(s):
        s = list(s)
        for w in range(8):
            q = s[32 * w: 32 * w + 32]
            for off in (16, 8, 4, 2, 1):
                q = [q[l] + q[l ^ off] for l in range(32)]
            s[32 * w: 32 * w + 32] = q
        tot = s[0]
        for w in range(1, 8):
            tot = tot + s[32 * w]
        return tot

    def red(vals):
        s = []
        for j in range(256):
            acc = 0.0
            for k in range(j, len(vals), 256):
                acc = acc + vals[k]
            s.append(acc)
        return fold(s)

    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(3000), rng.standard_normal(3000)
    prods = a * b
    parts = [red(prods[t:t + 1024]) for t in range(0, 3000, 1024)]
    assert R.dot(a, b, R.RED_TREE) == red(parts)


# ---- known answers of the reference ---------------------------------------------------

def test_simple_test_known_answer():
    """cel_sp_mat_generate_simple_test: A * 1 = b exactly (checked by the
    reference at tests/cel_cg/src/cel_cg.f90:810-837 with tol 1e-7)."""
    rp, ci, v, b, xth = synth.simple_test(512, 16)
    assert np.array_equal(R.spmv_csr(rp, ci, v, xth), b)
    assert np.array_equal(R.spmv_csr(rp, ci, v, xth, nworkers=3), b)


def test_reference_poisson_spmv_known_answer(ref_poisson):
    """The reference generator's quadratic solution satisfies A u = b."""
    for key, d in ref_poisson.items():
        y = R.spmv_csr(d["rp"], d["ci"], d["v"], d["u"])
        scale = np.abs(d["v"]).max() * np.abs(d["u"]).max()
        assert np.abs(y - d["b"]).max() <= 1e-13 * scale, key


@pytest.mark.parametrize("red", [R.RED_SEQ, R.RED_TREE])
def test_reference_poisson_pcg_known_answer(ref_poisson, red):
    """Jacobi-PCG from the reference's x0 = 1 recovers u = x^2+y^2+z^2
    (check of tests/cel_cg/src/cel_cg.f90:838-858)."""
    for key, d in ref_poisson.items():
        A = R.Matrix(d["rp"], d["ci"], d["v"])
        J = R.jacobi(R.diag(d["rp"], d["ci"], d["v"]))
        x, info = R.pcg_jacobi(A, J, d["b"], x0_mode=R.X0_ONES, eps_abs=1e-10 * np.linalg.norm(d["b"]),
                               eps_rel=0.0, iter_max=2000, red=red)
        assert info["err"] == 0
        assert np.abs(x - d["u"]).max() < 1e-8 * np.abs(d["u"]).max(), key


def test_reference_poisson_gmres_known_answer(ref_poisson):
    for key, d in ref_poisson.items():
        A = R.Matrix(d["rp"], d["ci"], d["v"])
        J = R.jacobi(R.diag(d["rp"], d["ci"], d["v"]))
        x, info = R.gmres_jacobi(A, J, d["b"], restart=10, x0_mode=R.X0_ONES, eps_abs=0.0,
                                 eps_rel=1e-11, iter_max=50)
        assert info["err"] == 0
        assert np.abs(x - d["u"]).max() < 1e-8 * np.abs(d["u"]).max(), key


# ---- JAD -------------------------------------------------------------------------------

def _random_csr(n, rng):
    return random_csr(n, rng)


def test_jad_perm_is_stable_descending_sort():
    rng = np.random.default_rng(7)
    for n in (1, 2, 17, 1000):
        rp, _, _ = _random_csr(n, rng)
        perm, mmax = R.jad_perm(rp)
        lens = np.diff(rp)
        assert mmax == lens.max()
        expect = np.array(sorted(range(n), key=lambda i: (-lens[i], i)), np.int32)
        assert np.array_equal(perm, expect)


def test_jad_literal_counts_document_reference_defect():
    """The reference leaves count(len > ilo+k-1) in jad_begin (wrong offsets),
    e.g. lengths [4,5,6,7,7,6,5,4] give 6,4,2,0 where diagonals 1..7 need
    8,8,8,8,6,4,2 rows."""
    lens = np.array([4, 5, 6, 7, 7, 6, 5, 4])
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    lit, lo, hi = R.jad_begin_literal(rp)
    assert (lo, hi) == (4, 7)
    assert list(lit) == [6, 4, 2, 0]
    ci = np.concatenate([np.arange(l) for l in lens]).astype(np.int32)
    jad = R.jad_build(rp, ci, np.ones(rp[-1]))
    assert list(np.diff(jad["jbegin"])) == [8, 8, 8, 8, 6, 4, 2]


def test_jad_spmv_equals_csr_bitwise():
    rng = np.random.default_rng(9)
    for n in (1, 50, 3000):
        rp, ci, v = _random_csr(n, rng)
        x = rng.standard_normal(n)
        jad = R.jad_build(rp, ci, v)
        assert np.array_equal(R.spmv_jad(jad, x, n), R.spmv_csr(rp, ci, v, x))


# ---- solvers -----------------------------------------------------------------------------

@pytest.fixture(scope="module")
def small_poisson():
    rp, ci, v, xt = synth.plain(32, 0)
    b = R.spmv_csr(rp, ci, v, xt)
    J = R.jacobi(R.diag(rp, ci, v))
    return rp, ci, v, xt, b, J


def test_pcg_tree_vs_reference_order_within_1e10(small_poisson):
    """The GPU reduction order (tree) against the reference's sequential
    order: same iteration count, history and solution within 1e-10."""
    rp, ci, v, xt, b, J = small_poisson
    A = R.Matrix(rp, ci, v)
    x1, i1 = R.pcg_jacobi(A, J, b, red=R.RED_SEQ)
    x2, i2 = R.pcg_jacobi(A, J, b, red=R.RED_TREE)
    assert abs(i1["iter_done"] - i2["iter_done"]) <= 1
    m = min(len(i1["history"]), len(i2["history"]))
    assert np.max(np.abs(i1["history"][:m] - i2["history"][:m]) / i1["history"][:m]) < 1e-10
    assert np.abs(x1 - x2).max() / np.abs(x1).max() < 1e-10
    assert i1["final_norm"] <= 1e-8 * i1["bnorm"]


def test_pcg_threaded_reference_order(small_poisson):
    rp, ci, v, xt, b, J = small_poisson
    A = R.Matrix(rp, ci, v)
    x1, i1 = R.pcg_jacobi(A, J, b, red=R.RED_SEQ, nworkers=1)
    x4, i4 = R.pcg_jacobi(A, J, b, red=R.RED_SEQ, nworkers=4)
    xt4, it4 = R.pcg_jacobi(A, J, b, red=R.RED_TREE, nworkers=4)
    xt1, it1 = R.pcg_jacobi(A, J, b, red=R.RED_TREE, nworkers=1)
    assert np.array_equal(xt4, xt1)  # tree order does not depend on the thread count
    assert abs(i4["iter_done"] - i1["iter_done"]) <= 1
    assert np.abs(x4 - x1).max() / np.abs(x1).max() < 1e-10


def test_pcg_jad_equals_csr(small_poisson):
    rp, ci, v, xt, b, J = small_poisson
    xc, ic = R.pcg_jacobi(R.Matrix(rp, ci, v), J, b, red=R.RED_SEQ)
    xj, ij = R.pcg_jacobi(R.Matrix(rp, ci, v, R.FMT_JAD), J, b, red=R.RED_SEQ)
    assert np.array_equal(xc, xj) and ic["iter_done"] == ij["iter_done"]


def test_cg_corrected_and_literal(small_poisson):
    rp, ci, v, xt, b, J = small_poisson
    A = R.Matrix(rp, ci, v)
    x, info = R.cg(A, b, x0_mode=R.X0_ZERO, eps_abs=0.0, eps_rel=1e-8)
    assert info["err"] == 0 and np.abs(x - xt).max() < 1e-5
    # the reference's d = alpha d + r (cel_cgalg_module.f90:151) does not converge
    xl, il = R.cg(A, b, x0_mode=R.X0_ONES, eps_abs=1e-7, literal=True, iter_max=200)
    assert il["iter_done"] == 200 and il["final_norm"] > 1e-3 * il["bnorm"]


def test_gmres_corrected_and_literal(small_poisson):
    rp, ci, v, xt, b, J = small_poisson
    A = R.Matrix(rp, ci, v)
    x, info = R.gmres_jacobi(A, J, b, restart=30, iter_max=20)
    assert info["err"] == 0 and info["final_norm"] <= 1e-8 * info["bnorm"] * 1.01
    # the unrotated Givens update (cel_gmresalg_module.f90:722-727) stops with
    # a small |gamma| while the true residual is still large
    xl, il = R.gmres_jacobi(A, J, b, restart=30, iter_max=3, literal=True)
    assert il["final_norm"] > 1e-3 * il["bnorm"]


def test_pcg_breakdown_on_singular_system():
    """A zero row/column makes p.Ap = 0: the oracle stops with BREAKDOWN where
    the reference divides by zero (its guard at
    src/fop/cel_fop_vec_distr_module.f90:704-706 calls cel_error with err_code 0)."""
    rp = np.array([0, 1, 1], np.int32)
    ci = np.array([0], np.int32)
    v = np.array([1.0])
    A = R.Matrix(rp, ci, v)
    J = np.array([1.0, 1.0])
    x, info = R.pcg_jacobi(A, J, np.array([0.0, 1.0]), eps_rel=1e-8, iter_max=10)
    assert info["err"] == R.ERR_BREAKDOWN


def test_fp32_inner_pcg_reaches_tolerance(small_poisson):
    rp, ci, v, xt, b, J = small_poisson
    x32, info = R.pcg_jacobi_f32(rp, ci, v.astype(np.float32), J.astype(np.float32),
                                 b.astype(np.float32), eps_rel=1e-4)
    assert info["err"] == 0
    r = b - R.spmv_csr(rp, ci, v, x32.astype(np.float64))
    assert np.linalg.norm(r) <= 2e-4 * np.linalg.norm(b)
