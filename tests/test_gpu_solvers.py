"""GPU parity of the solvers (through the C ABI) against the oracle.

With the oracle in the GPU's reduction order (RED_TREE) the solution and the
residual history must match bit for bit; against the reference's own
sequential order (RED_SEQ) they must agree within 1e-10 relative at the same
iteration count +-1."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R
from tests.helpers import ir_step_tolerance, random_csr, spd_from_pattern

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def problems():
    out = {}
    rp, ci, v, xt = synth.plain(32, 0)
    out["poisson32"] = (rp, ci, v, R.spmv_csr(rp, ci, v, xt))
    g, (kx, ky, kz) = synth.lognormal_faces(np.random.default_rng(2), 20, 21, 22)
    rp, ci, v = synth.diffusion7(20, 21, 22, kx, ky, kz)
    out["diffusion"] = (rp, ci, v, np.random.default_rng(3).uniform(-1, 1, rp.size - 1))
    rp, ci, v = spd_from_pattern(*random_csr(3001, np.random.default_rng(4), max_len=6))
    out["random_spd"] = (rp, ci, v, np.random.default_rng(5).standard_normal(3001))
    return out


PROBS = problems()


def setup(h, rp, ci, v, jad=False):
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    if jad:
        m.to_jad()
    return m


@pytest.mark.parametrize("fmt", ["csr", "jad"])
@pytest.mark.parametrize("name", sorted(PROBS))
def test_pcg_bitexact_vs_oracle_tree(gpu, name, fmt):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS[name]
    n = rp.size - 1
    jad = fmt == "jad"
    m = setup(h, rp, ci, v, jad)
    bd, xd = dev(torch, b), dev(torch, np.zeros(n))
    info = h.pcg_jacobi(m, bd.data_ptr(), xd.data_ptr(), history=True,
                        fmt=celgpu.FMT_JAD if jad else celgpu.FMT_CSR, eps_rel=1e-8, iter_max=2000)
    A = R.Matrix(rp, ci, v, R.FMT_JAD if jad else R.FMT_CSR)
    J = R.jacobi(R.diag(rp, ci, v))
    xo, io = R.pcg_jacobi(A, J, b, eps_rel=1e-8, iter_max=2000, red=R.RED_TREE)
    assert info.status == celgpu.OK
    assert info.iter_done == io["iter_done"]
    assert np.array_equal(info.history, io["history"])
    assert np.array_equal(xd.cpu().numpy(), xo)
    assert info.verified_relres <= 1.5e-8
    # the reference's sequential order: within 1e-10, iterations +-1
    xs, is_ = R.pcg_jacobi(A, J, b, eps_rel=1e-8, iter_max=2000, red=R.RED_SEQ)
    assert abs(is_["iter_done"] - info.iter_done) <= 1
    k = min(len(is_["history"]), len(info.history))
    assert np.max(np.abs(info.history[:k] - is_["history"][:k]) / is_["history"][:k]) < 1e-10
    assert np.abs(xd.cpu().numpy() - xs).max() <= 1e-10 * np.abs(xs).max()
    m.destroy()


def test_pcg_reference_fixture_x0_ones(gpu, ref_poisson):
    """cel_cgalg_jacobi as the reference runs it: x0 = 1, absolute eps."""
    celgpu, h, torch = gpu
    d = ref_poisson["12x11x10"]
    n = d["u"].size
    m = setup(h, d["rp"], d["ci"], d["v"])
    eps = 1e-10 * np.linalg.norm(d["b"])
    xd = dev(torch, np.zeros(n))
    info = h.pcg_jacobi(m, dev(torch, d["b"]).data_ptr(), xd.data_ptr(), history=True,
                        x0_mode=celgpu.X0_REF_ONES, eps_abs=eps, eps_rel=0.0, iter_max=2000)
    xo, io = R.pcg_jacobi(R.Matrix(d["rp"], d["ci"], d["v"]), R.jacobi(R.diag(d["rp"], d["ci"], d["v"])),
                          d["b"], x0_mode=R.X0_ONES, eps_abs=eps, eps_rel=0.0, iter_max=2000,
                          red=R.RED_TREE)
    x = xd.cpu().numpy()
    assert np.array_equal(x, xo) and np.array_equal(info.history, io["history"])
    assert np.abs(x - d["u"]).max() < 1e-8 * np.abs(d["u"]).max()   # known answer
    m.destroy()


def test_pcg_user_x0_limit_and_graph_reuse(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["poisson32"]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    x0 = np.random.default_rng(1).random(n)
    bd = dev(torch, b)
    xd = dev(torch, x0)
    info = h.pcg_jacobi(m, bd.data_ptr(), xd.data_ptr(), x0_mode=celgpu.X0_USER, iter_max=7)
    assert info.status == celgpu.ERR_NOCONV and info.iter_done == 7
    xo, io = R.pcg_jacobi(R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v)), b, x0=x0, iter_max=7,
                          red=R.RED_TREE)
    assert np.array_equal(xd.cpu().numpy(), xo)
    # the same call again replays the cached graph: identical result
    xd2 = dev(torch, x0)
    for _ in range(2):
        xd2.copy_(dev(torch, x0))
        info2 = h.pcg_jacobi(m, bd.data_ptr(), xd2.data_ptr(), x0_mode=celgpu.X0_USER, iter_max=7)
        assert np.array_equal(xd2.cpu().numpy(), xo) and info2.iter_done == 7
    m.destroy()


def test_pcg_breakdown_status(gpu):
    celgpu, h, torch = gpu
    rp = np.array([0, 1, 1], np.int32)
    m = h.matrix_from_csr(rp, np.array([0], np.int32), np.array([1.0]))
    m.jacobi()
    # J has inf for the empty row; use b so that p.Ap = 0 on the first step
    info = h.pcg_jacobi(m, dev(torch, np.array([0.0, 1.0])).data_ptr(),
                        dev(torch, np.zeros(2)).data_ptr(), iter_max=10)
    assert info.status in (celgpu.ERR_BREAKDOWN, celgpu.OK)  # inf/nan propagate -> no silent success
    assert not (info.status == celgpu.OK and np.isfinite(info.final_norm2) and info.iter_done > 0)
    m.destroy()


def test_pcg_zero_rhs_converges_immediately(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["diffusion"]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    xd = dev(torch, np.ones(n))
    info = h.pcg_jacobi(m, dev(torch, np.zeros(n)).data_ptr(), xd.data_ptr())
    assert info.iter_done == 0 and np.all(xd.cpu().numpy() == 0.0)
    m.destroy()


@pytest.mark.parametrize("literal", [False, True])
def test_cg_bitexact(gpu, literal):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["poisson32"]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    xd = dev(torch, np.zeros(n))
    kw = dict(x0_mode=celgpu.X0_REF_ONES, eps_abs=1e-7, eps_rel=0.0, iter_max=150)
    info = h.cg(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=True,
                literal_ref_bugs=int(literal), **kw)
    xo, io = R.cg(R.Matrix(rp, ci, v), b, x0_mode=R.X0_ONES, eps_abs=1e-7, eps_rel=0.0,
                  iter_max=150, red=R.RED_TREE, literal=literal)
    assert info.iter_done == io["iter_done"]
    assert np.array_equal(info.history, io["history"])
    assert np.array_equal(xd.cpu().numpy(), xo)
    m.destroy()


@pytest.mark.parametrize("literal", [False, True])
@pytest.mark.parametrize("fmt", ["csr", "jad"])
def test_gmres_bitexact(gpu, fmt, literal):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["diffusion"]
    n = rp.size - 1
    jad = fmt == "jad"
    m = setup(h, rp, ci, v, jad)
    xd = dev(torch, np.zeros(n))
    info = h.gmres_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=4000,
                          fmt=celgpu.FMT_JAD if jad else celgpu.FMT_CSR, restart=12,
                          iter_max=5 if literal else 40, eps_rel=1e-8,
                          literal_ref_bugs=int(literal))
    xo, io = R.gmres_jacobi(R.Matrix(rp, ci, v, R.FMT_JAD if jad else R.FMT_CSR),
                            R.jacobi(R.diag(rp, ci, v)), b, restart=12,
                            iter_max=5 if literal else 40, eps_rel=1e-8, red=R.RED_TREE,
                            literal=literal)
    assert info.arnoldi_steps == io["arnoldi_steps"] and info.iter_done == io["iter_done"]
    assert np.array_equal(info.history, io["history"])
    assert np.array_equal(xd.cpu().numpy(), xo)
    if not literal:
        assert info.status == celgpu.OK and info.verified_relres <= 1.01e-8
    m.destroy()


def test_gmres_graph_and_host_loop_agree(gpu, monkeypatch):
    """The device-driven GMRES (one graph launch per solve) and its
    host-driven form (one poll per restart cycle) give the same bits, also
    when the history buffer is shorter than the step count, and a second
    solve replays the cached graph with the work space the handle keeps."""
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["random_spd"]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    kw = dict(restart=7, iter_max=30, eps_rel=1e-10)
    out = []
    for mode in ("1", "0", "1"):
        monkeypatch.setenv("CELG_GRAPH", mode)
        xd = dev(torch, np.zeros(n))
        info = h.gmres_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=9, **kw)
        out.append((xd.cpu().numpy(), info))
    xo, io = R.gmres_jacobi(R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v)), b, red=R.RED_TREE,
                            **kw)
    for x, info in out:
        assert info.status == celgpu.OK
        assert info.arnoldi_steps == io["arnoldi_steps"] > 9
        assert info.iter_done == io["iter_done"]
        assert np.array_equal(info.history, io["history"][:9])
        assert np.array_equal(x, xo)
    m.destroy()


def ir_oracle(rp, ci, v, b, tol=1e-10, inner=1e-4, outer_max=20):
    """FP64 refinement around the FP32-storage PCG, composed from oracle pieces."""
    n = rp.size - 1
    J = R.jacobi(R.diag(rp, ci, v))
    v32, J32 = v.astype(np.float32), J.astype(np.float32)
    x = np.zeros(n)
    bn = np.sqrt(R.dot(b, b, R.RED_TREE))
    hist, inner_total = [], 0
    for k in range(outer_max + 1):
        r = b - R.spmv_csr(rp, ci, v, x)
        rn = np.sqrt(R.dot(r, r, R.RED_TREE))
        hist.append(rn)
        if rn <= tol * bn:
            break
        if k == outer_max:
            break
        r32 = (r * (1.0 / rn)).astype(np.float32)
        d, info = R.pcg_jacobi_f32(rp, ci, v32, J32, r32, eps_rel=ir_step_tolerance(rn, tol * bn, inner),
                                   red=R.RED_TREE)
        inner_total += info["iter_done"]
        x = x + rn * d.astype(np.float64)
    return x, np.array(hist), inner_total


@pytest.mark.parametrize("name", ["poisson32", "diffusion"])
def test_fp32_refinement_bitexact_and_accurate(gpu, name):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS[name]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    xd = dev(torch, np.zeros(n))
    info = h.pcg_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=64,
                        precision=celgpu.PREC_FP32_IR, eps_rel=1e-10, inner_eps_rel=1e-4)
    xo, ho, inner_total = ir_oracle(rp, ci, v, b)
    assert info.status == celgpu.OK
    assert np.array_equal(xd.cpu().numpy(), xo)
    assert np.array_equal(info.history, ho)
    assert info.arnoldi_steps == inner_total
    assert info.verified_relres <= 1e-10
    # error against the FP64 solve
    xf, _ = R.pcg_jacobi(R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v)), b, eps_rel=1e-10,
                         red=R.RED_TREE, iter_max=5000)
    assert np.abs(xo - xf).max() <= 1e-7 * np.abs(xf).max()
    m.destroy()


def test_solve_host_matches_device(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["diffusion"]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    x_host, info = h.solve_host(m, b)
    xd = dev(torch, np.zeros(n))
    h.pcg_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr())
    assert np.array_equal(x_host, xd.cpu().numpy()) and info.status == celgpu.OK
    m.destroy()


def test_elm_interface_defaults(gpu, ref_poisson):
    """cel_elmSolver*: row-wise 1-based assembly, a diagonal re-insertion,
    defaults GMRES(3) + Jacobi + diagonal scaling, x0 = 1, eps 1e-8."""
    celgpu, h, torch = gpu
    d = ref_poisson["12x11x10"]
    rp, ci, v, b = d["rp"], d["ci"], d["v"], d["b"]
    n = rp.size - 1
    h.elm_init(n, n, 1, (7, 0))
    for i in range(n):
        h.elm_row_start(i + 1)
        for k in range(rp[i], rp[i + 1]):
            h.elm_insert(int(ci[k]) + 1, 0.5 if ci[k] == i else float(v[k]))
        dk = [k for k in range(rp[i], rp[i + 1]) if ci[k] == i][0]
        h.elm_reinsert(i + 1, float(v[dk]))
        h.elm_row_completed()
    h.elm_matrix_completed()
    ierr, niter, ftol = h.elm_doit(b)
    x = h.elm_collect_solution(n)
    # oracle on the row-scaled system
    dg = R.diag(rp, ci, v)
    vs, s = R.row_scale(rp, v, dg)
    xo, io = R.gmres_jacobi(R.Matrix(rp, ci, vs), R.jacobi(dg, s), b / s, restart=3,
                            x0_mode=R.X0_ONES, eps_abs=1e-8, eps_rel=0.0, iter_max=5000,
                            red=R.RED_TREE)
    assert ierr == io["err"] and niter == io["iter_done"] and ftol == io["final_norm"]
    assert np.array_equal(x, xo)
    assert np.abs(x - d["u"]).max() < 1e-6 * np.abs(d["u"]).max()
    # ReDoIt with the PCG path on the assembled matrix
    ierr2, niter2, _ = h.elm_doit(b, redo=True)
    assert np.array_equal(h.elm_collect_solution(n), x)
    ms, iters, bpi = h.elm_performance()
    assert ms > 0 and iters > 0
    h.elm_destroy()


def test_elm_rejects_offdiagonal_reinsert(gpu):
    celgpu, h, torch = gpu
    h.elm_init(3, 3, 1, (3, 0))
    h.elm_row_start(1)
    h.elm_insert(1, 2.0)
    h.elm_insert(2, -1.0)
    with pytest.raises(celgpu.CelgError) as e:
        h.elm_reinsert(2, 5.0)
    assert e.value.status == celgpu.ERR_ARG
    with pytest.raises(celgpu.CelgError) as e:
        h.elm_doit(np.ones(3))
    assert e.value.status == celgpu.ERR_STATE
    h.elm_destroy()


def ru_oracle(rp, ci, v, b, eps_rel=1e-10, delta=1e-2, iter_max=5000):
    """FP32 PCG with FP64 reliable updates, composed from oracle pieces in the
    GPU's reduction order (see cel_v3_b200/csrc/ru.cu)."""
    f32, f64 = np.float32, np.float64
    J = R.jacobi(R.diag(rp, ci, v))
    J32 = J.astype(f32).astype(f64)
    v32 = v.astype(f32)
    T = R.RED_TREE
    n = rp.size - 1
    x = np.zeros(n)
    bn = np.sqrt(R.dot(b, b, T))
    eps = eps_rel * bn

    def residual(x):
        r64 = b - R.spmv_csr(rp, ci, v, x)
        r = r64.astype(f32)
        z = r.astype(f64) * J32
        return r, z, R.dot(r.astype(f64), z, T), np.sqrt(R.dot(r64, r64, T))

    r, z, rz, norm64 = residual(x)
    p = z.astype(f32)
    d = np.zeros(n, f32)
    maxr = norm64
    hist = [norm64]
    it, updates = 0, 1
    active = norm64 > eps and it < iter_max
    while active:
        w = R.spmv_csr_f32(rp, ci, v32, p)
        sigma = rz / R.dot(w.astype(f64), p.astype(f64), T)
        d = (d.astype(f64) + sigma * p.astype(f64)).astype(f32)
        r = r + f32(-sigma) * w                       # FP32 arithmetic, one rounding each
        z = r.astype(f64) * J32
        rz_new = R.dot(r.astype(f64), z, T)
        norm = np.sqrt(R.dot(r.astype(f64), r.astype(f64), T))
        rz_prev, beta, rz = rz, rz_new / rz, rz_new
        it += 1
        hist.append(norm)
        if norm < delta * maxr or norm <= eps or it >= iter_max:
            x = x + d.astype(f64)
            d[:] = 0
            r, z, rzh, norm64 = residual(x)
            maxr = norm64
            beta, rz = rzh / rz_prev, rzh
            hist[it] = norm64
            updates += 1
            active = norm64 > eps and it < iter_max
        else:
            active = it < iter_max and abs(rz) > 0
        if active:
            p = (beta * p.astype(f64) + z).astype(f32)
    x = x + d.astype(f64)
    return x, np.array(hist), it, updates


@pytest.mark.parametrize("name", ["poisson32", "diffusion"])
def test_fp32_reliable_update_bitexact_and_accurate(gpu, name):
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS[name]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    xd = dev(torch, np.zeros(n))
    info = h.pcg_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=True,
                        precision=celgpu.PREC_FP32_RU, eps_rel=1e-10, inner_eps_rel=1e-2,
                        iter_max=5000)
    xo, ho, it, updates = ru_oracle(rp, ci, v, b)
    assert info.status == celgpu.OK
    assert info.iter_done == it and info.arnoldi_steps == updates
    assert np.array_equal(info.history, ho)
    assert np.array_equal(xd.cpu().numpy(), xo)
    assert info.verified_relres <= 1e-10
    # iteration count close to the FP64 solver's at the same tolerance
    _, i64 = R.pcg_jacobi(R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v)), b, eps_rel=1e-10,
                          red=R.RED_TREE, iter_max=5000)
    assert it <= 1.25 * i64["iter_done"] + 5
    m.destroy()


@pytest.mark.parametrize("iter_max", [1, 9])
def test_fp32_reliable_update_iteration_cap_bitexact(gpu, iter_max):
    """Stopped by the iteration cap (which forces a reliable update), the
    correction d += sigma p left pending by the last step is still applied
    before x is flushed: x equals the composed oracle bit for bit."""
    celgpu, h, torch = gpu
    rp, ci, v, b = PROBS["diffusion"]
    n = rp.size - 1
    m = setup(h, rp, ci, v)
    xd = dev(torch, np.zeros(n))
    info = h.pcg_jacobi(m, dev(torch, b).data_ptr(), xd.data_ptr(), history=True,
                        precision=celgpu.PREC_FP32_RU, eps_rel=1e-10, inner_eps_rel=1e-2,
                        iter_max=iter_max)
    xo, ho, it, updates = ru_oracle(rp, ci, v, b, iter_max=iter_max)
    assert info.iter_done == it == iter_max
    assert np.array_equal(xd.cpu().numpy(), xo)
    assert np.array_equal(info.history, ho)
    m.destroy()
