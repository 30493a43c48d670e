"""Batched Jacobi-PCG (celg_pcg_batched): every system of the batch must give
the same bits as solving it alone with celg_pcg_jacobi (same reduction order
per system), whatever the mix of sizes, including systems whose row count is
not a multiple of the 1024-row tile and an empty one."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def systems():
    rng = np.random.default_rng(4)
    out = []
    for side in (16, 5, 23, 31, 9, 40, 12):
        _, (kx, ky, kz) = synth.lognormal_faces(rng, side, side + 1, side, 0.5)
        rp, ci, v = synth.diffusion7(side, side + 1, side, kx, ky, kz)
        out.append((rp, ci, v, rng.uniform(-1.0, 1.0, rp.size - 1)))
    return out


@pytest.mark.parametrize("x0", ["zero", "ones"])
def test_batched_matches_single_solves_bitwise(gpu, x0):
    celgpu, h, torch = gpu
    sy = systems()
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for rp, ci, v, _ in sy]
    bs = [dev(torch, b) for *_, b in sy]
    xs = [dev(torch, np.zeros(b.size)) for *_, b in sy]
    mode = celgpu.X0_ZERO if x0 == "zero" else celgpu.X0_REF_ONES
    kw = dict(eps_rel=1e-9, iter_max=3000, x0_mode=mode)
    infos = h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], **kw)
    for s, ((rp, ci, v, b), m) in enumerate(zip(sy, mats)):
        xo = dev(torch, np.zeros(b.size))
        one = h.pcg_jacobi(m, bs[s].data_ptr(), xo.data_ptr(), **kw)
        assert infos[s].status == celgpu.OK and one.status == celgpu.OK
        assert infos[s].iter_done == one.iter_done
        assert infos[s].final_norm2 == one.final_norm2
        assert infos[s].verified_relres == one.verified_relres
        assert np.array_equal(xs[s].cpu().numpy(), xo.cpu().numpy())
    # and against the oracle in tree order for one of them
    rp, ci, v, b = sy[3]
    xr, ir = R.pcg_jacobi(R.Matrix(rp, ci, v), R.jacobi(R.diag(rp, ci, v)), b, eps_rel=1e-9,
                          iter_max=3000, red=R.RED_TREE,
                          x0_mode=R.X0_ZERO if x0 == "zero" else R.X0_ONES)
    assert np.array_equal(xs[3].cpu().numpy(), xr) and ir["iter_done"] == infos[3].iter_done
    # a second launch of the cached batch graph gives the same bits
    xs2 = [dev(torch, np.zeros(b.size)) for *_, b in sy]
    infos2 = h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs2], **kw)
    for s in range(len(sy)):
        assert np.array_equal(xs2[s].cpu().numpy(), xs[s].cpu().numpy())
        assert infos2[s].iter_done == infos[s].iter_done
    for m in mats:
        m.destroy()


def test_batched_with_empty_system_and_cap(gpu):
    celgpu, h, torch = gpu
    sy = systems()[:3]
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for rp, ci, v, _ in sy]
    empty = h.matrix_from_csr(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)).jacobi()
    bs = [dev(torch, b) for *_, b in sy]
    xs = [dev(torch, np.zeros(b.size)) for *_, b in sy]
    infos = h.pcg_batched(mats + [empty], [b.data_ptr() for b in bs] + [0],
                          [x.data_ptr() for x in xs] + [0], eps_rel=1e-12, iter_max=5)
    for s in range(3):
        assert infos[s].iter_done == 5 and infos[s].status == celgpu.ERR_NOCONV
        # the capped systems' x equal single solves capped the same way
        xs1 = dev(torch, np.zeros(bs[s].numel()))
        h.pcg_jacobi(mats[s], bs[s].data_ptr(), xs1.data_ptr(), eps_rel=1e-12, iter_max=5)
        assert torch.equal(xs[s], xs1)
    assert infos[3].iter_done == 0 and infos[3].status == celgpu.OK
    for m in mats + [empty]:
        m.destroy()


@pytest.mark.parametrize("mode", ["graph", "host_loop"])
def test_batched_fp32_refinement_matches_single_refinement(gpu, mode, monkeypatch):
    """FP32 refinement of the whole batch (CELG_PREC_FP32_IR): each system's
    solution, outer and inner iteration counts and verified residual equal
    the single-system refinement's bit for bit."""
    celgpu, h, torch = gpu
    if mode == "host_loop":
        monkeypatch.setenv("CELG_GRAPH", "0")
    sy = systems()
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for rp, ci, v, _ in sy]
    bs = [dev(torch, b) for *_, b in sy]
    xs = [dev(torch, np.zeros(b.size)) for *_, b in sy]
    kw = dict(eps_rel=1e-10, iter_max=3000, precision=celgpu.PREC_FP32_IR, inner_eps_rel=1e-4,
              inner_iter_max=1500, outer_max=20, x0_mode=celgpu.X0_ZERO)
    infos = h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], **kw)
    for s, ((rp, ci, v, b), m) in enumerate(zip(sy, mats)):
        xo = dev(torch, np.zeros(b.size))
        one = h.pcg_jacobi(m, bs[s].data_ptr(), xo.data_ptr(), **kw)
        assert infos[s].status == one.status == celgpu.OK, s
        assert infos[s].iter_done == one.iter_done, s            # outer steps
        assert infos[s].arnoldi_steps == one.arnoldi_steps, s    # inner iterations
        assert infos[s].verified_relres == one.verified_relres, s
        assert infos[s].verified_relres <= 1e-10
        assert np.array_equal(xs[s].cpu().numpy(), xo.cpu().numpy()), s
    for m in mats:
        m.destroy()


@pytest.mark.parametrize("mode", ["graph", "host_loop"])
@pytest.mark.parametrize("iter_max", [3000, 7])
def test_batched_fp32_reliable_updates_match_single_solves(gpu, mode, iter_max, monkeypatch):
    """FP32 PCG with FP64 reliable updates of the whole batch
    (CELG_PREC_FP32_RU): each system's solution, iteration and update counts,
    last FP64 residual norm, status and verified residual equal the single
    reliable-update solve's bit for bit, also when the iteration cap forces
    the last update; an empty system is skipped."""
    celgpu, h, torch = gpu
    if mode == "host_loop":
        monkeypatch.setenv("CELG_GRAPH", "0")
    sy = systems()
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for rp, ci, v, _ in sy]
    empty = h.matrix_from_csr(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)).jacobi()
    bs = [dev(torch, b) for *_, b in sy]
    xs = [dev(torch, np.zeros(b.size)) for *_, b in sy]
    kw = dict(eps_rel=1e-10, iter_max=iter_max, precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2,
              x0_mode=celgpu.X0_ZERO)
    infos = h.pcg_batched(mats + [empty], [b.data_ptr() for b in bs] + [0],
                          [x.data_ptr() for x in xs] + [0], **kw)
    for s, ((rp, ci, v, b), m) in enumerate(zip(sy, mats)):
        xo = dev(torch, np.zeros(b.size))
        one = h.pcg_jacobi(m, bs[s].data_ptr(), xo.data_ptr(), **kw)
        assert infos[s].status == one.status, s
        assert infos[s].iter_done == one.iter_done, s
        assert infos[s].arnoldi_steps == one.arnoldi_steps, s      # reliable updates
        assert infos[s].final_norm2 == one.final_norm2, s
        assert infos[s].verified_relres == one.verified_relres, s
        assert np.array_equal(xs[s].cpu().numpy(), xo.cpu().numpy()), s
        if iter_max == 3000:
            assert one.status == celgpu.OK and one.verified_relres <= 1e-10
        else:
            assert one.status == celgpu.ERR_NOCONV and one.iter_done == iter_max
    assert infos[-1].iter_done == 0 and infos[-1].status == celgpu.OK
    for m in mats + [empty]:
        m.destroy()


def test_batched_launch_shapes_give_the_same_bits(gpu, monkeypatch):
    """Every launch shape the batch tuner chooses from (CTAs per SM of the
    SpMV and vector sweeps, forced with CELG_BATCH_SHAPE on a fresh handle)
    gives the same bits, and celg_tuned_config reports the shape in use."""
    celgpu, h, torch = gpu
    sy = systems()[:5]
    kw = dict(eps_rel=1e-9, iter_max=3000, x0_mode=celgpu.X0_ZERO)
    shapes = [(0, 8), (0, 6), (0, 4), (2, 8), (2, 4), (1, 8)]
    ref = None
    for c, shape in enumerate(shapes + [None]):
        if shape is None:
            monkeypatch.delenv("CELG_BATCH_SHAPE", raising=False)   # the tuner's own pick
        else:
            monkeypatch.setenv("CELG_BATCH_SHAPE", str(c))
        hq = celgpu.Handle(0, torch.cuda.current_stream().cuda_stream)
        mats = [hq.matrix_from_csr(rp, ci, v).jacobi() for rp, ci, v, _ in sy]
        bs = [dev(torch, b) for *_, b in sy]
        xs = [dev(torch, np.zeros(b.size)) for *_, b in sy]
        infos = hq.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], **kw)
        got = hq.tuned_config(celgpu.TUNE_BATCH)
        assert got in shapes and (shape is None or got == shape)
        out = [x.cpu().numpy() for x in xs] + [i.iter_done for i in infos]
        if ref is None:
            ref = out
        for a, b in zip(out, ref):
            assert np.array_equal(a, b)
        for m in mats:
            m.destroy()
        hq.close()


def test_batched_fp32_reliable_updates_unstructured(gpu):
    """Unstructured systems (the batch reads int32 columns): each system
    still equals its single reliable-update solve bit for bit."""
    celgpu, h, torch = gpu
    from tests.helpers import random_csr, spd_from_pattern
    rng = np.random.default_rng(22)
    sy = []
    for n in (1500, 700, 2300):
        rp, ci, v = spd_from_pattern(*random_csr(n, rng, max_len=9, empty_frac=0.0))
        sy.append((rp, ci, v, rng.uniform(-1.0, 1.0, n)))
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for rp, ci, v, _ in sy]
    bs = [dev(torch, b) for *_, b in sy]
    xs = [dev(torch, np.zeros(b.size)) for *_, b in sy]
    kw = dict(eps_rel=1e-10, iter_max=3000, precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2,
              x0_mode=celgpu.X0_ZERO)
    infos = h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], **kw)
    for s, m in enumerate(mats):
        xo = dev(torch, np.zeros(bs[s].numel()))
        one = h.pcg_jacobi(m, bs[s].data_ptr(), xo.data_ptr(), **kw)
        assert infos[s].status == one.status == celgpu.OK, s
        assert infos[s].iter_done == one.iter_done and infos[s].arnoldi_steps == one.arnoldi_steps, s
        assert np.array_equal(xs[s].cpu().numpy(), xo.cpu().numpy()), s
    for m in mats:
        m.destroy()
