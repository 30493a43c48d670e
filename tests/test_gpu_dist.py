"""Distributed Jacobi-PCG phases (celg_dist_*) on one GPU.

Several ranks are emulated in this process: each rank's kernels run in turn
on the one device, and LocalComm sums the exchange buffers in rank order and
copies the halos (no kernel waits on another rank's).  Checked bit for bit
against the CPU mirror of the same ranks, and -- for one rank -- against the
single-system solve.  The last test runs one rank through torch.distributed
with NCCL (world size 1) to check the stream ordering of the collectives."""
import numpy as np
import pytest

from cel_v3_b200 import dist as D
from cel_v3_b200 import synth
from oracle import celref as R
from tests import dist_mirror as M
from tests.helpers import random_csr, spd_from_pattern

pytestmark = pytest.mark.gpu

GRID = (20, 18, 16)


def poisson():
    rp, ci, v = synth.poisson7(*GRID)
    xt = np.random.default_rng(12).random(rp.size - 1)
    return rp, ci, v, R.spmv_csr(rp, ci, v, xt)


def random_spd(n=5000, seed=8):
    rp, ci, v = spd_from_pattern(*random_csr(n, np.random.default_rng(seed), max_len=7,
                                             empty_frac=0.0))
    return rp, ci, v, np.random.default_rng(seed + 1).uniform(-1, 1, n)


def blocks_of(rp, ci, v, world, align):
    bounds = D.partition(rp.size - 1, world, align)
    return [D.RowBlock(rp, ci, v, bounds, q) for q in range(world)]


def run_gpu(h, blocks, b, comm=None, overlap=False, windows=None, **kw):
    ranks = [D.GpuRank(h, blk, b[blk.r0:blk.r1], history=True, **kw) for blk in blocks]
    try:
        if windows is not None:
            windows.extend(r.interior_rows() for r in ranks)
        res = D.run_pcg(ranks, comm or D.LocalComm(), check_every=5, overlap=overlap)
        x = np.concatenate([r.x().cpu().numpy() for r in ranks])
    finally:
        for r in ranks:
            r.close()
    return x, res


def run_cpu(blocks, b, x0=None, **kw):
    ranks = [M.CpuRank(blk, b[blk.r0:blk.r1], x0=None if x0 is None else x0[blk.r0:blk.r1], **kw)
             for blk in blocks]
    res = D.run_pcg(ranks, D.LocalComm(), check_every=5)
    return np.concatenate([r.x() for r in ranks]), res


def test_one_rank_equals_single_system_solve(gpu):
    celgpu, h, torch = gpu
    rp, ci, v, b = poisson()
    x, (res,) = run_gpu(h, blocks_of(rp, ci, v, 1, 1), b, eps_rel=1e-8, iter_max=1000)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    info = h.pcg_jacobi(m, bd.data_ptr(), xd.data_ptr(), history=True, eps_rel=1e-8, iter_max=1000)
    m.destroy()
    assert res.status == celgpu.OK and info.status == celgpu.OK
    assert res.iter_done == info.iter_done
    assert np.array_equal(res.history, info.history)
    assert np.array_equal(x, xd.cpu().numpy())
    assert res.verified_relres == info.verified_relres


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("world", [2, 3, 4])
def test_emulated_slab_ranks_match_cpu_mirror(gpu, world, overlap):
    celgpu, h, torch = gpu
    rp, ci, v, b = poisson()
    blocks = blocks_of(rp, ci, v, world, GRID[0] * GRID[1])
    x, res = run_gpu(h, blocks, b, overlap=overlap, eps_rel=1e-8, iter_max=1000)
    xc, rc = run_cpu(blocks, b, eps_rel=1e-8, iter_max=1000)
    assert all(r.status == celgpu.OK for r in res)
    assert len({r.iter_done for r in res}) == 1
    assert res[0].iter_done == rc[0]["iter_done"]
    assert np.array_equal(res[0].history, rc[0]["history"])
    assert np.array_equal(x, xc)
    assert res[0].verified_relres == rc[0]["verified_relres"]
    assert res[0].verified_relres <= 1.5e-8


@pytest.mark.parametrize("world", [2, 3])
def test_split_spmv_phase_interior_windows_and_bits(gpu, world):
    """The SpMV phase in two launches around the halo (interior tiles while
    the halo copies run on a side stream, then the rest): on z-slabs of
    32x32x24 every 1024-row tile is one plane, the interior window leaves
    out exactly the planes next to a neighbour, and the solve has the bits
    of the one-launch phase and of the CPU mirror."""
    celgpu, h, torch = gpu
    rp, ci, v = synth.poisson7(32, 32, 24)
    b = R.spmv_csr(rp, ci, v, np.random.default_rng(13).random(rp.size - 1))
    blocks = blocks_of(rp, ci, v, world, 32 * 32)
    win = []
    x1, r1 = run_gpu(h, blocks, b, overlap=True, windows=win, eps_rel=1e-8, iter_max=1000)
    x0, r0 = run_gpu(h, blocks, b, eps_rel=1e-8, iter_max=1000)
    xc, rc = run_cpu(blocks, b, eps_rel=1e-8, iter_max=1000)
    for q, (blk, (lo, hi)) in enumerate(zip(blocks, win)):
        assert lo == (1024 if q > 0 else 0)
        assert hi == blk.n - (1024 if q < world - 1 else 0)
    assert all(r.status == celgpu.OK for r in r1)
    assert r1[0].iter_done == r0[0].iter_done == rc[0]["iter_done"]
    assert np.array_equal(r1[0].history, r0[0].history)
    assert np.array_equal(x1, x0)
    assert np.array_equal(x1, xc)


def test_emulated_general_partition_user_start(gpu):
    """Unaligned blocks of an unstructured matrix (scattered send lists),
    a user start vector and an iteration cap."""
    celgpu, h, torch = gpu
    rp, ci, v, b = random_spd()
    blocks = blocks_of(rp, ci, v, 3, 1)
    x0 = np.random.default_rng(2).random(rp.size - 1)
    kw = dict(eps_rel=1e-30, iter_max=12)
    ranks = [D.GpuRank(h, blk, b[blk.r0:blk.r1], x0=x0[blk.r0:blk.r1], history=True, **kw)
             for blk in blocks]
    res = D.run_pcg(ranks, D.LocalComm(), check_every=4)
    x = np.concatenate([r.x().cpu().numpy() for r in ranks])
    for r in ranks:
        r.close()
    ranks = [D.GpuRank(h, blk, b[blk.r0:blk.r1], x0=x0[blk.r0:blk.r1], history=True, **kw)
             for blk in blocks]
    res_o = D.run_pcg(ranks, D.LocalComm(), check_every=4, overlap=True)
    x_o = np.concatenate([r.x().cpu().numpy() for r in ranks])
    for r in ranks:
        r.close()
    xc, rc = run_cpu(blocks, b, x0=x0, **kw)
    assert all(r.status == celgpu.ERR_NOCONV and r.iter_done == 12 for r in res)
    assert np.array_equal(x, xc)
    assert np.array_equal(x_o, xc)
    assert np.array_equal(res[0].history, rc[0]["history"])
    assert np.array_equal(res_o[0].history, rc[0]["history"])


def banded_spd(n=40000, half_width=300, seed=5):
    """An unstructured banded SPD matrix: 6 random columns within
    half_width of each row, symmetrised."""
    rng = np.random.default_rng(seed)
    cols = [np.unique(np.clip(i + rng.integers(-half_width, half_width + 1, 6), 0, n - 1))
            for i in range(n)]
    rp = np.concatenate([[0], np.cumsum([c.size for c in cols])])
    rp, ci, v = spd_from_pattern(rp, np.concatenate(cols), rng.random(int(rp[-1])))
    return rp, ci, v, rng.uniform(-1, 1, n)


def test_interior_window_matches_host_restatement_on_unaligned_blocks(gpu):
    """The library's interior window (celg_dist_interior_rows) equals the
    host restatement (RowBlock.interior_rows: longest run of halo-free
    1024-row tiles, the first of equal runs) on unaligned blocks of an
    unstructured banded matrix, and the split SpMV phase over that window
    keeps the bits of the CPU mirror."""
    celgpu, h, torch = gpu
    rp, ci, v, b = banded_spd()
    blocks = blocks_of(rp, ci, v, 3, 1)
    assert any(blk.r0 % 1024 for blk in blocks)            # bounds cut tiles
    win = []
    x1, r1 = run_gpu(h, blocks, b, overlap=True, windows=win, eps_rel=1e-8, iter_max=400)
    for blk, w in zip(blocks, win):
        assert tuple(w) == blk.interior_rows()
        assert w[1] - w[0] >= 8 * 1024                    # halo reads only near the ends
    xc, rc = run_cpu(blocks, b, eps_rel=1e-8, iter_max=400)
    assert r1[0].iter_done == rc[0]["iter_done"]
    assert np.array_equal(r1[0].history, rc[0]["history"])
    assert np.array_equal(x1, xc)


def test_nccl_world_one(gpu):
    """One rank over torch.distributed with NCCL: the collectives queue on
    torch's stream between the phases; same bits as the single solve."""
    celgpu, h, torch = gpu
    import socket
    from datetime import timedelta

    import torch.distributed as td
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    td.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                          timeout=timedelta(seconds=60))
    try:
        rp, ci, v, b = poisson()
        x, (res,) = run_gpu(h, blocks_of(rp, ci, v, 1, 1), b, comm=D.TorchComm(), eps_rel=1e-8,
                            iter_max=1000)
    finally:
        td.destroy_process_group()
    xl, (rl,) = run_gpu(h, blocks_of(rp, ci, v, 1, 1), b, eps_rel=1e-8, iter_max=1000)
    assert res.status == celgpu.OK
    assert res.iter_done == rl.iter_done
    assert np.array_equal(x, xl)
