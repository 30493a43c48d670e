"""Row-block distribution (cel_v3_b200.dist) on the CPU: partition and halo
lists, the exchange code over gloo with two processes, and the distributed
PCG recurrence (tests/dist_mirror.py) against the single-system oracle."""
import os
import socket

import numpy as np
import pytest

from cel_v3_b200 import dist as D
from cel_v3_b200 import synth
from oracle import celref as R
from tests import dist_mirror as M
from tests.helpers import random_csr, spd_from_pattern

GRID = (9, 8, 7)


def poisson():
    rp, ci, v = synth.poisson7(*GRID)
    xt = np.random.default_rng(11).random(rp.size - 1)
    return rp, ci, v, R.spmv_csr(rp, ci, v, xt)


def random_spd(n=700, seed=3):
    rp, ci, v = spd_from_pattern(*random_csr(n, np.random.default_rng(seed), max_len=6,
                                             empty_frac=0.0))
    b = np.random.default_rng(seed + 1).uniform(-1, 1, n)
    return rp, ci, v, b


def test_partition():
    assert D.partition(10, 1) == [0, 10]
    assert D.partition(100, 3, 4) == [0, 32, 64, 100]
    nx, ny, nz = GRID
    b = D.partition(nx * ny * nz, 4, nx * ny)
    assert b[0] == 0 and b[-1] == nx * ny * nz
    assert all(x % (nx * ny) == 0 for x in b)
    assert all(b[i] <= b[i + 1] for i in range(4))
    with pytest.raises(ValueError):
        D.partition(10, 0)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
@pytest.mark.parametrize("kind", ["slab", "random"])
def test_row_blocks_reproduce_global_spmv(world, kind):
    if kind == "slab":
        rp, ci, v, _ = poisson()
        bounds = D.partition(rp.size - 1, world, GRID[0] * GRID[1])
    else:
        rp, ci, v, _ = random_spd()
        bounds = D.partition(rp.size - 1, world)
    n = rp.size - 1
    x = np.random.default_rng(5).standard_normal(n)
    y = R.spmv_csr(rp, ci, v, x)
    blocks = [D.RowBlock(rp, ci, v, bounds, q) for q in range(world)]
    for q, blk in enumerate(blocks):
        x_ext = np.concatenate([x[blk.r0:blk.r1], x[blk.halo]])
        assert np.array_equal(R.spmv_csr(blk.rp, blk.ci, blk.v, x_ext), y[blk.r0:blk.r1])
        # what q receives from r is what r sends to q, in halo order
        for r, (off, cnt) in blk.recv.items():
            sent = blocks[r].send[q] + blocks[r].r0
            assert np.array_equal(sent, blk.halo[off:off + cnt])
        assert set(blk.send) == {r for r in range(world) if q in blocks[r].recv}
    if kind == "slab" and world > 1:
        # z-slabs exchange one plane with each neighbour, contiguously
        plane = GRID[0] * GRID[1]
        for blk in blocks:
            assert set(blk.neighbours()) <= {blk.rank - 1, blk.rank + 1}
            for q in blk.send:
                assert blk.send_range(q) is not None and blk.send_range(q)[1] == plane


def run_mirror(rp, ci, v, b, world, align=1, **kw):
    bounds = D.partition(rp.size - 1, world, align)
    blocks = [D.RowBlock(rp, ci, v, bounds, q) for q in range(world)]
    ranks = [M.CpuRank(blk, b[blk.r0:blk.r1], **kw) for blk in blocks]
    res = D.run_pcg(ranks, D.LocalComm(), check_every=3)
    return np.concatenate([r.x() for r in ranks]), res


def test_mirror_one_rank_is_the_oracle_solve():
    rp, ci, v, b = poisson()
    x, (res,) = run_mirror(rp, ci, v, b, 1, eps_rel=1e-10, iter_max=500)
    A = R.Matrix(rp, ci, v)
    xo, io = R.pcg_jacobi(A, R.jacobi(R.diag(rp, ci, v)), b, eps_rel=1e-10, iter_max=500,
                          red=R.RED_TREE)
    assert res["iter_done"] == io["iter_done"]
    assert np.array_equal(res["history"], io["history"])
    assert np.array_equal(x, xo)
    # the reference's absolute |r.z| guard ends this small solve near 1e-9
    assert res["verified_relres"] <= 1e-8


@pytest.mark.parametrize("world", [2, 3, 4])
def test_mirror_ranks_converge_like_one(world):
    rp, ci, v, b = poisson()
    x1, (r1,) = run_mirror(rp, ci, v, b, 1, eps_rel=1e-10, iter_max=500)
    xw, rw = run_mirror(rp, ci, v, b, world, align=GRID[0] * GRID[1], eps_rel=1e-10, iter_max=500)
    assert len({r["iter_done"] for r in rw}) == 1          # every rank stops together
    assert abs(rw[0]["iter_done"] - r1["iter_done"]) <= 1
    assert np.abs(xw - x1).max() <= 1e-9 * np.abs(x1).max()
    assert rw[0]["verified_relres"] <= 1e-8


def test_interior_rows_of_slabs_and_general_blocks():
    """The interior window: on z-slabs of 32x32x24 (one plane per 1024-row
    tile) every plane but those next to a neighbour; on general blocks, a
    run of tiles with no halo column that no other such run outgrows."""
    rp, ci, v = synth.poisson7(32, 32, 24)
    for world in (1, 2, 3):
        bounds = D.partition(rp.size - 1, world, 32 * 32)
        for q in range(world):
            blk = D.RowBlock(rp, ci, v, bounds, q)
            assert blk.interior_rows() == (1024 if q > 0 else 0,
                                           blk.n - (1024 if q < world - 1 else 0))
    # a banded unstructured matrix (columns within 100 of the row), cut at
    # unaligned bounds: the halo reads sit near the block ends
    rng = np.random.default_rng(5)
    n = 5000
    cols = [np.unique(np.clip(i + rng.integers(-100, 101, 6), 0, n - 1)) for i in range(n)]
    rp = np.concatenate([[0], np.cumsum([c.size for c in cols])])
    ci = np.concatenate(cols)
    rp, ci, v = spd_from_pattern(rp, ci, rng.random(ci.size))
    bounds = D.partition(n, 3)
    for q in range(3):
        blk = D.RowBlock(rp, ci, v, bounds, q)
        lo, hi = blk.interior_rows(tile=64)
        assert hi - lo >= 1024
        assert lo % 64 == 0 and lo <= hi <= blk.n
        assert (blk.ci[blk.rp[lo]:blk.rp[hi]] < blk.n).all()
        # the run cannot grow: the tiles on either side read the halo
        if lo >= 64:
            assert (blk.ci[blk.rp[lo - 64]:blk.rp[lo]] >= blk.n).any()
        if hi < blk.n:
            assert (blk.ci[blk.rp[hi]:blk.rp[min(blk.n, hi + 64)]] >= blk.n).any()


def test_mirror_split_spmv_phase_same_bits():
    """The driver's overlapped sequence (halo_begin, interior half, halo_end,
    boundary half) gives the bits of the plain sequence."""
    rp, ci, v, b = poisson()
    bounds = D.partition(rp.size - 1, 3, GRID[0] * GRID[1])
    out = []
    for overlap in (False, True):
        ranks = [M.CpuRank(D.RowBlock(rp, ci, v, bounds, q), b[bounds[q]:bounds[q + 1]],
                           eps_rel=1e-10, iter_max=500) for q in range(3)]
        res = D.run_pcg(ranks, D.LocalComm(), check_every=3, overlap=overlap)
        out.append((np.concatenate([r.x() for r in ranks]), res[0]["history"]))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_mirror_reference_start_and_iteration_cap():
    rp, ci, v, b = random_spd()
    x, res = run_mirror(rp, ci, v, b, 3, eps_rel=1e-14, iter_max=7, x0_mode=M.X0_ONES)
    assert all(r["iter_done"] == 7 for r in res)
    A = R.Matrix(rp, ci, v)
    xo, io = R.pcg_jacobi(A, R.jacobi(R.diag(rp, ci, v)), b, eps_rel=1e-14, iter_max=7,
                          x0_mode=R.X0_ONES, red=R.RED_TREE)
    assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, out_dir, overlap=False):
    import torch.distributed as td
    from datetime import timedelta
    td.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                          world_size=world, timeout=timedelta(seconds=60))
    try:
        rp, ci, v, b = poisson()
        bounds = D.partition(rp.size - 1, world, GRID[0] * GRID[1])
        blk = D.RowBlock(rp, ci, v, bounds, rank)
        rk = M.CpuRank(blk, b[blk.r0:blk.r1], eps_rel=1e-10, iter_max=500)
        (res,) = D.run_pcg([rk], D.TorchComm(), check_every=4, overlap=overlap)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), x=rk.x(), iters=res["iter_done"],
                 hist=res["history"], vres=res["verified_relres"])
    finally:
        td.destroy_process_group()


@pytest.mark.parametrize("world,overlap", [(2, False), (3, False), (2, True)])
def test_gloo_ranks_match_in_process_emulation(world, overlap, tmp_path):
    """The exchanges over torch.distributed (gloo, one process per rank)
    give the same bits as the in-process emulation, also with the SpMV
    phase split around the halo exchange."""
    import torch.multiprocessing as mp
    mp.start_processes(_gloo_worker, args=(world, _free_port(), str(tmp_path), overlap),
                       nprocs=world, start_method="spawn", join=True)
    parts = [np.load(tmp_path / f"rank{q}.npz") for q in range(world)]
    rp, ci, v, b = poisson()
    x_emul, res = run_mirror(rp, ci, v, b, world, align=GRID[0] * GRID[1], eps_rel=1e-10,
                             iter_max=500)
    assert all(int(p["iters"]) == res[0]["iter_done"] for p in parts)
    if world == 2:
        # two summands: gloo's sum equals the emulation's bit for bit
        assert np.array_equal(np.concatenate([p["x"] for p in parts]), x_emul)
        assert np.array_equal(parts[0]["hist"], res[0]["history"])
    else:
        assert np.abs(np.concatenate([p["x"] for p in parts]) - x_emul).max() <= 1e-12


def _gloo_fail_worker(rank, world, port, out_dir):
    import torch.distributed as td
    from datetime import timedelta
    td.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                          world_size=world, timeout=timedelta(seconds=60))
    try:
        rp, ci, v, b = poisson()
        bounds = D.partition(rp.size - 1, world, GRID[0] * GRID[1])
        blk = D.RowBlock(rp, ci, v, bounds, rank)
        rk = M.CpuRank(blk, b[blk.r0:blk.r1], eps_rel=1e-10, iter_max=500,
                       fail_at=6 if rank == world - 1 else None)
        (res,) = D.run_pcg([rk], D.TorchComm(), check_every=4)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), iters=res["iter_done"], err=res["err"])
    finally:
        td.destroy_process_group()


def test_gloo_one_rank_fails_all_stop_together(tmp_path):
    """A failure on one rank travels with the reduced sums: every rank stops
    at the same iteration with the timeout status, and no rank is left
    waiting in a collective."""
    import torch.multiprocessing as mp
    world = 3
    mp.start_processes(_gloo_fail_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    parts = [np.load(tmp_path / f"rank{q}.npz") for q in range(world)]
    assert {int(p["iters"]) for p in parts} == {5}
    assert all(int(p["err"]) == 5 for p in parts)
