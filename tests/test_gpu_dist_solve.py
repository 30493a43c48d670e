"""The distributed Jacobi-PCG in one library call (celg_dist_pcg_solve and
celg_dist_pcg_solve_nccl): the phase loop and the exchanges run inside the
library, as the reference runs its halo exchange and all-reduces inside the
solver.

Several ranks share the one GPU here: each rank is a host thread with its own
handle and stream, and the exchange callbacks synchronise the rank's stream
and meet the other threads at a barrier before copying (no kernel waits for
another rank's).  The all-reduce sums the ranks' buffers in rank order, so
the results equal the CPU mirror's bit for bit.  NCCL runs at world size 1
(one GPU per call here), and a C program drives a two-rank solve through the
C ABI with pthreads."""
import os
import subprocess
import threading

import numpy as np
import pytest

from cel_v3_b200 import dist as D
from cel_v3_b200 import synth
from oracle import celref as R
from tests import dist_mirror as M

pytestmark = pytest.mark.gpu

GRID = (20, 18, 16)
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def poisson(grid=GRID, seed=12):
    rp, ci, v = synth.poisson7(*grid)
    xt = np.random.default_rng(seed).random(rp.size - 1)
    return rp, ci, v, R.spmv_csr(rp, ci, v, xt)


def run_cpu(blocks, b, **kw):
    ranks = [M.CpuRank(blk, b[blk.r0:blk.r1], **kw) for blk in blocks]
    res = D.run_pcg(ranks, D.LocalComm(), check_every=5)
    return np.concatenate([r.x() for r in ranks]), res


class _DevPtr:
    """A device vector at a raw pointer, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3}


class ThreadComm:
    """Exchanges between ranks that are threads of this process: each callback
    waits for its rank's stream, the ranks meet at a barrier, rank 0 does the
    rank-order sum (or the halo copies) for all, and they meet again."""

    def __init__(self, torch, blocks):
        self.torch = torch
        self.blocks = blocks
        self.bar = threading.Barrier(len(blocks), timeout=60)
        self.ptrs = [None] * len(blocks)

    def _meet(self, q, ptr, stream):
        self.torch.cuda.ExternalStream(stream).synchronize()
        self.ptrs[q] = ptr
        self.bar.wait()

    def allreduce(self, q, ptr, count, stream):
        self._meet(q, ptr, stream)
        if q == 0:
            bufs = [self.torch.as_tensor(_DevPtr(p, count), device="cuda") for p in self.ptrs]
            D.LocalComm().allreduce(bufs)
            self.torch.cuda.synchronize()
        self.bar.wait()

    def halo(self, q, ptr, stream):
        self._meet(q, ptr, stream)
        if q == 0:
            vecs = [self.torch.as_tensor(_DevPtr(p, blk.ncols), device="cuda")
                    for p, blk in zip(self.ptrs, self.blocks)]
            D.LocalComm().halo(vecs, self.blocks)
            self.torch.cuda.synchronize()
        self.bar.wait()


def solve_in_threads(celgpu, torch, blocks, b, poll_every=4, **kw):
    handles = [celgpu.Handle(0) for _ in blocks]
    ranks = [D.GpuRank(hq, blk, b[blk.r0:blk.r1], history=True, **kw)
             for hq, blk in zip(handles, blocks)]
    torch.cuda.synchronize()
    comm = ThreadComm(torch, blocks)
    out = [None] * len(ranks)
    errs = []

    def work(q):
        try:
            out[q] = ranks[q].solve(lambda p, c, s: comm.allreduce(q, p, c, s),
                                    lambda p, s: comm.halo(q, p, s), poll_every=poll_every)
        except BaseException as e:  # noqa: BLE001 - reported below
            errs.append(e)
            comm.bar.abort()

    threads = [threading.Thread(target=work, args=(q,)) for q in range(len(ranks))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    try:
        assert not errs, errs
        x = np.concatenate([r.x().cpu().numpy() for r in ranks])
    finally:
        for r in ranks:
            r.close()
        for hq in handles:
            hq.close()
    return x, out


@pytest.mark.parametrize("world", [2, 3])
def test_thread_ranks_one_call_solve_match_cpu_mirror(gpu, world):
    celgpu, h, torch = gpu
    rp, ci, v, b = poisson()
    blocks = [D.RowBlock(rp, ci, v, D.partition(rp.size - 1, world, GRID[0] * GRID[1]), q)
              for q in range(world)]
    x, res = solve_in_threads(celgpu, torch, blocks, b, eps_rel=1e-8, iter_max=1000)
    xc, rc = run_cpu(blocks, b, eps_rel=1e-8, iter_max=1000)
    assert all(r.status == celgpu.OK for r in res)
    assert len({r.iter_done for r in res}) == 1 and res[0].iter_done == rc[0]["iter_done"]
    assert np.array_equal(res[0].history, rc[0]["history"])
    assert np.array_equal(x, xc)
    assert res[0].verified_relres == rc[0]["verified_relres"] <= 1.5e-8


@pytest.mark.parametrize("iter_max", [9, 13])
def test_thread_ranks_unstructured_blocks_iteration_cap(gpu, iter_max):
    """Unaligned blocks of an unstructured matrix (scattered send lists) and
    an iteration cap: every rank stops at the same step with the status of
    the phase-by-phase driver (CELG_ERR_NOCONV at the cap; CELG_OK when the
    reference's absolute guard |r.z| <= 1.1 eps_mach ends the loop there),
    and the solution has the mirror's bits."""
    celgpu, h, torch = gpu
    from tests.helpers import random_csr, spd_from_pattern
    rp, ci, v = spd_from_pattern(*random_csr(5000, np.random.default_rng(8), max_len=7,
                                             empty_frac=0.0))
    b = np.random.default_rng(9).uniform(-1, 1, 5000)
    blocks = [D.RowBlock(rp, ci, v, D.partition(5000, 3), q) for q in range(3)]
    x, res = solve_in_threads(celgpu, torch, blocks, b, eps_rel=1e-30, iter_max=iter_max)
    xc, rc = run_cpu(blocks, b, eps_rel=1e-30, iter_max=iter_max)
    ranks = [D.GpuRank(h, blk, b[blk.r0:blk.r1], eps_rel=1e-30, iter_max=iter_max)
             for blk in blocks]
    res_p = D.run_pcg(ranks, D.LocalComm(), check_every=4)
    for r in ranks:
        r.close()
    assert [r.status for r in res] == [r.status for r in res_p]
    assert all(r.iter_done == iter_max == rc[0]["iter_done"] for r in res)
    assert res[0].status == (celgpu.ERR_NOCONV if iter_max == 9 else celgpu.OK)
    assert np.array_equal(x, xc)


@pytest.mark.parametrize("overlap", [False, True])
def test_nccl_world_one_one_call(gpu, overlap):
    """The library's own NCCL communicator at world size 1: same bits as the
    single-system solve."""
    celgpu, h, torch = gpu
    rp, ci, v, b = poisson()
    comm = D.nccl_communicator(0, 1, torch.cuda.current_device())
    try:
        blk = D.RowBlock(rp, ci, v, [0, rp.size - 1], 0)
        rk = D.GpuRank(h, blk, b, eps_rel=1e-8, iter_max=1000, history=True)
        res = rk.solve_nccl(comm, poll_every=8, overlap=overlap)
        x = rk.x().cpu().numpy()
        rk.close()
    finally:
        celgpu.nccl_comm_destroy(comm)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    info = h.pcg_jacobi(m, bd.data_ptr(), xd.data_ptr(), history=True, eps_rel=1e-8, iter_max=1000)
    m.destroy()
    assert res.status == celgpu.OK and res.iter_done == info.iter_done
    assert np.array_equal(res.history, info.history)
    assert np.array_equal(x, xd.cpu().numpy())


def test_c_program_drives_two_rank_solve(gpu, tmp_path):
    """tests/c/dist_two_ranks.c: two pthreads, one rank each, run
    celg_dist_pcg_solve on z-slabs of a 7-point Poisson system with C
    callbacks (stream sync, barrier, rank-order sums, halo planes through
    host memory).  Its solution equals the CPU mirror's bit for bit."""
    celgpu, h, torch = gpu
    exe = tmp_path / "dist_two_ranks"
    lib_dir = os.path.join(ROOT, "cel_v3_b200")
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
                           "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "c",
                                                                         "dist_two_ranks.c"),
                           "-o", str(exe), "-L", lib_dir, "-lcelgpu", "-Wl,-rpath," + lib_dir,
                           "-L", "/usr/local/cuda/lib64", "-lcudart",
                           "-Wl,-rpath,/usr/local/cuda/lib64", "-lpthread"])
    out = tmp_path / "x.bin"
    nx, ny, nz = 20, 18, 16
    r = subprocess.run([str(exe), str(nx), str(ny), str(nz), str(out)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    iters = int(r.stdout.split("iterations=")[1].split()[0])
    x = np.fromfile(out, dtype=np.float64)
    rp, ci, v = synth.poisson7(nx, ny, nz)
    n = rp.size - 1
    b = np.ones(n)
    blocks = [D.RowBlock(rp, ci, v, D.partition(n, 2, nx * ny), q) for q in range(2)]
    xc, rc = run_cpu(blocks, b, eps_rel=1e-8, iter_max=1000)
    assert iters == rc[0]["iter_done"]
    assert np.array_equal(x, xc)
