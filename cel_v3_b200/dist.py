"""Row-block distribution of a CSR system over ranks and the driver of the
distributed Jacobi-PCG (celg_dist_* in include/celgpu.h).

The reference splits rows into contiguous blocks (`vtxdist`,
src/fspmtdistr/cel_sp_mat_distr_module.f90:330-339), exchanges the halo
values each SpMV needs from the neighbouring blocks
(src/fspmtdistr/cel_sp_mat_distr_vec_module.f90:265-724) and all-reduces one
scalar per dot product (src/fop/cel_fop_vec_distr_module.f90:419-832).  Here:

  * `partition(n, world, align)` cuts [0, n) into contiguous blocks whose
    boundaries are multiples of `align` (nx*ny gives z-slabs of a grid);
  * `RowBlock` holds one block's rows as local CSR: columns inside the block
    become local indices 0..n-1, the others (the halo) are numbered n, n+1,
    ... in ascending global order; every row keeps its stored entry order, so
    each row sum is the single-matrix row sum bit for bit.  It also holds the
    exchange lists: per other rank, the local rows it sends and the
    contiguous range of the halo it receives;
  * `TorchComm` runs the exchanges with torch.distributed (NCCL for CUDA
    tensors, gloo for CPU tensors) -- point-to-point halo transfers and a sum
    all-reduce of the exchange buffer -- on torch's current stream;
  * with `overlap=True`, the halo of p goes out on a side stream while the
    SpMV of the rows that read no halo value runs, and the other rows follow
    once it has arrived (cel_fop_mv_axy_distr,
    src/fop/cel_fop_mv_module.f90:28-87, has the master thread exchange the
    halo while the workers multiply the local block).  Same results either
    way;
  * `GpuRank` is one rank's device side (libcelgpu.so phases); `run_pcg`
    sequences phases and exchanges for a list of ranks held by this process
    (one rank per process in a distributed run).

Every rank issues the same exchanges in the same order; the stopping
decision is taken on the device from reduced values only, so it agrees on
every rank.
"""
import numpy as np


def partition(n, world, align=1):
    """Block boundaries b[0] = 0 <= ... <= b[world] = n; interior boundaries
    are multiples of `align`, blocks as even as the alignment allows."""
    if world < 1 or align < 1:
        raise ValueError("world and align must be positive")
    units = -(-n // align)
    bounds = [min(n, (units * r // world) * align) for r in range(world + 1)]
    bounds[-1] = n
    return bounds


class RowBlock:
    """Rows [r0, r1) of a global 0-based CSR matrix (rp, ci, v) with the
    halo columns renumbered after the local ones, and the exchange lists of
    this block against every other block of `bounds`."""

    def __init__(self, rp, ci, v, bounds, rank):
        rp = np.asarray(rp, dtype=np.int64)
        ci = np.asarray(ci, dtype=np.int64)
        self.bounds = list(bounds)
        self.rank = rank
        self.world = len(bounds) - 1
        r0, r1 = bounds[rank], bounds[rank + 1]
        self.r0, self.r1, self.n = r0, r1, r1 - r0
        lo, hi = int(rp[r0]), int(rp[r1])
        cols = ci[lo:hi]
        outside = (cols < r0) | (cols >= r1)
        self.halo = np.unique(cols[outside])            # global indices, ascending
        local = np.empty_like(cols)
        local[~outside] = cols[~outside] - r0
        local[outside] = self.n + np.searchsorted(self.halo, cols[outside])
        self.rp = (rp[r0:r1 + 1] - lo).astype(np.int32)
        self.ci = local.astype(np.int32)
        self.v = np.ascontiguousarray(np.asarray(v, dtype=np.float64)[lo:hi])
        self.ncols = self.n + self.halo.size
        ends = np.asarray(bounds[1:])
        owner = np.searchsorted(ends, self.halo, side="right")
        # halo values from rank q: one contiguous range of the halo part
        self.recv = {}
        for q in np.unique(owner):
            idx = np.flatnonzero(owner == q)
            self.recv[int(q)] = (int(idx[0]), int(idx.size))
        # rows of this block that rank q needs, as local indices (ascending,
        # the order of q's halo)
        self.send = {}
        for q in range(self.world):
            if q == rank:
                continue
            qc = ci[int(rp[bounds[q]]):int(rp[bounds[q + 1]])]
            need = np.unique(qc[(qc >= r0) & (qc < r1)])
            if need.size:
                self.send[q] = (need - r0).astype(np.int64)

    def send_range(self, q):
        """(start, count) when the rows sent to q are contiguous, else None."""
        idx = self.send[q]
        if idx[-1] - idx[0] + 1 == idx.size:
            return int(idx[0]), int(idx.size)
        return None

    def neighbours(self):
        return sorted(set(self.send) | set(self.recv))

    def interior_rows(self, tile=1024):
        """[lo, hi): the longest run of `tile`-row tiles (the first of equal
        runs) whose rows read no halo column -- the rows the interior half of
        the split SpMV phase covers (celg_dist_interior_rows)."""
        rows = np.repeat(np.arange(self.n), np.diff(self.rp))
        nt = -(-self.n // tile)
        halo = np.zeros(nt, dtype=bool)
        halo[rows[self.ci >= self.n] // tile] = True
        best, t = (0, 0), 0
        while t < nt:
            if halo[t]:
                t += 1
                continue
            u = t
            while u < nt and not halo[u]:
                u += 1
            if u - t > best[1] - best[0]:
                best = (t, u)
            t = u
        return min(self.n, best[0] * tile), min(self.n, best[1] * tile)


class _SideHalo:
    """halo_begin / halo_end: the halo exchange of `halo` on a side stream
    that first waits for the work queued so far (CUDA tensors), so that
    kernels queued in between overlap it; CPU tensors exchange at once."""

    _side = None
    _side_busy = False

    def halo_begin(self, vecs, blocks):
        import torch
        self._side_busy = False
        if not vecs[0].is_cuda:
            self.halo(vecs, blocks)
            return
        if self._side is None:
            self._side = torch.cuda.Stream(device=vecs[0].device)
        self._side.wait_stream(torch.cuda.current_stream(vecs[0].device))
        with torch.cuda.stream(self._side):
            self.halo(vecs, blocks)
        self._side_busy = True

    def halo_end(self):
        """The current stream waits for the halo started by halo_begin."""
        import torch
        if self._side_busy:
            torch.cuda.current_stream(self._side.device).wait_stream(self._side)
            self._side_busy = False


class TorchComm(_SideHalo):
    """Exchanges over torch.distributed for the single rank of this process:
    halo transfers with isend/irecv (lower rank's send first within each
    pair, as every rank walks its neighbours in ascending order) and a sum
    all-reduce of the exchange buffer.  Tensors may be CUDA (NCCL) or CPU
    (gloo)."""

    def __init__(self, group=None):
        import torch.distributed as td
        self.td = td
        self.group = group

    def allreduce(self, bufs):
        (buf,) = bufs
        self.td.all_reduce(buf, group=self.group)

    def halo(self, vecs, blocks):
        import torch
        (vec,), (blk,) = vecs, blocks
        ops, keep = [], []
        for q in blk.neighbours():
            if q in blk.send:
                rng = blk.send_range(q)
                if rng is not None:
                    src = vec[rng[0]:rng[0] + rng[1]]
                else:
                    src = vec.index_select(0, torch.as_tensor(blk.send[q], device=vec.device))
                keep.append(src)
                ops.append(self.td.P2POp(self.td.isend, src, q, group=self.group))
            if q in blk.recv:
                off, cnt = blk.recv[q]
                ops.append(self.td.P2POp(self.td.irecv, vec[blk.n + off:blk.n + off + cnt], q,
                                         group=self.group))
        if ops:
            for w in self.td.batch_isend_irecv(ops):
                w.wait()


class LocalComm(_SideHalo):
    """All ranks in this process (one device or host): the all-reduce sums
    the ranks' buffers in rank order, the halo copies between the ranks'
    vectors.  Used to run several ranks' kernels on one GPU in turn."""

    def allreduce(self, bufs):
        tot = bufs[0].clone()
        for b in bufs[1:]:
            tot += b
        for b in bufs:
            b.copy_(tot)

    def halo(self, vecs, blocks):
        import torch
        for r, blk in enumerate(blocks):
            for q, (off, cnt) in sorted(blk.recv.items()):
                src = blocks[q].send[r]
                vecs[r][blk.n + off:blk.n + off + cnt] = vecs[q].index_select(
                    0, torch.as_tensor(src, device=vecs[q].device))


class GpuRank:
    """One rank's device side: its row block as a libcelgpu matrix with
    halo columns, the celg_dist state and the vectors (torch CUDA tensors)."""

    def __init__(self, handle, block, b, x0=None, eps_rel=1e-8, eps_abs=0.0, iter_max=1000,
                 x0_mode=None, history=False):
        import torch
        from . import celgpu
        self.celgpu = celgpu
        self.block = block
        self.h = handle
        dev = torch.device("cuda", torch.cuda.current_device())
        f64 = dict(dtype=torch.float64, device=dev)
        self.mat = handle.matrix_from_csr_ext(block.rp, block.ci, block.v, block.ncols).jacobi()
        self.b = torch.as_tensor(np.ascontiguousarray(b), **f64)
        self.x_ext = torch.zeros(block.ncols, **f64)
        if x0 is not None:
            self.x_ext[:block.n] = torch.as_tensor(np.ascontiguousarray(x0), **f64)
        self.p_ext = torch.zeros(block.ncols, **f64)
        self.r = torch.zeros(block.n, **f64)
        self.v = torch.zeros(block.n, **f64)
        self.state = torch.zeros(celgpu.DIST_STATE_BYTES // 8, **f64)
        self.xch = self.state[:celgpu.DIST_NEXCH]
        self.hist = torch.zeros(iter_max + 1, **f64) if history else None
        if x0_mode is None:
            x0_mode = celgpu.X0_USER if x0 is not None else celgpu.X0_ZERO
        p = celgpu.params(x0_mode=x0_mode, eps_rel=eps_rel, eps_abs=eps_abs, iter_max=iter_max)
        self.d = celgpu.Dist(handle, self.mat, p, self.state.data_ptr(),
                             self.hist.data_ptr() if history else 0, iter_max + 1 if history else 0)

    def begin(self):
        self.d.begin(self.b.data_ptr(), self.x_ext.data_ptr())

    def init(self):
        self.d.init(self.b.data_ptr(), self.x_ext.data_ptr(), self.r.data_ptr(), self.p_ext.data_ptr())

    def start(self):
        self.d.start()

    def ap(self):
        self.d.ap(self.p_ext.data_ptr(), self.v.data_ptr())

    def ap_interior(self):
        self.d.ap_interior(self.p_ext.data_ptr(), self.v.data_ptr())

    def ap_boundary(self):
        self.d.ap_boundary(self.p_ext.data_ptr(), self.v.data_ptr())

    def interior_rows(self):
        return self.d.interior_rows()

    def update(self):
        self.d.update(self.r.data_ptr(), self.v.data_ptr())

    def direction(self):
        self.d.direction(self.x_ext.data_ptr(), self.r.data_ptr(), self.p_ext.data_ptr())

    def poll(self):
        return self.d.poll()[0]

    def verify(self):
        self.d.verify(self.b.data_ptr(), self.x_ext.data_ptr())

    def result(self):
        return self.d.result(history=self.hist is not None)

    def x(self):
        return self.x_ext[:self.block.n]

    def exchange_plan(self):
        """The block's exchange lists as celg_dist_set_exchange takes them:
        neighbours in ascending order, the local rows each one reads and the
        halo range it provides."""
        blk = self.block
        peers = blk.neighbours()
        return (peers, [blk.send.get(q, np.zeros(0, np.int64)) for q in peers],
                [blk.recv.get(q, (0, 0)) for q in peers])

    def solve(self, allreduce_sum, halo, poll_every=8):
        """The whole solve in one library call (celg_dist_pcg_solve), the
        exchanges done by the callables allreduce_sum(buf_d, count, stream)
        and halo(vec_ext_d, stream)."""
        return self.d.solve(allreduce_sum, halo, self.b.data_ptr(), self.x_ext.data_ptr(),
                            poll_every, history=self.hist is not None)

    def solve_nccl(self, nccl_comm, poll_every=8, overlap=False):
        """The whole solve in one library call over NCCL
        (celg_dist_pcg_solve_nccl) with this block's exchange plan."""
        self.d.set_exchange(*self.exchange_plan())
        return self.d.solve_nccl(nccl_comm, self.b.data_ptr(), self.x_ext.data_ptr(), poll_every,
                                 overlap, history=self.hist is not None)

    def close(self):
        self.d.destroy()
        self.mat.destroy()


def nccl_communicator(rank, world, device):
    """The library's own NCCL communicator over the ranks of the default
    torch.distributed group: rank 0 makes the unique id, a broadcast on the
    group carries it to the others (celg_nccl_unique_id,
    celg_nccl_comm_create).  Release it with celgpu.nccl_comm_destroy."""
    import torch
    import torch.distributed as td
    from . import celgpu
    uid = celgpu.nccl_unique_id() if rank == 0 else bytes(celgpu.NCCL_ID_BYTES)
    if world > 1:
        t = torch.tensor(list(uid), dtype=torch.uint8, device=torch.device("cuda", device))
        td.broadcast(t, 0)
        uid = bytes(t.cpu().tolist())
    return celgpu.nccl_comm_create(uid, world, rank, device)


def iterate(ranks, comm, count, overlap=False):
    """`count` PCG iterations (each a no-op once the solve has stopped).
    overlap: the halo of p travels while the interior rows' SpMV runs."""
    for _ in range(count):
        if overlap:
            comm.halo_begin([r.p_ext for r in ranks], [r.block for r in ranks])
            for r in ranks:
                r.ap_interior()
            comm.halo_end()
            for r in ranks:
                r.ap_boundary()
        else:
            comm.halo([r.p_ext for r in ranks], [r.block for r in ranks])
            for r in ranks:
                r.ap()
        comm.allreduce([r.xch for r in ranks])
        for r in ranks:
            r.update()
        comm.allreduce([r.xch for r in ranks])
        for r in ranks:
            r.direction()


def run_pcg(ranks, comm, check_every=8, overlap=False):
    """Distributed Jacobi-PCG over `ranks` (this process's ranks, each with
    the phase methods of GpuRank) with `comm` for the exchanges; polls the
    stopping flag every `check_every` iterations; overlap as in iterate.
    Returns the ranks' results."""
    blocks = [r.block for r in ranks]
    for r in ranks:
        r.begin()
    comm.allreduce([r.xch for r in ranks])
    comm.halo([r.x_ext for r in ranks], blocks)
    for r in ranks:
        r.init()
    comm.allreduce([r.xch for r in ranks])
    for r in ranks:
        r.start()
    while ranks[0].poll():
        iterate(ranks, comm, check_every, overlap)
    comm.halo([r.x_ext for r in ranks], blocks)
    for r in ranks:
        r.verify()
    comm.allreduce([r.xch for r in ranks])
    return [r.result() for r in ranks]
