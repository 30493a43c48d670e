"""CPU mirror of one rank of the distributed Jacobi-PCG (test infrastructure).

Implements the phase interface of cel_v3_b200.dist.GpuRank with numpy and
the oracle: local sweeps in the GPU's operation order (row sums in stored
order from 0.0, dot products in the fixed tile-tree order over the local
rows), the exchange buffer as a torch CPU tensor so that the same exchange
code (cel_v3_b200.dist.TorchComm over gloo, or LocalComm) moves it.  The
recurrence is cel_cgalg_jacobi (src/fcgalg/cel_cgalg_module.f90:205-304)
with its global scalars taken from the reduced buffer.
"""
import numpy as np
import torch

from oracle import celref as R

X0_ZERO, X0_ONES, X0_USER = "zero", "ones", "user"


def tdot(a, b):
    return R.dot(np.ascontiguousarray(a), np.ascontiguousarray(b), red=R.RED_TREE)


class CpuRank:
    def __init__(self, block, b, x0=None, eps_rel=1e-8, eps_abs=0.0, iter_max=1000, x0_mode=None,
                 fail_at=None):
        self.block = block
        n = block.n
        self.b = np.ascontiguousarray(b, dtype=np.float64)
        self.J = R.jacobi(R.diag(block.rp, block.ci, block.v))
        self.x_ext = torch.zeros(block.ncols, dtype=torch.float64)
        self.p_ext = torch.zeros(block.ncols, dtype=torch.float64)
        self.xch = torch.zeros(5, dtype=torch.float64)
        self.x0 = x0
        self.x0_mode = x0_mode or (X0_USER if x0 is not None else X0_ZERO)
        self.eps_rel, self.eps_abs, self.iter_max = eps_rel, eps_abs, iter_max
        self.r = np.zeros(n)
        self.v = np.zeros(n)
        self.err = 0
        self.active = 0
        # a local failure (as a bounded-wait timeout on this rank's device)
        # raised during the SpMV of iteration `fail_at`
        self.fail_at = fail_at

    # numpy views sharing the torch tensors' memory
    def _xe(self):
        return self.x_ext.numpy()

    def _pe(self):
        return self.p_ext.numpy()

    def _spmv(self, vec):
        return R.spmv_csr(self.block.rp, self.block.ci, self.block.v, np.ascontiguousarray(vec))

    def _store(self, s0=0.0, s1=0.0, s2=0.0, s3=0.0):
        self.xch[:] = torch.tensor([s0, s1, s2, s3, 1.0 if self.err else 0.0], dtype=torch.float64)

    def _go(self):
        return int(self.err == 0 and self.iter < self.iter_max and abs(self.alpha) > R.REAL_SMALL
                   and self.norm > self.eps)

    def begin(self):
        n = self.block.n
        xe = self._xe()
        if self.x0_mode == X0_ZERO:
            xe[:n] = 0.0
        elif self.x0_mode == X0_ONES:
            xe[:n] = 1.0
        else:
            xe[:n] = self.x0
        self.err, self.iter, self.active, self.alpha, self.norm = 0, 0, 1, 0.0, 0.0
        self.sigma = 0.0
        self._store(tdot(self.b, self.b))

    def init(self):
        n = self.block.n
        self.bnorm = float(np.sqrt(float(self.xch[0])))
        e = self.eps_abs
        if self.eps_rel > 0.0 and self.eps_rel * self.bnorm > e:
            e = self.eps_rel * self.bnorm
        self.eps = e
        s = self._spmv(self._xe())
        self.r = self.b - (0.0 + s)
        z = self.r * self.J
        self._pe()[:n] = z
        self._store(0.0, tdot(self.r, z), tdot(self.r, self.r))

    def start(self):
        self.alpha = float(self.xch[1])
        self.norm = float(np.sqrt(float(self.xch[2])))
        self.iter = 0
        self.hist = [self.norm]
        self.active = self._go()

    def ap(self):
        if not self.active:
            return
        n = self.block.n
        if self.fail_at is not None and self.iter + 1 == self.fail_at:
            self.err = 5
        self.v = 0.0 + self._spmv(self._pe())
        self._store(0.0, 0.0, 0.0, tdot(self.v, self._pe()[:n]))

    # the split SpMV phase: every row in the second half (same sums)
    def ap_interior(self):
        pass

    def ap_boundary(self):
        self.ap()

    def update(self):
        if not self.active:
            return
        n = self.block.n
        sg = self.alpha / float(self.xch[3])
        rz = rr = 0.0
        flagged = float(self.xch[4]) != 0.0
        self.sigma = sg
        if np.isfinite(sg) and not flagged:
            self.r = self.r + (-sg) * self.v
            z = self.r * self.J
            rz, rr = tdot(self.r, z), tdot(self.r, self.r)
        else:
            if self.err == 0:
                self.err = 5 if flagged else 3
            self.active = 0
        self._store(0.0, rz, rr)

    def direction(self):
        if not self.active:
            return
        n = self.block.n
        bt = float(self.xch[1]) / self.alpha
        xe, pe = self._xe(), self._pe()
        xe[:n] = xe[:n] + self.sigma * pe[:n]  # the update's step, old p
        pe[:n] = bt * pe[:n] + self.r * self.J
        self.alpha = float(self.xch[1])
        self.norm = float(np.sqrt(float(self.xch[2])))
        self.iter += 1
        self.hist.append(self.norm)
        self.active = self._go()

    def poll(self):
        return self.active

    def verify(self):
        s = self._spmv(self._xe())
        r = self.b - (0.0 + s)
        self._store(tdot(r, r))

    def result(self):
        vres = float(np.sqrt(float(self.xch[0])))
        return dict(iter_done=self.iter, final_norm2=self.norm, bnorm=self.bnorm,
                    verified_relres=vres / self.bnorm if self.bnorm > 0 else vres,
                    history=np.array(self.hist), err=self.err)

    def x(self):
        return self._xe()[:self.block.n].copy()
