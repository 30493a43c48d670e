"""Shared test inputs."""
import numpy as np


def random_csr(n, rng, max_len=9, empty_frac=0.1, long_rows=0, long_len=3000):
    """Random square CSR (0-based, columns ascending) with uneven rows, some
    empty rows and optionally a few very long rows."""
    lens = rng.integers(0, max_len + 1, n) if n else np.zeros(0, np.int64)
    lens = np.minimum(lens, n)
    if n:
        lens[rng.random(n) < empty_frac] = 0
        for r in rng.choice(n, size=min(long_rows, n), replace=False):
            lens[r] = min(long_len, n)
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    parts = [np.sort(rng.choice(n, size=int(l), replace=False)) for l in lens if l]
    ci = np.concatenate(parts).astype(np.int32) if parts else np.zeros(0, np.int32)
    v = rng.standard_normal(int(rp[-1]))
    return rp.astype(np.int32), ci, v


def spd_from_pattern(rp, ci, v):
    """Make a diagonally dominant symmetric matrix with the given pattern
    symmetrised (for solver tests)."""
    import scipy.sparse as sp
    n = rp.size - 1
    A = sp.csr_matrix((np.abs(v), ci, rp), shape=(n, n))
    A = A + A.T
    d = np.asarray(abs(A).sum(axis=1)).ravel() + 1.0
    A = (A * -0.5 + sp.diags(d)).tocsr()
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)


def ir_step_tolerance(rn, tol, tau):
    """Inner tolerance of an FP32-refinement step (ir_step_tolerance in
    cel_v3_b200/csrc/celg_device.cuh): the goal g = tol / (2 rn) if one
    inner solve at tau reaches it, sqrt(g) if two do, else tau."""
    import math
    if not (tol > 0 and rn > tol and 0 < tau < 1 and rn < 1e308):
        return tau
    g = tol / (2.0 * rn)
    if tau <= g:
        return g
    if tau * tau <= g:
        return max(math.sqrt(g), tau)
    return tau
