"""Seeded synthetic inputs for the solver workloads (numpy, host side).

The reference benchmarks on matrices from its own generator; the workloads
used here are defined by their shapes and seeds instead:

  poisson7(nx, ny, nz)            interior 7-point Poisson, diagonal 6,
                                  off-diagonal -1 for in-domain neighbours
                                  (Dirichlet boundary eliminated)
  diffusion7(nx, ny, nz, kx, ky, kz)
                                  -div(k grad u) with one coefficient per cell
                                  face: A_ii = sum of the cell's six faces
                                  (boundary faces included), A_ij = -k_f
  simple_test(n, block)           the block matrix of the reference's
                                  cel_sp_mat_generate_simple_test
                                  (src/fspmt/cel_sp_mat_generate_module.f90:157-215)
                                  with A * 1 = b known

Row order is lexicographic with x fastest (row = x + nx*(y + ny*z), as in
src/base/cel_domain_3d.c:62-92 for one block); columns ascend inside a row.
Face coefficients use k_f as given (no averaging); the layout of a face
array is (nz, ny, nx+1) for x-faces, (nz, ny+1, nx) for y-faces and
(nz+1, ny, nx) for z-faces, x fastest; faces 0 and n of each direction are
the Dirichlet boundary faces.
"""
import numpy as np


def face_counts(nx, ny, nz):
    return nz * ny * (nx + 1), nz * (ny + 1) * nx, (nz + 1) * ny * nx


def _stencil7(nx, ny, nz, coef=None):
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    nxy = nx * ny
    ones = np.ones(n, dtype=bool)
    present = [z > 0, y > 0, x > 0, ones, x < nx - 1, y < ny - 1, z < nz - 1]
    offsets = [-nxy, -nx, -1, 0, 1, nx, nxy]
    counts = np.zeros(n, dtype=np.int64)
    for m in present:
        counts += m
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    nnz = int(rp[-1])
    if nnz >= 2**31:
        raise ValueError("nnz does not fit int32 indices")
    ci = np.empty(nnz, dtype=np.int32)
    v = np.empty(nnz, dtype=np.float64)
    pos = rp[:-1].copy()
    if coef is not None:
        kx, ky, kz = coef
        kx = kx.reshape(nz, ny, nx + 1)
        ky = ky.reshape(nz, ny + 1, nx)
        kz = kz.reshape(nz + 1, ny, nx)
        west = kx[:, :, :-1].reshape(-1)
        east = kx[:, :, 1:].reshape(-1)
        south = ky[:, :-1, :].reshape(-1)
        north = ky[:, 1:, :].reshape(-1)
        bottom = kz[:-1, :, :].reshape(-1)
        top = kz[1:, :, :].reshape(-1)
        diag = ((((west + east) + south) + north) + bottom) + top
        vals = [-bottom, -south, -west, diag, -east, -north, -top]
    else:
        vals = [-1.0, -1.0, -1.0, 6.0, -1.0, -1.0, -1.0]
    for m, off, val in zip(present, offsets, vals):
        if m is ones:
            p = pos
            ci[p] = (idx + off).astype(np.int32)
            v[p] = val
            pos += 1
        else:
            rows = idx[m]
            p = pos[m]
            ci[p] = (rows + off).astype(np.int32)
            v[p] = val[m] if isinstance(val, np.ndarray) else val
            pos[m] += 1
    return rp.astype(np.int32), ci, v


def poisson7(nx, ny=None, nz=None):
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    return _stencil7(nx, ny, nz)


def diffusion7(nx, ny, nz, kx, ky, kz):
    return _stencil7(nx, ny, nz, (np.asarray(kx, np.float64), np.asarray(ky, np.float64),
                                  np.asarray(kz, np.float64)))


def lognormal_faces(rng, nx, ny, nz, sigma=1.0):
    """k = exp(g), g ~ N(0, sigma^2) i.i.d. per face, drawn in one call and split
    as x-faces, y-faces, z-faces."""
    cx, cy, cz = face_counts(nx, ny, nz)
    g = rng.normal(0.0, sigma, cx + cy + cz) if sigma != 1.0 else rng.standard_normal(cx + cy + cz)
    k = np.exp(g)
    return g, (k[:cx], k[cx:cx + cy], k[cx + cy:])


def simple_test(num_rows, block_size):
    """Block-diagonal matrix of cel_sp_mat_generate_simple_test for one rank
    (master 0 of 1, mult_factor 1): block ii (1-based) is dense with every
    entry equal to ii; b = ii*block_size on its rows; x_th = 1."""
    if num_rows % block_size:
        raise ValueError("num_rows must be a multiple of block_size")
    nb = num_rows // block_size
    rp = np.arange(num_rows + 1, dtype=np.int64) * block_size
    blk = np.arange(num_rows) // block_size
    ci = (blk[:, None] * block_size + np.arange(block_size)[None, :]).reshape(-1)
    v = np.repeat((blk + 1).astype(np.float64), block_size)
    b = ((blk + 1) * block_size).astype(np.float64)
    assert nb * block_size == num_rows
    return rp.astype(np.int32), ci.astype(np.int32), v, b, np.ones(num_rows)


# ---- the five workloads ------------------------------------------------------

def plain(side, seed):
    """Poisson side^3, x_true ~ U[0,1) from default_rng(seed); b = A x_true is
    left to the caller (computed with the library's or the oracle's SpMV)."""
    rp, ci, v = poisson7(side)
    x_true = np.random.default_rng(seed).random(side ** 3)
    return rp, ci, v, x_true


def precision_problem(side=256):
    """-div(k grad u), k = exp(g), g ~ N(0,1) per face (seed 2); b ~ U[-1,1) (seed 3)."""
    g, (kx, ky, kz) = lognormal_faces(np.random.default_rng(2), side, side, side)
    rp, ci, v = diffusion7(side, side, side, kx, ky, kz)
    b = np.random.default_rng(3).uniform(-1.0, 1.0, side ** 3)
    return rp, ci, v, b


def batch_problems(count=64, lo=16, hi=96, seed=4, sigma=0.5):
    """`count` systems: all sides drawn first (integers in [lo, hi]), then for
    each system its face coefficients k = exp(N(0, sigma^2)) and b ~ U[-1,1),
    all from one default_rng(seed)."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=count)
    out = []
    for s in sides:
        s = int(s)
        _, (kx, ky, kz) = lognormal_faces(rng, s, s, s, sigma)
        rp, ci, v = diffusion7(s, s, s, kx, ky, kz)
        b = rng.uniform(-1.0, 1.0, s ** 3)
        out.append((s, rp, ci, v, b))
    return out


def multirhs_problem(side=128, k=32, seed=5):
    rp, ci, v = poisson7(side)
    B = np.random.default_rng(seed).uniform(-1.0, 1.0, (side ** 3, k))
    return rp, ci, v, B


def differentiation_problems(side=128, batch=8):
    """`batch` instances of the gradient workload on a side^3 grid: per
    instance g ~ N(0,1) per face (drawn in order from default_rng(6)), then
    b ~ U[-1,1) and x_target ~ U[0,1) (drawn in order from default_rng(7))."""
    r6, r7 = np.random.default_rng(6), np.random.default_rng(7)
    cx, cy, cz = face_counts(side, side, side)
    n = side ** 3
    out = []
    for _ in range(batch):
        g = r6.standard_normal(cx + cy + cz)
        b = r7.uniform(-1.0, 1.0, n)
        xt = r7.random(n)
        out.append((g, b, xt))
    return out


def diffusion7_device(nx, ny, nz, k, device="cuda"):
    """The diffusion7 assembly computed with torch on `device` (same entry
    order and the same additions for the diagonal, so the values equal the
    host assembly's bit for bit): k is the concatenated per-face coefficient
    vector (x-, y-, z-faces) as a float64 tensor or array.  Returns int32
    row pointers, int32 columns and float64 values on the device."""
    import torch
    k = torch.as_tensor(k, dtype=torch.float64, device=device)
    cx, cy, cz = face_counts(nx, ny, nz)
    n, nxy = nx * ny * nz, nx * ny
    idx = torch.arange(n, dtype=torch.int64, device=device)
    x, y, z = idx % nx, (idx // nx) % ny, idx // nxy
    west = (z * ny + y) * (nx + 1) + x
    south = cx + (z * (ny + 1) + y) * nx + x
    bottom = cx + cy + (z * ny + y) * nx + x
    kw, ke = k[west], k[west + 1]
    ks, kn = k[south], k[south + nx]
    kb, kt = k[bottom], k[bottom + nxy]
    diag = ((((kw + ke) + ks) + kn) + kb) + kt
    present = [z > 0, y > 0, x > 0, None, x < nx - 1, y < ny - 1, z < nz - 1]
    offsets = [-nxy, -nx, -1, 0, 1, nx, nxy]
    vals = [-kb, -ks, -kw, diag, -ke, -kn, -kt]
    counts = torch.ones(n, dtype=torch.int64, device=device)
    for m in present:
        if m is not None:
            counts += m
    rp = torch.zeros(n + 1, dtype=torch.int64, device=device)
    torch.cumsum(counts, 0, out=rp[1:])
    nnz = int(rp[-1])
    if nnz >= 2**31:
        raise ValueError("nnz does not fit int32 indices")
    ci = torch.empty(nnz, dtype=torch.int32, device=device)
    v = torch.empty(nnz, dtype=torch.float64, device=device)
    pos = rp[:-1].clone()
    for m, off, val in zip(present, offsets, vals):
        if m is None:
            ci[pos] = (idx + off).to(torch.int32)
            v[pos] = val
            pos += 1
        else:
            p = pos[m]
            ci[p] = (idx[m] + off).to(torch.int32)
            v[p] = val[m]
            pos += m
    return rp.to(torch.int32), ci, v
