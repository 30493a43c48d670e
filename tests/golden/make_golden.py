"""Generates the known-answer fixtures of tests/golden/ from the reference's
own C Poisson generator (src/base/*.c of hpcdkhab/cel_v3, compiled in place
by oracle/ref.mk into oracle/_ref/ref_poisson).

For each grid the generator discretises -Laplace(u) = -6 on [0,1]^3 with the
7-point stencil (scaled by 1/h^2), Dirichlet data u = x^2+y^2+z^2 on the
boundary rows (identity rows, eliminated couplings kept as explicit zeros),
and returns the exact nodal solution u.  The stencil is exact for
quadratics, so A u = b holds to rounding and a converged solve returns u.
The fixture stores the COO output converted to 0-based CSR (rows in
generation order, columns ascending as the generator's bubble sort leaves
them), b and u.

Usage: python tests/golden/make_golden.py [/path/to/cel_v3]
Non-cubic grids are used because the reference's Fortran driver switches to
a 27-point stencil when nx = ny = nz (src/fspmt/cel_sp_mat_generate_module.f90:73-77).
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
GRIDS = [(6, 5, 4), (12, 11, 10)]


def read_ref(path):
    raw = open(path, "rb").read()
    n, nnz = np.frombuffer(raw[:8], dtype=np.int32)
    off = 8
    rows = np.frombuffer(raw, np.int32, nnz, off); off += 4 * nnz
    cols = np.frombuffer(raw, np.int32, nnz, off); off += 4 * nnz
    vals = np.frombuffer(raw, np.float64, nnz, off); off += 8 * nnz
    b = np.frombuffer(raw, np.float64, n, off); off += 8 * n
    u = np.frombuffer(raw, np.float64, n, off); off += 8 * n
    assert off == len(raw)
    return int(n), rows, cols, vals, b, u


def coo_to_csr(n, rows, cols, vals):
    assert np.all(np.diff(rows) >= 0), "generator emits rows in order"
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp).astype(np.int32), cols.astype(np.int32), vals.astype(np.float64)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CEL_REFERENCE_DIR")
    if not ref:
        raise SystemExit("usage: make_golden.py REFERENCE_TREE (or set CEL_REFERENCE_DIR): "
                         "the root of a hpcdkhab/cel_v3 checkout")
    subprocess.check_call(["make", "-s", "-f", os.path.join(REPO, "oracle", "ref.mk"), f"REF={ref}"])
    exe = os.path.join(REPO, "oracle", "_ref", "ref_poisson")
    for nx, ny, nz in GRIDS:
        tmp = os.path.join(REPO, "oracle", "_ref", f"poisson_{nx}x{ny}x{nz}.bin")
        subprocess.check_call([exe, str(nx), str(ny), str(nz), tmp])
        n, rows, cols, vals, b, u = read_ref(tmp)
        rp, ci, v = coo_to_csr(n, rows, cols, vals)
        out = os.path.join(HERE, f"ref_poisson7_{nx}x{ny}x{nz}.npz")
        np.savez_compressed(out, rp=rp, ci=ci, v=v, b=b, u=u, grid=np.array([nx, ny, nz]))
        print(out, n, len(vals))


if __name__ == "__main__":
    main()
