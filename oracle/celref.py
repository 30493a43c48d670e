"""ctypes binding of the CPU oracle (oracle/libcelref.so).

TEST INFRASTRUCTURE ONLY.  The oracle is a C restatement of the Fortran
reference's solver hot path (see celref.h); the test-suite, the smoke check
and the CPU-baseline leg of bench.py use it as the checker.  The product
library (libcelgpu.so) never loads it.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcelref.so")

RED_SEQ = 0
RED_TREE = 1
FMT_CSR = 0
FMT_JAD = 1
X0_ONES = 0
X0_ZERO = 1
X0_USER = 2
OK = 0
ERR_ARG = 1
ERR_BREAKDOWN = 3
ERR_NOCONV = 4
REAL_SMALL = 1.1 * np.finfo(np.float64).eps


class Mat(ctypes.Structure):
    _fields_ = [
        ("fmt", ctypes.c_int), ("n", ctypes.c_int), ("nnz", ctypes.c_int),
        ("rp", ctypes.c_void_p), ("ci", ctypes.c_void_p), ("v", ctypes.c_void_p),
        ("mmax", ctypes.c_int), ("jbegin", ctypes.c_void_p), ("jci", ctypes.c_void_p),
        ("jv", ctypes.c_void_p), ("perm", ctypes.c_void_p),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("x0_mode", ctypes.c_int), ("eps_abs", ctypes.c_double), ("eps_rel", ctypes.c_double),
        ("iter_max", ctypes.c_int), ("red", ctypes.c_int), ("nworkers", ctypes.c_int),
        ("literal", ctypes.c_int), ("restart", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("iter_done", ctypes.c_int), ("final_norm", ctypes.c_double), ("bnorm", ctypes.c_double),
        ("eps_used", ctypes.c_double), ("err", ctypes.c_int), ("arnoldi_steps", ctypes.c_int),
    ]


_lib = None


def lib():
    """Load (building on first use if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE])
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.celref_dot.restype = ctypes.c_double
        _lib.celref_dot_f32.restype = ctypes.c_double
        _lib.celref_reduce256.restype = ctypes.c_double
        _lib.celref_dot_tree_perm.restype = ctypes.c_double
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def work_chunk(length, nworkers, worker):
    s, e = ctypes.c_int(), ctypes.c_int()
    lib().celref_work_chunk(int(length), int(nworkers), int(worker), ctypes.byref(s), ctypes.byref(e))
    return s.value, e.value


def spmv_csr(rp, ci, v, x, y=None, accumulate=False, nworkers=1):
    rp, ci, v, x = _i32(rp), _i32(ci), _f64(v), _f64(x)
    n = rp.size - 1
    y = np.zeros(n) if y is None else _f64(y).copy()
    lib().celref_spmv_csr(n, _p(rp), _p(ci), _p(v), _p(x), _p(y), int(accumulate), int(nworkers))
    return y


def spmv_csr_f32(rp, ci, v, x, y=None, accumulate=False):
    rp, ci, v, x = _i32(rp), _i32(ci), _f32(v), _f32(x)
    n = rp.size - 1
    y = np.zeros(n, np.float32) if y is None else _f32(y).copy()
    lib().celref_spmv_csr_f32(n, _p(rp), _p(ci), _p(v), _p(x), _p(y), int(accumulate))
    return y


def jad_perm(rp):
    rp = _i32(rp)
    n = rp.size - 1
    perm = np.zeros(max(n, 1), np.int32)
    mmax = ctypes.c_int()
    lib().celref_jad_perm(n, _p(rp), _p(perm), ctypes.byref(mmax))
    return perm[:n], mmax.value


def jad_build(rp, ci, v):
    rp, ci, v = _i32(rp), _i32(ci), _f64(v)
    n = rp.size - 1
    nnz = int(rp[-1])
    _, mmax = jad_perm(rp)
    perm = np.zeros(max(n, 1), np.int32)
    jb = np.zeros(mmax + 1, np.int32)
    jci = np.zeros(max(nnz, 1), np.int32)
    jv = np.zeros(max(nnz, 1), np.float64)
    mm = ctypes.c_int()
    lib().celref_jad_build(n, _p(rp), _p(ci), _p(v), _p(perm), _p(jb), _p(jci), _p(jv), ctypes.byref(mm))
    return dict(perm=perm[:n], jbegin=jb, jci=jci[:nnz], jv=jv[:nnz], mmax=mm.value)


def jad_begin_literal(rp):
    rp = _i32(rp)
    n = rp.size - 1
    lens = np.diff(rp)
    span = int(lens.max() - min(lens.min(), n) + 1) if n else 1
    out = np.zeros(max(span, 1), np.int32)
    lo, hi = ctypes.c_int(), ctypes.c_int()
    lib().celref_jad_begin_literal(n, _p(rp), _p(out), ctypes.byref(lo), ctypes.byref(hi))
    return out[: hi.value - lo.value + 1], lo.value, hi.value


def spmv_jad(jad, x, n):
    x = _f64(x)
    y = np.zeros(n)
    lib().celref_spmv_jad(n, jad["mmax"], _p(jad["jbegin"]), _p(jad["jci"]), _p(jad["jv"]),
                          _p(jad["perm"]), _p(x), _p(y))
    return y


def diag(rp, ci, v):
    rp, ci, v = _i32(rp), _i32(ci), _f64(v)
    n = rp.size - 1
    d = np.zeros(n)
    lib().celref_diag(n, _p(rp), _p(ci), _p(v), _p(d))
    return d


def jacobi(d, s=None):
    d = _f64(d)
    J = np.zeros_like(d)
    lib().celref_jacobi(d.size, _p(d), _p(_f64(s)) if s is not None else None, _p(J))
    return J


def block_jacobi_inv(rp, ci, v, bs):
    """n x bs inverse diagonal blocks (celref_block_jacobi_inv); returns
    (inv, ok)."""
    rp, ci, v = _i32(rp), _i32(ci), _f64(v)
    n = rp.size - 1
    inv = np.zeros((n, bs))
    bad = lib().celref_block_jacobi_inv(n, _p(rp), _p(ci), _p(v), int(bs), _p(inv))
    return inv, bad == 0


def block_jacobi_apply(inv, r):
    inv, r = _f64(inv), _f64(r)
    n, bs = inv.shape
    z = np.zeros(n)
    lib().celref_block_jacobi_apply(n, bs, _p(inv), _p(r), _p(z))
    return z


def row_scale(rp, v, d):
    rp, d = _i32(rp), _f64(d)
    v = _f64(v).copy()
    s = np.zeros(d.size)
    lib().celref_row_scale(d.size, _p(rp), _p(v), _p(d), _p(s))
    return v, s


def dot(a, b, red=RED_SEQ, nworkers=1):
    a, b = _f64(a), _f64(b)
    return lib().celref_dot(a.size, _p(a), _p(b), int(red), int(nworkers))


def dot_f32(a, b, red=RED_TREE):
    a, b = _f32(a), _f32(b)
    return lib().celref_dot_f32(a.size, _p(a), _p(b), int(red))


def reduce256(vals):
    vals = _f64(vals)
    return lib().celref_reduce256(_p(vals), ctypes.c_long(vals.size))


class Matrix:
    """CSR matrix (0-based) with an optional JAD copy, kept alive for ctypes."""

    def __init__(self, rp, ci, v, fmt=FMT_CSR):
        self.rp, self.ci, self.v = _i32(rp), _i32(ci), _f64(v)
        self.n = self.rp.size - 1
        self.fmt = fmt
        self.jad = jad_build(self.rp, self.ci, self.v) if fmt == FMT_JAD else None

    def cstruct(self):
        m = Mat()
        m.fmt, m.n, m.nnz = self.fmt, self.n, int(self.rp[-1])
        m.rp, m.ci, m.v = _p(self.rp), _p(self.ci), _p(self.v)
        if self.jad is not None:
            m.mmax = self.jad["mmax"]
            m.jbegin, m.jci, m.jv, m.perm = (_p(self.jad[k]) for k in ("jbegin", "jci", "jv", "perm"))
        return m


def _params(x0_mode, eps_abs, eps_rel, iter_max, red, nworkers, literal=0, restart=0):
    return Params(int(x0_mode), float(eps_abs), float(eps_rel), int(iter_max), int(red),
                  int(nworkers), int(literal), int(restart))


def _res_dict(r, hist, nh):
    return dict(iter_done=r.iter_done, final_norm=r.final_norm, bnorm=r.bnorm,
                eps_used=r.eps_used, err=r.err, arnoldi_steps=r.arnoldi_steps,
                history=hist[:nh].copy())


def pcg_jacobi(A, J, b, x0=None, x0_mode=X0_ZERO, eps_abs=0.0, eps_rel=1e-8, iter_max=1000,
               red=RED_SEQ, nworkers=1):
    """Jacobi-PCG of the reference (cel_cgalg_jacobi); returns (x, info)."""
    b, J = _f64(b), _f64(J)
    x = np.zeros(A.n) if x0 is None else _f64(x0).copy()
    if x0 is not None:
        x0_mode = X0_USER
    hist = np.zeros(iter_max + 1)
    res = Result()
    m = A.cstruct()
    p = _params(x0_mode, eps_abs, eps_rel, iter_max, red, nworkers)
    lib().celref_pcg_jacobi(ctypes.byref(m), _p(J), _p(b), _p(x), ctypes.byref(p), _p(hist),
                            ctypes.byref(res))
    return x, _res_dict(res, hist, res.iter_done + 1)


def cg(A, b, x0_mode=X0_ONES, eps_abs=1e-7, eps_rel=0.0, iter_max=1000, red=RED_SEQ,
       literal=False):
    b = _f64(b)
    x = np.zeros(A.n)
    hist = np.zeros(iter_max + 1)
    res = Result()
    m = A.cstruct()
    p = _params(x0_mode, eps_abs, eps_rel, iter_max, red, 1, int(literal))
    lib().celref_cg(ctypes.byref(m), _p(b), _p(x), ctypes.byref(p), _p(hist), ctypes.byref(res))
    return x, _res_dict(res, hist, res.iter_done + 1)


def gmres_jacobi(A, J, b, restart=30, x0_mode=X0_ZERO, eps_abs=0.0, eps_rel=1e-8, iter_max=50,
                 red=RED_SEQ, literal=False, hist_cap=None):
    """Restarted GMRES(m) with right Jacobi (cel_gmresalg_2jacobi, Givens corrected)."""
    b, J = _f64(b), _f64(J)
    x = np.zeros(A.n)
    cap = hist_cap or ((iter_max + 1) * (restart + 1) * restart + 2)
    hist = np.zeros(cap)
    res = Result()
    m = A.cstruct()
    p = _params(x0_mode, eps_abs, eps_rel, iter_max, red, 1, int(literal), restart)
    lib().celref_gmres_jacobi(ctypes.byref(m), _p(J), _p(b), _p(x), ctypes.byref(p), _p(hist),
                              ctypes.byref(res))
    return x, _res_dict(res, hist, res.arnoldi_steps + 1)


def pcg_jacobi_f32(rp, ci, v32, J32, b32, x0_mode=X0_ZERO, eps_abs=0.0, eps_rel=1e-4,
                   iter_max=1000, red=RED_TREE):
    rp, ci, v32, J32, b32 = _i32(rp), _i32(ci), _f32(v32), _f32(J32), _f32(b32)
    n = rp.size - 1
    x = np.zeros(n, np.float32)
    hist = np.zeros(iter_max + 1)
    res = Result()
    p = _params(x0_mode, eps_abs, eps_rel, iter_max, red, 1)
    lib().celref_pcg_jacobi_f32(n, _p(rp), _p(ci), _p(v32), _p(J32), _p(b32), _p(x),
                                ctypes.byref(p), _p(hist), ctypes.byref(res))
    return x, _res_dict(res, hist, res.iter_done + 1)
