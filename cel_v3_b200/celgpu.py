"""ctypes binding of libcelgpu.so (include/celgpu.h).

The Python names mirror the reference's entry points so that tests read
like the reference's own drivers:

  Handle                      one GPU, one stream (cel_omp / solver context)
  Handle.matrix_from_csr      cel_sp_mat_to_csr + cel_sp_mat_distr_from_sp_mat_local
  Matrix.to_jad               cel_sp_mat_jad_from_sp_mat_local
  Matrix.jacobi               cel_sp_mat_distr_set_jacobi
  Matrix.scale_diagonal       cel_sp_mat_distr_scale
  Handle.spmv                 cel_fop_mv_axy_distr
  Handle.dot / norm2 / axpy / xpby / jacobi_apply
                              cel_fop_vec_distr_* (dot, norm2, scale, scale_1,
                              vec_mult_distr_jacobi)
  Handle.pcg_jacobi / cg / gmres_jacobi
                              cel_cgalg_jacobi / cel_cgalg / cel_gmresalg_2jacobi
  Handle.elm_*                cel_elmSolver* (Initialization ... Destroy)

Device vectors are passed as integer device pointers (e.g.
torch.Tensor.data_ptr()); host vectors as numpy arrays.  Every call raises
CelgError with the library's status code on failure; there is no CPU
fallback: if the library cannot be loaded, importing the binding fails.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcelgpu.so")

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_BREAKDOWN = 3
ERR_NOCONV = 4
ERR_TIMEOUT = 5
ERR_STATE = 6
ERR_COMM = 7

FMT_CSR = 0
FMT_JAD = 1
COLS_INT32, COLS_OFFSET8, COLS_PATTERN = 0, 1, 2
TUNE_BATCH = 0
TUNE_SPMM = 1
PRECOND_JACOBI = 0
PRECOND_BLOCK_JACOBI = 1

X0_REF_ONES = 0
X0_ZERO = 1
X0_USER = 2
PREC_FP64 = 0
PREC_FP32_IR = 1
PREC_FP32_RU = 2
SOLVER_PCG = 0
SOLVER_CG = 1
SOLVER_GMRES = 2


class CelgError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


class Params(ctypes.Structure):
    _fields_ = [
        ("x0_mode", ctypes.c_int), ("eps_abs", ctypes.c_double), ("eps_rel", ctypes.c_double),
        ("iter_max", ctypes.c_int), ("fmt", ctypes.c_int), ("precision", ctypes.c_int),
        ("literal_ref_bugs", ctypes.c_int), ("restart", ctypes.c_int),
        ("inner_eps_rel", ctypes.c_double), ("inner_iter_max", ctypes.c_int),
        ("outer_max", ctypes.c_int), ("precond", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("iter_done", ctypes.c_int), ("final_norm2", ctypes.c_double), ("bnorm", ctypes.c_double),
        ("verified_relres", ctypes.c_double), ("err", ctypes.c_int),
        ("arnoldi_steps", ctypes.c_int), ("history", ctypes.POINTER(ctypes.c_double)),
        ("history_cap", ctypes.c_int), ("history_len", ctypes.c_int),
    ]


# celg_dist_comm: the caller's exchange callbacks of celg_dist_pcg_solve
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                ctypes.c_void_p)
HALO_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


class DistComm(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("allreduce_sum", ALLREDUCE_FN), ("halo", HALO_FN)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libcelgpu.so not built ({LIB_PATH}); run `python -m cel_v3_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    sigs = {
        "celg_params_default": (None, [ctypes.POINTER(Params)]),
        "celg_create": (i, [ctypes.POINTER(vp), i, vp]),
        "celg_destroy": (i, [vp]),
        "celg_set_stream": (i, [vp, vp]),
        "celg_status_string": (ctypes.c_char_p, [i]),
        "celg_sm_count": (i, [vp, ip]),
        "celg_mat_from_csr": (i, [vp, i, i, vp, vp, vp, i, ctypes.POINTER(vp)]),
        "celg_mat_from_csr_device": (i, [vp, i, i, vp, vp, vp, ctypes.POINTER(vp)]),
        "celg_mat_destroy": (i, [vp]),
        "celg_mat_info": (i, [vp, ip, ip, ip]),
        "celg_mat_to_jad": (i, [vp, vp]),
        "celg_mat_get_jad": (i, [vp, vp, vp, vp, vp]),
        "celg_mat_jacobi": (i, [vp]),
        "celg_mat_get_jacobi": (i, [vp, vp]),
        "celg_mat_scale_diagonal": (i, [vp]),
        "celg_mat_make_fp32": (i, [vp]),
        "celg_spmv": (i, [vp, vp, i, vp, vp, i]),
        "celg_spmv_f32": (i, [vp, vp, vp, vp, i]),
        "celg_dot": (i, [vp, i, vp, vp, dp]),
        "celg_norm2": (i, [vp, i, vp, dp]),
        "celg_axpy": (i, [vp, i, d, vp, vp]),
        "celg_xpby": (i, [vp, i, vp, d, vp]),
        "celg_jacobi_apply": (i, [vp, vp, vp, vp]),
        "celg_pcg_jacobi": (i, [vp, vp, vp, vp, ctypes.POINTER(Params), ctypes.POINTER(Result)]),
        "celg_cg": (i, [vp, vp, vp, vp, ctypes.POINTER(Params), ctypes.POINTER(Result)]),
        "celg_gmres_jacobi": (i, [vp, vp, vp, vp, ctypes.POINTER(Params), ctypes.POINTER(Result)]),
        "celg_solve_host": (i, [vp, vp, i, vp, vp, ctypes.POINTER(Params), ctypes.POINTER(Result)]),
        "celg_elm_init": (i, [vp, i, i, i, vp]),
        "celg_elm_set_solver": (i, [vp, i, ctypes.POINTER(Params), i]),
        "celg_elm_row_start": (i, [vp, i]),
        "celg_elm_insert": (i, [vp, i, d]),
        "celg_elm_reinsert": (i, [vp, i, d]),
        "celg_elm_row_completed": (i, [vp]),
        "celg_elm_insert_rows": (i, [vp, i, i, vp, vp, vp]),
        "celg_elm_matrix_completed": (i, [vp]),
        "celg_elm_doit": (i, [vp, vp, ip, ip, dp]),
        "celg_elm_redoit": (i, [vp, vp, ip, ip, dp]),
        "celg_elm_collect_solution": (i, [vp, vp]),
        "celg_elm_performance": (i, [vp, dp, ip, dp]),
        "celg_elm_destroy": (i, [vp]),
        "celg_dot_noalloc": (i, [i, vp, vp, vp, vp]),
        "celg_pcg_batched": (i, [vp, i, vp, vp, vp, ctypes.POINTER(Params), vp]),
        "celg_check_bounded_wait": (i, [vp, i, ip]),
        "celg_pcg_multirhs": (i, [vp, vp, i, vp, vp, ctypes.POINTER(Params), vp]),
        "celg_pcg_adjoint": (i, [vp, vp, vp, vp, vp, vp, ctypes.POINTER(Params), ctypes.POINTER(Result)]),
        "celg_diffusion7_face_grad": (i, [vp, i, i, i, vp, vp, vp, vp, vp]),
        "celg_mat_from_csr_ext": (i, [vp, i, i, i, vp, vp, vp, i, ctypes.POINTER(vp)]),
        "celg_mat_from_coo": (i, [vp, i, i, i, vp, vp, vp, i, ctypes.POINTER(vp)]),
        "celg_mat_block_jacobi": (i, [vp, i]),
        "celg_mat_get_block_jacobi": (i, [vp, vp]),
        "celg_block_jacobi_apply": (i, [vp, vp, vp, vp]),
        "celg_mm_info": (i, [ctypes.c_char_p, i, ip, ip, ip, ip]),
        "celg_mm_read": (i, [ctypes.c_char_p, i, i, vp, vp, vp]),
        "celg_dist_create": (i, [vp, vp, ctypes.POINTER(Params), vp, vp, i, ctypes.POINTER(vp)]),
        "celg_dist_destroy": (i, [vp]),
        "celg_dist_exchange_buffer": (i, [vp, ctypes.POINTER(vp)]),
        "celg_dist_pcg_begin": (i, [vp, vp, vp]),
        "celg_dist_pcg_init": (i, [vp, vp, vp, vp, vp]),
        "celg_dist_pcg_start": (i, [vp]),
        "celg_dist_pcg_ap": (i, [vp, vp, vp]),
        "celg_dist_pcg_ap_interior": (i, [vp, vp, vp]),
        "celg_dist_pcg_ap_boundary": (i, [vp, vp, vp]),
        "celg_dist_interior_rows": (i, [vp, ip, ip]),
        "celg_dist_pcg_update": (i, [vp, vp, vp]),
        "celg_dist_pcg_direction": (i, [vp, vp, vp, vp]),
        "celg_dist_pcg_poll": (i, [vp, ip, ip]),
        "celg_dist_pcg_verify": (i, [vp, vp, vp]),
        "celg_dist_pcg_result": (i, [vp, ctypes.POINTER(Result)]),
        "celg_dist_pcg_solve": (i, [vp, ctypes.POINTER(DistComm), vp, vp, i, ctypes.POINTER(Result)]),
        "celg_dist_set_exchange": (i, [vp, i, vp, vp, vp, vp, vp]),
        "celg_nccl_unique_id": (i, [vp]),
        "celg_nccl_comm_create": (i, [vp, i, i, i, ctypes.POINTER(vp)]),
        "celg_nccl_comm_destroy": (i, [vp]),
        "celg_dist_pcg_solve_nccl": (i, [vp, vp, vp, vp, i, i, ctypes.POINTER(Result)]),
        "celg_tuned_config": (i, [vp, i, ip]),
        "celg_mat_column_form": (i, [vp, ip]),
    }
    for name, (res, args) in sigs.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    return lib


lib = _load()


def status_string(s):
    return lib.celg_status_string(int(s)).decode()


def _check(status, what, allow=()):
    if status != OK and status not in allow:
        raise CelgError(status, what)
    return status


def _host_ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def params(**kw):
    """celg_params with the library defaults, overridden by keyword."""
    p = Params()
    lib.celg_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


NOALLOC_MAX_ROWS = 67108864


def dot_noalloc(n, a_d, b_d, out_d, stream=0):
    """celg_dot_noalloc: a.b into out_d[0] without any device allocation (see
    include/celgpu.h); returns the status code."""
    return lib.celg_dot_noalloc(int(n), ctypes.c_void_p(a_d), ctypes.c_void_p(b_d),
                                ctypes.c_void_p(out_d), ctypes.c_void_p(int(stream)) if stream else None)


MM_GENERAL, MM_SYMMETRIC, MM_SKEW = 0, 1, 2


def mm_read(path, expand=False):
    """MatrixMarket file -> (nrows, ncols, symmetry, rows, cols, vals), 1-based
    entries as stored (celg_mm_info + celg_mm_read; host only)."""
    p = str(path).encode()
    nr, nc, nz, sy = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib.celg_mm_info(p, int(expand), ctypes.byref(nr), ctypes.byref(nc), ctypes.byref(nz),
                            ctypes.byref(sy)), "celg_mm_info")
    rows = np.zeros(nz.value, np.int32)
    cols = np.zeros(nz.value, np.int32)
    vals = np.zeros(nz.value, np.float64)
    _check(lib.celg_mm_read(p, int(expand), nz.value, _host_ptr(rows), _host_ptr(cols),
                            _host_ptr(vals)), "celg_mm_read")
    return nr.value, nc.value, sy.value, rows, cols, vals


DIST_NEXCH = 5
DIST_STATE_BYTES = 256


class Dist:
    """celg_dist: the phases of a distributed Jacobi-PCG on one rank's row
    block (device pointers; see include/celgpu.h for the sequence)."""

    def __init__(self, handle, mat, p, state_d=0, hist_d=0, hist_cap=0):
        self.handle = handle
        self.ptr = ctypes.c_void_p()
        _check(lib.celg_dist_create(handle.ptr, mat.ptr, ctypes.byref(p),
                                    ctypes.c_void_p(state_d) if state_d else None,
                                    ctypes.c_void_p(hist_d) if hist_d else None, int(hist_cap),
                                    ctypes.byref(self.ptr)), "celg_dist_create")
        self.iter_max = p.iter_max

    def _call(self, name, *ptrs):
        _check(getattr(lib, name)(self.ptr, *[ctypes.c_void_p(q) for q in ptrs]), name)

    def exchange_buffer(self):
        out = ctypes.c_void_p()
        _check(lib.celg_dist_exchange_buffer(self.ptr, ctypes.byref(out)), "celg_dist_exchange_buffer")
        return out.value

    def begin(self, b_d, x_ext_d):
        self._call("celg_dist_pcg_begin", b_d, x_ext_d)

    def init(self, b_d, x_ext_d, r_d, p_ext_d):
        self._call("celg_dist_pcg_init", b_d, x_ext_d, r_d, p_ext_d)

    def start(self):
        self._call("celg_dist_pcg_start")

    def ap(self, p_ext_d, v_d):
        self._call("celg_dist_pcg_ap", p_ext_d, v_d)

    def ap_interior(self, p_ext_d, v_d):
        self._call("celg_dist_pcg_ap_interior", p_ext_d, v_d)

    def ap_boundary(self, p_ext_d, v_d):
        self._call("celg_dist_pcg_ap_boundary", p_ext_d, v_d)

    def interior_rows(self):
        """[lo, hi): the rows the interior half of the split SpMV covers."""
        lo, hi = ctypes.c_int(), ctypes.c_int()
        _check(lib.celg_dist_interior_rows(self.ptr, ctypes.byref(lo), ctypes.byref(hi)),
               "celg_dist_interior_rows")
        return lo.value, hi.value

    def update(self, r_d, v_d):
        self._call("celg_dist_pcg_update", r_d, v_d)

    def direction(self, x_ext_d, r_d, p_ext_d):
        self._call("celg_dist_pcg_direction", x_ext_d, r_d, p_ext_d)

    def poll(self):
        a, it = ctypes.c_int(), ctypes.c_int()
        _check(lib.celg_dist_pcg_poll(self.ptr, ctypes.byref(a), ctypes.byref(it)), "celg_dist_pcg_poll")
        return a.value, it.value

    def verify(self, b_d, x_ext_d):
        self._call("celg_dist_pcg_verify", b_d, x_ext_d)

    def result(self, history=False):
        res = Result()
        hist = None
        if history:
            hist = np.zeros(self.iter_max + 1)
            res.history = hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            res.history_cap = hist.size
        st = lib.celg_dist_pcg_result(self.ptr, ctypes.byref(res))
        _check(st, "celg_dist_pcg_result", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return _info(res, hist, st)

    def _result_buffers(self, history):
        res = Result()
        hist = None
        if history:
            hist = np.zeros(self.iter_max + 1)
            res.history = hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            res.history_cap = hist.size
        return res, hist

    def solve(self, allreduce_sum, halo, b_d, x_ext_d, poll_every=8, history=False):
        """celg_dist_pcg_solve: the whole solve with the exchanges done by the
        Python callables allreduce_sum(buf_d, count, stream) and
        halo(vec_ext_d, stream) (device pointers as ints; return None or 0)."""
        errors = []

        def guarded(fn, *a):
            try:
                return int(fn(*a) or 0)
            except BaseException as e:  # noqa: BLE001 - re-raised after the call
                errors.append(e)
                return 1

        def ar(ctx, buf, count, stream):
            return guarded(allreduce_sum, buf, count, stream)

        def hl(ctx, vec, stream):
            return guarded(halo, vec, stream)

        comm = DistComm(None, ALLREDUCE_FN(ar), HALO_FN(hl))
        res, hist = self._result_buffers(history)
        st = lib.celg_dist_pcg_solve(self.ptr, ctypes.byref(comm), ctypes.c_void_p(b_d),
                                     ctypes.c_void_p(x_ext_d), int(poll_every), ctypes.byref(res))
        if errors:
            raise errors[0]
        _check(st, "celg_dist_pcg_solve", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return _info(res, hist, st)

    def set_exchange(self, peers, send_rows, recv):
        """celg_dist_set_exchange: peers[q] with send_rows[q] (local rows, any
        int array) and recv[q] = (halo start, count)."""
        peers = np.asarray(peers, np.int32)
        counts = np.asarray([len(r) for r in send_rows], np.int32)
        rows = (np.concatenate([np.asarray(r, np.int32) for r in send_rows])
                if len(send_rows) else np.zeros(0, np.int32)).astype(np.int32)
        starts = np.asarray([r[0] for r in recv], np.int32)
        rcount = np.asarray([r[1] for r in recv], np.int32)
        _check(lib.celg_dist_set_exchange(self.ptr, int(peers.size), _host_ptr(peers),
                                          _host_ptr(counts), _host_ptr(rows), _host_ptr(starts),
                                          _host_ptr(rcount)), "celg_dist_set_exchange")

    def solve_nccl(self, nccl_comm, b_d, x_ext_d, poll_every=8, overlap=False, history=False):
        """celg_dist_pcg_solve_nccl: the whole solve, exchanges over NCCL."""
        res, hist = self._result_buffers(history)
        st = lib.celg_dist_pcg_solve_nccl(self.ptr, ctypes.c_void_p(nccl_comm), ctypes.c_void_p(b_d),
                                          ctypes.c_void_p(x_ext_d), int(poll_every), int(overlap),
                                          ctypes.byref(res))
        _check(st, "celg_dist_pcg_solve_nccl", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return _info(res, hist, st)

    def destroy(self):
        if self.ptr:
            lib.celg_dist_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()


NCCL_ID_BYTES = 128


def nccl_unique_id():
    """celg_nccl_unique_id: 128 bytes, made on one rank, broadcast by the caller."""
    buf = (ctypes.c_ubyte * NCCL_ID_BYTES)()
    _check(lib.celg_nccl_unique_id(buf), "celg_nccl_unique_id")
    return bytes(buf)


def nccl_comm_create(uid, nranks, rank, device):
    """celg_nccl_comm_create (collective over the nranks ranks): the
    communicator as an int."""
    buf = (ctypes.c_ubyte * NCCL_ID_BYTES).from_buffer_copy(bytes(uid))
    out = ctypes.c_void_p()
    _check(lib.celg_nccl_comm_create(buf, int(nranks), int(rank), int(device), ctypes.byref(out)),
           "celg_nccl_comm_create")
    return out.value


def nccl_comm_destroy(comm):
    _check(lib.celg_nccl_comm_destroy(ctypes.c_void_p(comm)), "celg_nccl_comm_destroy")


class SolveInfo(dict):
    __getattr__ = dict.__getitem__


def _info(res, hist, status):
    out = SolveInfo(iter_done=res.iter_done, final_norm2=res.final_norm2, bnorm=res.bnorm,
                    verified_relres=res.verified_relres, err=res.err, status=status,
                    arnoldi_steps=res.arnoldi_steps)
    out["history"] = hist[: res.history_len].copy() if hist is not None else None
    return out


class Matrix:
    def __init__(self, handle, ptr):
        self.handle = handle
        self.ptr = ptr

    def info(self):
        n, nnz, mm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.celg_mat_info(self.ptr, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(mm)),
               "celg_mat_info")
        return n.value, nnz.value, mm.value

    @property
    def n(self):
        return self.info()[0]

    def column_form(self):
        """celg_mat_column_form: COLS_INT32, COLS_OFFSET8 or COLS_PATTERN."""
        f = ctypes.c_int()
        _check(lib.celg_mat_column_form(self.ptr, ctypes.byref(f)), "celg_mat_column_form")
        return f.value

    def to_jad(self):
        n = self.n
        perm = np.zeros(max(n, 1), np.int32)
        _check(lib.celg_mat_to_jad(self.ptr, _host_ptr(perm)), "celg_mat_to_jad")
        return perm[:n]

    def get_jad(self):
        n, nnz, mmax = self.info()
        perm = np.zeros(max(n, 1), np.int32)
        jb = np.zeros(mmax + 1, np.int32)
        jci = np.zeros(max(nnz, 1), np.int32)
        jv = np.zeros(max(nnz, 1), np.float64)
        _check(lib.celg_mat_get_jad(self.ptr, _host_ptr(perm), _host_ptr(jb), _host_ptr(jci),
                                    _host_ptr(jv)), "celg_mat_get_jad")
        return dict(perm=perm[:n], jbegin=jb, jci=jci[:nnz], jv=jv[:nnz], mmax=mmax)

    def jacobi(self):
        _check(lib.celg_mat_jacobi(self.ptr), "celg_mat_jacobi")
        return self

    def get_jacobi(self):
        J = np.zeros(max(self.n, 1))
        _check(lib.celg_mat_get_jacobi(self.ptr, _host_ptr(J)), "celg_mat_get_jacobi")
        return J[: self.n]

    def block_jacobi(self, block_size):
        """Inverse diagonal blocks for PCG with precond=PRECOND_BLOCK_JACOBI."""
        _check(lib.celg_mat_block_jacobi(self.ptr, int(block_size)), "celg_mat_block_jacobi")
        self.bj_bs = int(block_size)
        return self

    def get_block_jacobi(self):
        n = self.n
        inv = np.zeros((n, self.bj_bs))
        _check(lib.celg_mat_get_block_jacobi(self.ptr, _host_ptr(inv)), "celg_mat_get_block_jacobi")
        return inv

    def scale_diagonal(self):
        _check(lib.celg_mat_scale_diagonal(self.ptr), "celg_mat_scale_diagonal")
        return self

    def make_fp32(self):
        _check(lib.celg_mat_make_fp32(self.ptr), "celg_mat_make_fp32")
        return self

    def destroy(self):
        if self.ptr:
            lib.celg_mat_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


STREAM_LEGACY = 0x1  # cudaStreamLegacy: the legacy default stream


def _stream_arg(stream):
    """None -> library-owned stream; 0 (torch's default stream) -> the legacy
    default stream; anything else is a cudaStream_t handle."""
    if stream is None:
        return None
    return ctypes.c_void_p(STREAM_LEGACY if int(stream) == 0 else int(stream))


class Handle:
    """One GPU and one CUDA stream.  stream=None: the library creates its own;
    otherwise the caller's cudaStream_t (0 = the legacy default stream, e.g.
    torch.cuda.current_stream().cuda_stream on the default stream)."""

    def __init__(self, device=0, stream=None):
        h = ctypes.c_void_p()
        _check(lib.celg_create(ctypes.byref(h), int(device), _stream_arg(stream)), "celg_create")
        self.ptr = h
        self.mats = []

    def close(self):
        if self.ptr:
            for m in self.mats:
                m.destroy()
            self.mats = []
            lib.celg_destroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sm_count(self):
        s = ctypes.c_int()
        _check(lib.celg_sm_count(self.ptr, ctypes.byref(s)), "celg_sm_count")
        return s.value

    def set_stream(self, stream):
        _check(lib.celg_set_stream(self.ptr, _stream_arg(stream)), "celg_set_stream")

    # ---- matrices
    def matrix_from_csr(self, rp, ci, v, index_base=0):
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        m = ctypes.c_void_p()
        n = rp.size - 1
        _check(lib.celg_mat_from_csr(self.ptr, n, int(ci.size), _host_ptr(rp), _host_ptr(ci),
                                     _host_ptr(v), int(index_base), ctypes.byref(m)),
               "celg_mat_from_csr")
        mat = Matrix(self, m)
        self.mats.append(mat)
        return mat

    def matrix_from_coo(self, n, rows, cols, vals, index_base=0, ncols=None):
        """COO triplets -> CSR on the device (celg_mat_from_coo)."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        m = ctypes.c_void_p()
        _check(lib.celg_mat_from_coo(self.ptr, int(n), int(n if ncols is None else ncols),
                                     int(vals.size), _host_ptr(rows), _host_ptr(cols),
                                     _host_ptr(vals), int(index_base), ctypes.byref(m)),
               "celg_mat_from_coo")
        mat = Matrix(self, m)
        self.mats.append(mat)
        return mat

    def matrix_from_csr_ext(self, rp, ci, v, ncols, index_base=0):
        """A row block with halo columns n..ncols-1 (celg_mat_from_csr_ext)."""
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        m = ctypes.c_void_p()
        _check(lib.celg_mat_from_csr_ext(self.ptr, rp.size - 1, int(ncols), int(ci.size),
                                         _host_ptr(rp), _host_ptr(ci), _host_ptr(v),
                                         int(index_base), ctypes.byref(m)),
               "celg_mat_from_csr_ext")
        mat = Matrix(self, m)
        self.mats.append(mat)
        return mat

    def matrix_from_csr_device(self, n, nnz, rp_d, ci_d, v_d):
        m = ctypes.c_void_p()
        _check(lib.celg_mat_from_csr_device(self.ptr, int(n), int(nnz), ctypes.c_void_p(rp_d),
                                            ctypes.c_void_p(ci_d), ctypes.c_void_p(v_d),
                                            ctypes.byref(m)), "celg_mat_from_csr_device")
        mat = Matrix(self, m)
        self.mats.append(mat)
        return mat

    # ---- operators on device pointers
    def spmv(self, mat, x_d, y_d, fmt=FMT_CSR, accumulate=False):
        _check(lib.celg_spmv(self.ptr, mat.ptr, int(fmt), ctypes.c_void_p(x_d),
                             ctypes.c_void_p(y_d), int(accumulate)), "celg_spmv")

    def spmv_f32(self, mat, x_d, y_d, accumulate=False):
        _check(lib.celg_spmv_f32(self.ptr, mat.ptr, ctypes.c_void_p(x_d), ctypes.c_void_p(y_d),
                                 int(accumulate)), "celg_spmv_f32")

    def dot(self, n, a_d, b_d):
        out = ctypes.c_double()
        _check(lib.celg_dot(self.ptr, int(n), ctypes.c_void_p(a_d), ctypes.c_void_p(b_d),
                            ctypes.byref(out)), "celg_dot")
        return out.value

    def norm2(self, n, a_d):
        out = ctypes.c_double()
        _check(lib.celg_norm2(self.ptr, int(n), ctypes.c_void_p(a_d), ctypes.byref(out)),
               "celg_norm2")
        return out.value

    def axpy(self, n, alpha, x_d, y_d):
        _check(lib.celg_axpy(self.ptr, int(n), float(alpha), ctypes.c_void_p(x_d),
                             ctypes.c_void_p(y_d)), "celg_axpy")

    def xpby(self, n, x_d, beta, y_d):
        _check(lib.celg_xpby(self.ptr, int(n), ctypes.c_void_p(x_d), float(beta),
                             ctypes.c_void_p(y_d)), "celg_xpby")

    def block_jacobi_apply(self, mat, r_d, z_d):
        _check(lib.celg_block_jacobi_apply(self.ptr, mat.ptr, ctypes.c_void_p(r_d), ctypes.c_void_p(z_d)),
               "celg_block_jacobi_apply")

    def jacobi_apply(self, mat, r_d, z_d):
        _check(lib.celg_jacobi_apply(self.ptr, mat.ptr, ctypes.c_void_p(r_d), ctypes.c_void_p(z_d)),
               "celg_jacobi_apply")

    # ---- solvers on device pointers
    def _solve(self, fn, name, mat, b_d, x_d, p, history):
        res = Result()
        hist = None
        if history:
            cap = history if isinstance(history, int) and history > 1 else p.iter_max + 1
            hist = np.zeros(cap)
            res.history = hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            res.history_cap = cap
        st = fn(self.ptr, mat.ptr, ctypes.c_void_p(b_d), ctypes.c_void_p(x_d), ctypes.byref(p),
                ctypes.byref(res))
        _check(st, name, allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return _info(res, hist, st)

    def pcg_jacobi(self, mat, b_d, x_d, p=None, history=False, **kw):
        p = p or params(**kw)
        return self._solve(lib.celg_pcg_jacobi, "celg_pcg_jacobi", mat, b_d, x_d, p, history)

    def cg(self, mat, b_d, x_d, p=None, history=False, **kw):
        p = p or params(**kw)
        return self._solve(lib.celg_cg, "celg_cg", mat, b_d, x_d, p, history)

    def gmres_jacobi(self, mat, b_d, x_d, p=None, history=False, **kw):
        p = p or params(**kw)
        return self._solve(lib.celg_gmres_jacobi, "celg_gmres_jacobi", mat, b_d, x_d, p, history)

    def pcg_batched(self, mats, b_ptrs, x_ptrs, p=None, **kw):
        """Jacobi-PCG on many systems in one device-driven loop; returns a list
        of per-system SolveInfo."""
        p = p or params(**kw)
        k = len(mats)
        M = (ctypes.c_void_p * k)(*[m.ptr for m in mats])
        B = (ctypes.c_void_p * k)(*[ctypes.c_void_p(int(b)) for b in b_ptrs])
        X = (ctypes.c_void_p * k)(*[ctypes.c_void_p(int(x)) for x in x_ptrs])
        res = (Result * k)()
        st = lib.celg_pcg_batched(self.ptr, k, M, B, X, ctypes.byref(p), res)
        _check(st, "celg_pcg_batched", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return [_info(r, None, r.err) for r in res]

    def pcg_multirhs(self, mat, k, B_d, X_d, p=None, **kw):
        """Jacobi-PCG on k right-hand sides (n x k row-major device arrays);
        returns a list of per-column SolveInfo."""
        p = p or params(**kw)
        res = (Result * k)()
        st = lib.celg_pcg_multirhs(self.ptr, mat.ptr, int(k), ctypes.c_void_p(B_d),
                                   ctypes.c_void_p(X_d), ctypes.byref(p), res)
        _check(st, "celg_pcg_multirhs", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return [_info(r, None, r.err) for r in res]

    def pcg_adjoint(self, mat, x_d, g_d, lambda_d, grad_vals_d=None, p=None, **kw):
        """lambda = A^{-1} g (dL/db) and optionally dL/dA on the pattern."""
        p = p or params(**kw)
        res = Result()
        st = lib.celg_pcg_adjoint(self.ptr, mat.ptr, ctypes.c_void_p(x_d), ctypes.c_void_p(g_d),
                                  ctypes.c_void_p(lambda_d),
                                  ctypes.c_void_p(grad_vals_d) if grad_vals_d else None,
                                  ctypes.byref(p), ctypes.byref(res))
        _check(st, "celg_pcg_adjoint", allow=(ERR_NOCONV,))
        return _info(res, None, st)

    def tuned_config(self, what):
        """celg_tuned_config: the autotuner's pick for the last batched
        (TUNE_BATCH: (SpMV CTAs per SM, vector-sweep CTAs per SM)) or
        multi-RHS (TUNE_SPMM: (FP64 variant, FP32 shape or -1)) solve."""
        out = (ctypes.c_int * 2)()
        _check(lib.celg_tuned_config(self.ptr, int(what), out), "celg_tuned_config")
        return out[0], out[1]

    def diffusion7_face_grad(self, nx, ny, nz, lambda_d, x_d, gkx_d, gky_d, gkz_d):
        _check(lib.celg_diffusion7_face_grad(self.ptr, int(nx), int(ny), int(nz),
                                             ctypes.c_void_p(lambda_d), ctypes.c_void_p(x_d),
                                             ctypes.c_void_p(gkx_d), ctypes.c_void_p(gky_d),
                                             ctypes.c_void_p(gkz_d)), "celg_diffusion7_face_grad")

    def check_bounded_wait(self, limit_ms=200):
        """Status reported by a bounded device wait that is never satisfied."""
        s = ctypes.c_int()
        _check(lib.celg_check_bounded_wait(self.ptr, int(limit_ms), ctypes.byref(s)),
               "celg_check_bounded_wait")
        return s.value

    def solve_host(self, mat, b, x=None, solver=SOLVER_PCG, p=None, **kw):
        """Solve from host arrays (the copies are part of the call)."""
        p = p or params(**kw)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x is None else np.ascontiguousarray(x, np.float64)
        res = Result()
        st = lib.celg_solve_host(self.ptr, mat.ptr, int(solver), _host_ptr(b), _host_ptr(x),
                                 ctypes.byref(p), ctypes.byref(res))
        _check(st, "celg_solve_host", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return x, _info(res, None, st)

    # ---- ELM assembly API
    def elm_init(self, n_total, n_local=None, row_low=1, nnz_hint=(7, 0)):
        hint = (ctypes.c_int * 2)(*nnz_hint)
        _check(lib.celg_elm_init(self.ptr, int(n_total), int(n_local if n_local is not None else n_total),
                                 int(row_low), hint), "celg_elm_init")

    def elm_set_solver(self, solver, p=None, diag_scaling=True, **kw):
        p = p or params(**kw)
        _check(lib.celg_elm_set_solver(self.ptr, int(solver), ctypes.byref(p), int(diag_scaling)),
               "celg_elm_set_solver")

    def elm_row_start(self, row):
        _check(lib.celg_elm_row_start(self.ptr, int(row)), "celg_elm_row_start")

    def elm_insert(self, col, value):
        _check(lib.celg_elm_insert(self.ptr, int(col), float(value)), "celg_elm_insert")

    def elm_reinsert(self, col, value):
        _check(lib.celg_elm_reinsert(self.ptr, int(col), float(value)), "celg_elm_reinsert")

    def elm_row_completed(self):
        _check(lib.celg_elm_row_completed(self.ptr), "celg_elm_row_completed")

    def elm_insert_rows(self, first_row, rp, ci, v):
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        _check(lib.celg_elm_insert_rows(self.ptr, int(first_row), rp.size - 1, _host_ptr(rp),
                                        _host_ptr(ci), _host_ptr(v)), "celg_elm_insert_rows")

    def elm_matrix_completed(self):
        _check(lib.celg_elm_matrix_completed(self.ptr), "celg_elm_matrix_completed")

    def elm_doit(self, b, redo=False):
        b = np.ascontiguousarray(b, np.float64)
        ierr, niter, ftol = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        fn = lib.celg_elm_redoit if redo else lib.celg_elm_doit
        st = fn(self.ptr, _host_ptr(b), ctypes.byref(ierr), ctypes.byref(niter), ctypes.byref(ftol))
        _check(st, "celg_elm_doit", allow=(ERR_NOCONV, ERR_BREAKDOWN))
        return ierr.value, niter.value, ftol.value

    def elm_collect_solution(self, n, out=None):
        x = np.zeros(n) if out is None else out
        _check(lib.celg_elm_collect_solution(self.ptr, _host_ptr(x)), "celg_elm_collect_solution")
        return x

    def elm_performance(self):
        ms, it, bpi = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
        _check(lib.celg_elm_performance(self.ptr, ctypes.byref(ms), ctypes.byref(it),
                                        ctypes.byref(bpi)), "celg_elm_performance")
        return ms.value, it.value, bpi.value

    def elm_destroy(self):
        _check(lib.celg_elm_destroy(self.ptr), "celg_elm_destroy")
