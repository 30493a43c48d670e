"""CPU-side checks of the C ABI: the library loads without a GPU and exports
every entry point declared in include/celgpu.h (no compute call is made)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "celgpu.h")
LIB = os.path.join(ROOT, "cel_v3_b200", "libcelgpu.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(celg_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from cel_v3_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for required in ("celg_spmv", "celg_mat_to_jad", "celg_mat_jacobi", "celg_pcg_jacobi",
                     "celg_cg", "celg_gmres_jacobi", "celg_dot", "celg_norm2", "celg_axpy",
                     "celg_xpby", "celg_jacobi_apply", "celg_elm_init", "celg_elm_doit",
                     "celg_elm_collect_solution", "celg_elm_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_without_gpu(lib):
    lib.celg_status_string.restype = ctypes.c_char_p
    assert lib.celg_status_string(0) == b"ok"
    assert b"iteration" in lib.celg_status_string(4)


def test_params_default_without_gpu(lib):
    from cel_v3_b200 import celgpu
    p = celgpu.params()
    assert p.eps_rel == 1e-8 and p.iter_max == 1000 and p.x0_mode == celgpu.X0_ZERO
    assert p.restart == 30 and p.inner_eps_rel == 1e-4


def test_build_is_sm100a():
    from cel_v3_b200 import build
    assert "arch=compute_100a,code=sm_100a" in build.ARCH


def test_null_arguments_return_status_without_gpu():
    """Every entry point that takes a handle, matrix or solver object
    returns a status for NULL arguments (ERR_ARG, or ERR_STATE for the
    ELM-mirroring calls with no assembly in progress) before any CUDA call;
    the destroy calls accept NULL as a no-op."""
    from cel_v3_b200 import celgpu
    scalar = (ctypes.c_int, ctypes.c_long, ctypes.c_size_t, ctypes.c_double, ctypes.c_float,
              ctypes.c_int64)
    no_status = {"celg_params_default", "celg_status_string"}
    seen = 0
    for name in declared_functions():
        if name in no_status:
            continue
        f = getattr(celgpu.lib, name)
        assert f.argtypes is not None, name  # every entry point has a ctypes signature
        args = [t(0) if t in scalar else None for t in f.argtypes]
        st = f(*args)
        if name.endswith("_destroy"):
            assert st == 0, name
        else:
            assert st in (1, 6), (name, st)
        seen += 1
    assert seen >= 60
