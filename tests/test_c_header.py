"""The C ABI from C: include/celgpu.h compiles as strict C99 (no C++ or CUDA
types leak into it) and a C program links every declared entry point from
libcelgpu.so and runs the calls that need no GPU."""
import os
import shutil
import subprocess

import pytest

from tests.test_lib_cpu import HEADER, LIB, ROOT, declared_functions


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")
def test_c99_program_links_every_entry_point(tmp_path):
    if not os.path.exists(LIB):
        from cel_v3_b200 import build
        build.build()
    names = declared_functions()
    src = ['#include <stdio.h>', '#include "celgpu.h"', "typedef void (*fn_t)(void);",
           "int main(void) {", "  const fn_t fns[] = {"]
    src += ["    (fn_t)&%s," % n for n in names]
    src += ["  };",
            "  size_t k, linked = 0;",
            "  celg_params p;",
            "  for (k = 0; k < sizeof(fns) / sizeof(fns[0]); ++k) linked += fns[k] != NULL;",
            "  celg_params_default(&p);",
            '  printf("%lu %s %d %g %d\\n", (unsigned long)linked, celg_status_string(CELG_OK),',
            "         p.iter_max, p.eps_rel, celg_create(NULL, 0, NULL));",
            "  return 0;", "}"]
    c_file = tmp_path / "abi.c"
    c_file.write_text("\n".join(src) + "\n")
    exe = tmp_path / "abi"
    lib_dir = os.path.dirname(LIB)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                         "-I", os.path.dirname(HEADER), str(c_file), "-L", lib_dir, "-lcelgpu",
                         "-Wl,-rpath," + lib_dir, "-o", str(exe)],
                        capture_output=True, text=True, cwd=ROOT)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    linked, ok, iter_max, eps_rel, create_null = run.stdout.split()
    assert int(linked) == len(names)
    assert ok == "ok" and int(iter_max) == 1000 and float(eps_rel) == 1e-8
    assert int(create_null) == 1  # CELG_ERR_ARG before any CUDA call
