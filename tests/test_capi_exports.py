"""The C-ABI library loads and exports every function include/tdem.h declares
(no compute call: runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "tdem.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][\w ]*[\s\*]+)([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "sizeof")))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("tdem_run_directory", "tdem_solver_create", "tdem_solver_run", "tdem_solver_results",
              "tdem_solver_info", "tdem_solver_destroy", "pardiso_64", "tdem_pardiso_64"):
        assert n in names


def test_library_exports_every_declared_symbol(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pkg.EXPORTED) <= set(declared_functions())


def test_header_is_plain_c(tmp_path):
    """The boundary header compiles as C99 with warnings as errors (cgo, FFI and C
    callers include it as is)."""
    import shutil
    import subprocess
    import pytest
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "use.c"
    src.write_text('#include "tdem.h"\nint main(void) { return tdem_version() == 0; }\n')
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-c", str(src), "-o", str(tmp_path / "use.o")], check=True)


def test_version_string(pkg):
    lib = pkg.load_library()
    assert b"sm_100a" in lib.tdem_version()


def test_no_gpu_fails_loudly(pkg, tmp_path):
    """Without a usable device or inputs the entry points return an error status;
    there is no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is present")
    try:
        pkg.run_directory(str(tmp_path), "A", 2)
    except pkg.TdemError as e:
        assert e.status in (2, 3)
    else:
        raise AssertionError("run_directory succeeded without a GPU")
