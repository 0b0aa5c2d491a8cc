"""The C-ABI library: loads, exports exactly what include/avbd.h declares, and
reports errors through status codes (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "avbd.h")).read()
    return sorted(set(re.findall(r"AVBD_API\s+(?:int|const char\*)\s+(avbd_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from avbd_b200 import build
    build.build()
    from avbd_b200 import _lib
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    decl = declared_symbols()
    assert len(decl) >= 30
    for name in decl:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "avbd_b200", "libavbd_b200.so")],
                         capture_output=True, text=True).stdout
    exported = sorted(set(l.split()[-1] for l in out.splitlines() if " T avbd_" in l))
    assert exported == decl


def test_binding_table_matches_header():
    from avbd_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_status_codes_without_device(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    rc = lib.avbd_create(C.byref(h), 0, 10, 10, 10, 10, 10)
    assert rc == 10  # AVBD_ERR_NO_DEVICE
    assert b"device" in lib.avbd_last_error_string()
    assert lib.avbd_step(None, 1) == 1  # AVBD_ERR_INVALID_ARG on a null context
    assert lib.avbd_version().startswith(b"avbd-b200")


def test_kernels_are_sm100a(lib):
    """The library carries sm_100a machine code (checked through cuobjdump's
    listing of ELF entries only, no disassembly)."""
    out = subprocess.run(["cuobjdump", "--list-elf", os.path.join(ROOT, "avbd_b200", "libavbd_b200.so")],
                         capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_header_is_plain_c(tmp_path):
    """include/avbd.h is what a cgo / FFI binding includes: it must compile as
    strict C99 on its own."""
    src = tmp_path / "c_abi.c"
    src.write_text('#include "avbd.h"\nint main(void) { return avbd_version() == 0; }\n')
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                           "-I" + os.path.join(ROOT, "include"), "-fsyntax-only", str(src)])


def test_cpp_facade_compiles_and_links(lib, tmp_path):
    """The C++ facade (include/avbd/avbd.hpp) with its test program compiles
    warning-free and links against the library (run by the GPU tests)."""
    lib_dir = os.path.join(ROOT, "avbd_b200")
    subprocess.check_call(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-O2",
                           "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "facade_step.cpp"),
                           "-L" + lib_dir, "-lavbd_b200", "-Wl,-rpath," + lib_dir, "-o", str(tmp_path / "facade_step")])
    assert (tmp_path / "facade_step").exists()
