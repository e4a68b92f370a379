"""CPU checks of the drop-in boundary: libTensorBLAS.so loads without a GPU,
exports every entry point include/*.h declares, and validates arguments on
the host before touching the device."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tensor-blas_b200", "lib", "libTensorBLAS.so")


def _declared(header):
    """Function names declared with TB_API in a header."""
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"TB_API\s+[\w\s\*]+?\b(\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    assert os.path.exists(LIB), "build first: make -C tensor-blas_b200"
    return ctypes.CDLL(LIB)


@pytest.fixture(scope="module")
def exported():
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    names = set()
    for line in out.splitlines():
        parts = line.split(None, 2)
        if len(parts) == 3 and parts[1] in ("T", "W"):
            names.add(parts[2].split("(")[0])
    return names


def test_c_abi_symbols(lib, exported):
    names = _declared("tb_capi.h")
    assert len(names) >= 10
    for n in names:
        assert n in exported, f"{n} declared in tb_capi.h but not exported"
        getattr(lib, n)  # dlsym


def test_reference_cpp_api_symbols(exported):
    names = _declared("TensorBLAS.h")
    assert {"tc_syrk", "tc_trsm"} <= set(names)
    for n in names:
        assert n in exported, f"{n} declared in TensorBLAS.h but not exported"


def _raw_exports():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {p[2] for p in (line.split() for line in out.splitlines()) if len(p) == 3 and p[1] in ("T", "W")}


def test_full_mangled_signatures_match_compiled_reference():
    """Every public entry point of the reference, compiled from its sources
    (tests/golden/ref_cxx_symbols.txt, recorded by make_ref_symbols.py), is
    exported under exactly the same mangled name, i.e. with the same
    parameter types (a long/int mismatch, as in tc_symm's int ldb, would
    change the name)."""
    want = open(os.path.join(ROOT, "tests", "golden", "ref_cxx_symbols.txt")).read().split()
    assert len(want) == 17
    have = _raw_exports()
    missing = [w for w in want if w not in have]
    assert not missing, f"not exported with the reference's signature: {missing}"


def test_symbol_fixture_is_current():
    """When the reference build is present, the fixture still matches it."""
    import importlib.util

    ref = os.path.join(ROOT, "oracle", "_ref", "libTensorBLAS_ref.so")
    if not os.path.exists(ref) or not os.path.isdir(os.path.join(ROOT, "oracle", "_ref", "cxx_sym")):
        pytest.skip("reference build oracle/_ref not present")
    spec = importlib.util.spec_from_file_location("make_ref_symbols",
                                                  os.path.join(ROOT, "tests", "golden", "make_ref_symbols.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    want = open(os.path.join(ROOT, "tests", "golden", "ref_cxx_symbols.txt")).read().split()
    assert mod.reference_symbols(ROOT) == want


def test_diagnostic_entry_points_without_gpu(lib):
    lib.tb_alloc_count.restype = __import__("ctypes").c_ulonglong
    assert lib.tb_alloc_count() == 0  # nothing allocated without a device
    lib.tb_debug_stall.argtypes = [__import__("ctypes").c_long, __import__("ctypes").c_ulonglong]
    assert lib.tb_debug_stall(-2, 0) == 1  # TB_ERROR_INVALID_VALUE before any device access


def test_no_cuda_driver_link():
    out = subprocess.run(["ldd", LIB], capture_output=True, text=True).stdout
    assert "libcuda.so" not in out and "libcublas" not in out


def test_argument_validation_without_gpu(lib):
    c = ctypes
    lib.tb_ssyrk.argtypes = [c.c_char, c.c_char, c.c_long, c.c_long, c.c_float, c.c_void_p, c.c_long, c.c_float,
                             c.c_void_p, c.c_long, c.c_long, c.c_int]
    lib.tb_strsm.argtypes = [c.c_char, c.c_long, c.c_long, c.c_void_p, c.c_long, c.c_void_p, c.c_long, c.c_long, c.c_int]
    lib.tb_sgemm.argtypes = [c.c_char, c.c_char, c.c_long, c.c_long, c.c_long, c.c_float, c.c_void_p, c.c_long,
                             c.c_void_p, c.c_long, c.c_float, c.c_void_p, c.c_long, c.c_int]
    lib.tb_status_string.restype = c.c_char_p
    INVALID, NOT_SUPPORTED = 1, 5
    assert lib.tb_ssyrk(b"L", b"N", -1, 4, 1.0, None, 4, 0.0, None, 4, 256, 0) == INVALID
    assert lib.tb_ssyrk(b"L", b"X", 4, 4, 1.0, None, 4, 0.0, None, 4, 256, 0) == INVALID
    assert lib.tb_ssyrk(b"L", b"N", 8, 4, 1.0, None, 4, 0.0, None, 8, 256, 0) == INVALID  # lda < n
    assert lib.tb_ssyrk(b"L", b"N", 4, 4, 1.0, None, 4, 0.0, None, 4, 0, 0) == INVALID   # nb <= 0
    assert lib.tb_ssyrk(b"L", b"N", 4, 4, 1.0, None, 4, 0.0, None, 4, 256, 7) == INVALID  # precision
    assert lib.tb_ssyrk(b"X", b"N", 4, 4, 1.0, None, 4, 0.0, None, 4, 256, 0) == INVALID
    assert lib.tb_ssyrk(b"L", b"N", 0, 4, 1.0, None, 1, 0.0, None, 1, 256, 0) == 0       # empty: no-op
    assert lib.tb_strsm(b"X", 4, 4, None, 4, None, 4, 64, 0) == INVALID
    assert lib.tb_strsm(b"L", 4, 4, None, 2, None, 4, 64, 0) == INVALID                # lda < m
    assert lib.tb_strsm(b"R", 0, 4, None, 4, None, 1, 64, 0) == 0                       # empty
    assert lib.tb_sgemm(b"Q", b"N", 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4, 0) == INVALID
    assert lib.tb_sgemm(b"N", b"N", 4, 4, 4, 1.0, None, 2, None, 4, 0.0, None, 4, 0) == INVALID
    assert lib.tb_status_string(4) == b"TB_ERROR_TIMEOUT"


def test_python_frontend_imports(tblas):
    assert tblas.PLAIN == 0 and tblas.SPLIT == 1
    assert callable(tblas.tc_syrk) and callable(tblas.tc_trsm)
