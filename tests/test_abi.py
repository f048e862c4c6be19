"""The C ABI without a GPU: libcucholesky.so loads, exports every entry point that
include/lapack.h declares, and the argument checks that run before any device
work behave like the reference's (lapack/dpotrf.c:173-179)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import pytest

import cucholesky

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols() -> set[str]:
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*(?:CUresult|void|int)\s+(cu\w+)\s*\(", text, flags=re.M))
        names |= set(re.findall(r"^\s*extern\s+\w+\s+(\w+)\s*;", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = cucholesky.lib()
    declared = _declared_symbols()
    assert len(declared) >= 26
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", cucholesky.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert declared <= exported, sorted(declared - exported)
    assert set(cucholesky.exported_symbols()) <= exported


@pytest.mark.parametrize("p", list("SDCZ"))
def test_argument_error_lda(p):
    """lda < n: *info = -4 (-5 for trtri), XERBLA called with the position, and
    CUDA_ERROR_INVALID_VALUE returned, before the handle is touched."""
    lib = cucholesky.lib()
    calls = []
    XERBLA = C.CFUNCTYPE(None, C.c_char_p, C.c_long)

    def hook(name, info):
        calls.append((name.decode(), info))

    cb = XERBLA(hook)
    xer = C.c_void_p.in_dll(lib, "xerbla")
    old = xer.value
    xer.value = C.cast(cb, C.c_void_p).value
    try:
        for name, pos in (("potrf", 4), ("lauum", 4), ("potri", 4)):
            info = C.c_long(0)
            rc = getattr(lib, f"cu{p}{name}")(None, ord("L"), 10, 0, 5, C.byref(info))
            assert rc == cucholesky.CUDA_ERROR_INVALID_VALUE
            assert info.value == -pos
            assert calls[-1] == (f"cu{p}{name}", pos)
        info = C.c_long(0)
        rc = getattr(lib, f"cu{p}trtri")(None, ord("U"), ord("N"), 10, 0, 5, C.byref(info))
        assert rc == cucholesky.CUDA_ERROR_INVALID_VALUE and info.value == -5
        assert calls[-1] == (f"cu{p}trtri", 5)
    finally:
        xer.value = old


@pytest.mark.parametrize("p", list("SDCZ"))
def test_empty_matrix_is_success(p):
    lib = cucholesky.lib()
    for name in ("potrf", "lauum", "potri"):
        info = C.c_long(123)
        assert getattr(lib, f"cu{p}{name}")(None, ord("L"), 0, 0, 0, C.byref(info)) == 0
        assert info.value == 0
    out = (C.c_float if p in "SC" else C.c_double)(5.0)
    assert getattr(lib, f"cu{p}logdet")(None, 0, 1, 0, C.byref(out), None) == 0
    assert out.value == 0.0


def test_binding_fails_loudly_without_library(tmp_path, monkeypatch):
    monkeypatch.setattr(cucholesky, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(cucholesky, "_lib", None)
    with pytest.raises(FileNotFoundError):
        cucholesky.lib()


def test_extension_argument_errors():
    """Argument checks of the additions run before any device work: XERBLA gets the
    position and CUDA_ERROR_INVALID_VALUE comes back (no handle needed)."""
    lib = cucholesky.lib()
    calls = []
    XERBLA = C.CFUNCTYPE(None, C.c_char_p, C.c_long)

    def hook(name, info):
        calls.append((name.decode(), info))

    cb = XERBLA(hook)
    xer = C.c_void_p.in_dll(lib, "xerbla")
    old = xer.value
    xer.value = C.cast(cb, C.c_void_p).value
    try:
        f = lib.cuDpotrs
        f.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_uint64, C.c_size_t, C.c_uint64, C.c_size_t,
                      C.POINTER(C.c_long)]
        info = C.c_long(0)
        assert f(None, ord("L"), 10, 1, 0, 10, 0, 5, C.byref(info)) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert info.value == -8 and calls[-1] == ("cuDpotrs", 8)
        g = lib.cuDcholMixedCreate
        g.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.c_int,
                      C.c_double, C.POINTER(C.c_long)]
        plan = C.c_void_p()
        assert g(C.byref(plan), None, ord("L"), 10, 0, 10, 3, -1.0, C.byref(info)) == \
            cucholesky.CUDA_ERROR_INVALID_VALUE
        assert info.value == -7 and calls[-1] == ("cuDcholMixedCreate", 7)
        assert g(C.byref(plan), None, ord("L"), 10, 0, 9, 1, -1.0, C.byref(info)) == \
            cucholesky.CUDA_ERROR_INVALID_VALUE
        assert info.value == -6
        k = lib.cuSsyrkLowp
        k.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_float, C.c_uint64, C.c_size_t, C.c_uint64,
                      C.c_size_t, C.c_void_p]
        assert k(None, 1, 16, 16, -1.0, 0, 12, 0, 16, None) == cucholesky.CUDA_ERROR_INVALID_VALUE   # 24 bytes
        assert calls[-1] == ("cuSsyrkLowp", 7)
        assert k(None, 2, 16, 16, -1.0, 0, 16, 0, 18, None) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert calls[-1] == ("cuSsyrkLowp", 9)
        assert k(None, 5, 16, 16, -1.0, 0, 16, 0, 16, None) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert calls[-1] == ("cuSsyrkLowp", 2)
        z = lib.cuDpotrfOzaki
        z.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.c_int, C.POINTER(C.c_long)]
        assert z(None, ord("L"), 10, 0, 10, 9, C.byref(info)) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert info.value == -6 and calls[-1] == ("cuDpotrfOzaki", 6)
        assert z(None, ord("L"), 10, 0, 5, 8, C.byref(info)) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert info.value == -5
    finally:
        xer.value = old


@pytest.mark.parametrize("p", list("SDCZ"))
def test_host_memory_argument_errors(p):
    """cuMultiGPU?potrf/?lauum/?potri check lda first (info -4, XERBLA position 4),
    ?trtri at position 5 (lapack/dpotrf.c:302-308, lapack/dtrtri.c:475-481); n = 0
    succeeds; a NULL handle or matrix is CUDA_ERROR_INVALID_VALUE.  No GPU touched."""
    lib = cucholesky.lib()
    calls = []
    XERBLA = C.CFUNCTYPE(None, C.c_char_p, C.c_long)

    def hook(name, info):
        calls.append((name.decode(), info))

    cb = XERBLA(hook)
    xer = C.c_void_p.in_dll(lib, "xerbla")
    old = xer.value
    xer.value = C.cast(cb, C.c_void_p).value
    try:
        for name, pos in (("potrf", 4), ("lauum", 4), ("potri", 4), ("trtri", 5)):
            rc, info = cucholesky.call_host(None, p, name, "L", 10, 0, 5)
            assert rc == cucholesky.CUDA_ERROR_INVALID_VALUE and info == -pos
            assert calls[-1] == (f"cuMultiGPU{p}{name}", pos)
            assert cucholesky.call_host(None, p, name, "U", 0, 0, 0) == (0, 0)
            n_calls = len(calls)
            rc, info = cucholesky.call_host(None, p, name, "L", 10, 0, 10)
            assert rc == cucholesky.CUDA_ERROR_INVALID_VALUE and info == 0
            assert len(calls) == n_calls
    finally:
        xer.value = old


def test_device_list_argument_errors():
    lib = cucholesky.lib()
    cucholesky._declare_host(lib)
    m = C.c_void_p()
    assert lib.cuMultiGPUCreate(None, None, 1) == cucholesky.CUDA_ERROR_INVALID_VALUE
    devs = (C.c_int * 1)(0)
    assert lib.cuMultiGPUCreate(C.byref(m), devs, 0) == cucholesky.CUDA_ERROR_INVALID_VALUE
    assert lib.cuMultiGPUGetContextCount(None) == 0
    assert lib.cuMultiGPUDestroy(None) == cucholesky.CUDA_ERROR_INVALID_VALUE
    assert lib.cuMultiGPUSynchronize(None) == cucholesky.CUDA_ERROR_INVALID_VALUE
    hh = C.c_void_p()
    assert lib.cuMultiGPULAPACKCreate(C.byref(hh), None) == cucholesky.CUDA_ERROR_INVALID_VALUE
    assert lib.cuMultiGPULAPACKDestroy(None) == cucholesky.CUDA_ERROR_INVALID_VALUE
    assert lib.cuMultiGPULAPACKSynchronize(None) == cucholesky.CUDA_ERROR_INVALID_VALUE


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_headers_compile(tmp_path, lang):
    """include/*.h are drop-in C99 and C++ headers (the reference's are C)."""
    import shutil
    cc_ = shutil.which("gcc" if lang == "c" else "g++")
    cuda_inc = "/usr/local/cuda/include"
    if cc_ is None or not os.path.exists(os.path.join(cuda_inc, "cuda.h")):
        pytest.skip("no host compiler or CUDA headers")
    src = tmp_path / ("h.c" if lang == "c" else "h.cpp")
    src.write_text('#include "lapack.h"\n#include "cucholesky_ext.h"\n#include "cumultigpu.h"\n'
                   "int main(void) { CUmultiGPULAPACKhandle h = 0; (void)h; return (int)CBlasLower - 'L'; }\n")
    std = ["-std=c99"] if lang == "c" else ["-std=c++17"]
    r = subprocess.run([cc_, *std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                        "-c", str(src), "-o", str(tmp_path / "h.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_rng_and_latmc_argument_errors():
    """cu?latmc checks n (position 2), c (3) and lda (5) before any device work; an
    unknown generator type or a NULL generator is CUDA_ERROR_INVALID_VALUE."""
    lib = cucholesky.lib()
    calls = []
    XERBLA = C.CFUNCTYPE(None, C.c_char_p, C.c_long)

    def hook(name, info):
        calls.append((name.decode(), info))

    cb = XERBLA(hook)
    xer = C.c_void_p.in_dll(lib, "xerbla")
    old = xer.value
    xer.value = C.cast(cb, C.c_void_p).value
    try:
        for p in "SDCZ":
            for (n, c, lda), pos in (((1, 10.0, 1), 2), ((10, 0.5, 10), 3), ((10, 10.0, 9), 5)):
                assert cucholesky.call_latmc(p, None, n, c, 0, lda) == cucholesky.CUDA_ERROR_INVALID_VALUE
                assert calls[-1] == (f"cu{p}latmc", pos)
            n_calls = len(calls)
            assert cucholesky.call_latmc(p, None, 10, 10.0, 0, 10) == cucholesky.CUDA_ERROR_INVALID_VALUE
            assert len(calls) == n_calls
    finally:
        xer.value = old
    for b in ("32", "64"):
        f = getattr(lib, f"cuRng{b}Create")
        f.argtypes = [C.POINTER(C.c_void_p), C.c_void_p]
        g = C.c_void_p()
        assert f(C.byref(g), None) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert f(None, C.c_void_p.in_dll(lib, f"philox{b}_t")) == cucholesky.CUDA_ERROR_INVALID_VALUE
        d = getattr(lib, f"cuRng{b}Destroy")
        d.argtypes = [C.c_void_p]
        assert d(None) == cucholesky.CUDA_ERROR_INVALID_VALUE


def test_tuning_table_file(tmp_path):
    """The tuning table: built-in FP64 rows; a file in the tuner's format replaces
    them; a malformed file or an unknown version is refused and changes nothing."""
    import importlib
    lib = cucholesky.lib()
    tune = importlib.import_module("cucholesky.tune")
    tune._declare(lib)

    def sub(t, n):
        v = C.c_int(0)
        assert lib.cuLAPACKGetPotrfBlocks(None, t.encode(), n, C.byref(v)) == 0
        return v.value

    assert sub("D", 1000) == 2 and sub("D", 16384) == 5 and sub("D", 65536) == 8 and sub("Z", 65536) == 12
    rows = tune.table_rows("D", {4096: 2, 8192: 3, 16384: 5})
    assert rows == ["potrf D 0 2", "potrf D 5793 3", "potrf D 11585 5"]
    good = tmp_path / "t.tuning"
    good.write_text("cucholesky-tuning 1\n# comment\n" + "\n".join(rows) + "\npotrf S 0 3\n")
    bad_version = tmp_path / "v.tuning"
    bad_version.write_text("cucholesky-tuning 2\npotrf D 0 4\n")
    bad_row = tmp_path / "r.tuning"
    bad_row.write_text("cucholesky-tuning 1\npotrf D 0 99\n")
    bad_type = tmp_path / "o.tuning"
    bad_type.write_text("cucholesky-tuning 1\nozaki Z 0 8\n")
    builtin = [(t, n, sub(t, n)) for t in "SDCZ" for n in (100, 7000, 20000, 70000)]
    try:
        assert lib.cuLAPACKLoadTuning(str(good).encode()) == 0
        assert sub("D", 5000) == 2 and sub("D", 6000) == 3 and sub("D", 100000) == 5
        assert sub("S", 10) == 3 and sub("Z", 10) == 2 and sub("C", 10**6) == 2   # no row: 2
        for f in (bad_version, bad_row, bad_type, tmp_path / "missing.tuning"):
            assert lib.cuLAPACKLoadTuning(str(f).encode()) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert sub("D", 100000) == 5
        assert lib.cuLAPACKGetPotrfBlocks(None, b"Q", 10, C.byref(C.c_int())) == cucholesky.CUDA_ERROR_INVALID_VALUE
        assert lib.cuLAPACKSetPotrfBlocks(None, 3) == cucholesky.CUDA_ERROR_INVALID_VALUE
    finally:
        restore = tmp_path / "builtin.tuning"
        lines = ["cucholesky-tuning 1"]
        lines += ["potrf D 0 2", "potrf D 11585 5", "potrf D 23170 8",
                  "potrf S 0 2", "potrf S 11585 4", "potrf C 0 2", "potrf C 5793 3",
                  "potrf C 11585 6", "potrf Z 0 2", "potrf Z 5793 6", "potrf Z 11585 12", "ozaki D 0 8", "ozaki D 49152 16"]
        restore.write_text("\n".join(lines) + "\n")
        assert lib.cuLAPACKLoadTuning(str(restore).encode()) == 0
    assert [(t, n, sub(t, n)) for t in "SDCZ" for n in (100, 7000, 20000, 70000)] == builtin
