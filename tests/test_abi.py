"""The C ABI surface (CPU only: the library loads and answers host-only calls;
nothing here touches a device)."""
import ctypes as C
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "sfb200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(sf_[a-z_0-9]+)\s*\(", text))


def test_header_declares_the_python_table(sf):
    from ncihackaton2023_b200 import _lib
    assert declared_symbols() == set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol(sf):
    lib = C.CDLL(sf.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_host_only_calls(sf):
    from ncihackaton2023_b200 import _lib
    lib = _lib.lib
    assert lib.sf_version() >= 100
    assert lib.sf_status_string(0) == b"ok"
    assert lib.sf_status_string(_lib.SF_ERR_NOT_CONVERGED) == b"not converged"
    assert lib.sf_destroy(None) == _lib.SF_OK
    assert lib.sf_last_error(None) == b"null handle"
    assert lib.sf_apply(None, 0, None, None, None) == _lib.SF_ERR_ARG
    assert lib.sf_cg(None, 0, None, None, 1e-10, 10, None, None, None) == _lib.SF_ERR_ARG
    out = C.c_void_p()
    # invalid arguments are rejected before any device work
    assert lib.sf_create(C.byref(out), 4, 3, 3, None, None, None) == _lib.SF_ERR_UNSUPPORTED
    assert lib.sf_create(C.byref(out), 2, 3, 3, None, None, None) == _lib.SF_ERR_ARG
    assert lib.sf_create(C.byref(out), 3, 11, 3, None, None, None) == _lib.SF_ERR_ARG
    assert lib.sf_create(None, 3, 3, 3, None, None, None) == _lib.SF_ERR_ARG
    assert out.value is None


def test_missing_library_fails_loudly(tmp_path):
    import subprocess
    import sys
    pkg = os.path.join(REPO, "ncihackaton2023.jl_b200")
    dst = tmp_path / "pkgcopy"
    dst.mkdir()
    for f in os.listdir(pkg):
        if f.endswith(".py"):
            (dst / f).write_text(open(os.path.join(pkg, f)).read())
    code = ("import importlib.util,sys;"
            f"s=importlib.util.spec_from_file_location('p', r'{dst}/__init__.py',"
            f"submodule_search_locations=[r'{dst}']);m=importlib.util.module_from_spec(s);"
            "sys.modules['p']=m;s.loader.exec_module(m)")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode != 0 and "ImportError" in r.stderr and "libsfb200.so" in r.stderr


def test_null_handles_are_rejected(sf):
    """Every entry point that takes a handle answers SF_ERR_ARG for a null one,
    without touching a device."""
    from ncihackaton2023_b200 import _lib
    lib = _lib.lib
    ARG = _lib.SF_ERR_ARG
    assert lib.sf_rhs(None, None, None, None) == ARG
    assert lib.sf_set_structured_slab(None, 2, 2, 4, 0, 2, None) == ARG
    assert lib.sf_cgd_start(None, None, None, None, None, None, None, None) == ARG
    assert lib.sf_cgd_init(None, None, 1e-10, None) == ARG
    assert lib.sf_cgd_apply(None, None, None, None, None) == ARG
    assert lib.sf_cgd_update(None, None, None, None, None) == ARG
    assert lib.sf_cgd_direction(None, None, None, None, None, None) == ARG
    assert lib.sf_set_structured(None, 2, 2, 2, None) == ARG
    assert lib.sf_mul_host(None, None, None) == ARG
    assert lib.sf_diagonal(None, 0, None, None) == ARG
    assert lib.sf_autotune(None, 0, None) == ARG
    assert lib.sf_kappa_vjp(None, 0, None, None, None, None) == ARG


def test_scalar_block_layout_matches_the_header(sf):
    """The distributed CG's scalar slots as the header documents them."""
    from ncihackaton2023_b200 import _lib
    text = open(HEADER).read()
    for name in ("SF_CGD_SCALARS", "SF_CGD_RR", "SF_CGD_BB", "SF_CGD_DONE", "SF_CGD_ITERS"):
        m = re.search(r"#define\s+" + name + r"\s+(\d+)", text)
        assert m and int(m.group(1)) == getattr(_lib, name), name
