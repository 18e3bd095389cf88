"""The C-ABI library loads and exports every entry point include/gatt_dns.h declares
(no device calls: this runs on machines without a GPU)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gatt_dns.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gatt_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ("gatt_create", "gatt_set_matrices", "gatt_set_bc", "gatt_rhs", "gatt_deriv_dir", "gatt_step",
              "gatt_destroy", "gatt_strerror"):
        assert s in syms


def test_library_exports_every_declared_symbol(cuda_lib):
    import ctypes
    for s in declared_symbols():
        assert hasattr(cuda_lib, s), s
    assert cuda_lib.gatt_strerror(4) == b"flow diverged"


def test_binding_covers_every_declared_symbol():
    from gatt_dns_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_fortran_interface_module_lists_every_symbol():
    src = open(os.path.join(ROOT, "include", "gatt_dns_mod.f90")).read().lower()
    for s in declared_symbols():
        assert "'%s'" % s in src or '"%s"' % s in src, s


def test_create_fails_cleanly_without_a_device(cuda_lib):
    import ctypes
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = cuda_lib.gatt_create(ctypes.byref(h), 8, 8, 8, 1)
    assert rc != 0 and not h.value
