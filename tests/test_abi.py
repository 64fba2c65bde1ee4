"""The C-ABI library loads and exports every entry point that
include/kaos_gpu.h declares (no compute: runs without a GPU)."""
import os
import re

import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import lib as klib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "kaos_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kaos_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    kbuild.build()
    return klib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_export_list_matches_header():
    assert sorted(klib.EXPORTS) == declared_symbols()


def test_fortran_module_binds_every_symbol():
    """The bind(C) module a Fortran host uses names every entry point."""
    src = open(os.path.join(ROOT, "kaos_b200", "fortran", "kaos_gpu_iface.f90")).read()
    bound = sorted(set(re.findall(r'bind\(C,\s*name\s*=\s*"(kaos_[a-z_0-9]+)"', src)))
    assert bound == declared_symbols()


def test_version_and_null_handle(lib):
    assert b"sm_100a" in lib.kaos_version()
    assert lib.kaos_last_error(None) == b"null handle"
    # null arguments are rejected before any device work
    assert lib.kaos_create(None, None, 0, None, None) == 1
    assert lib.kaos_step(None, 1) == 1
