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


def test_charge_exchange_tube_limit(lib):
    """With charge exchange on, more than KAOS_MAX_TUBES_CX tubes are
    rejected before any device work (the ENA push keeps a per-tube prefix in
    shared memory)."""
    import ctypes as C
    from kaos_b200.model_input import KaosTube, KaosVGrid, ModelInput
    src = open(os.path.join(ROOT, "include", "kaos_gpu.h")).read()
    limit = int(re.search(r"#define KAOS_MAX_TUBES_CX (\d+)", src).group(1))
    p = ModelInput(QEXCHANGEflag=1).to_c()
    tube, vg, out = KaosTube(), KaosVGrid(), C.c_void_p()
    rc = lib.kaos_create(C.byref(p), C.byref(tube), limit + 1, C.byref(vg), C.byref(out))
    assert rc == 1 and not out.value


def test_unknown_precision_mode_rejected(lib):
    """A precision mode other than KAOS_PREC_FP64, KAOS_PREC_MIXED and
    KAOS_PREC_MIXED_K64 is rejected before any device work, with a message."""
    import ctypes as C
    from kaos_b200.model_input import (KAOS_PREC_MIXED_K64, KaosTube, KaosVGrid,
                                       ModelInput)
    src = open(os.path.join(ROOT, "include", "kaos_gpu.h")).read()
    assert int(re.search(r"#define KAOS_PREC_MIXED_K64 (\d+)", src).group(1)) == \
        KAOS_PREC_MIXED_K64
    p = ModelInput(precision=7).to_c()
    tube, vg, out = KaosTube(), KaosVGrid(), C.c_void_p()
    rc = lib.kaos_create(C.byref(p), C.byref(tube), 1, C.byref(vg), C.byref(out))
    assert rc == 1
    assert b"precision" in lib.kaos_last_error(out)
    lib.kaos_destroy(out)


def test_sample_kinds_match_header():
    """The sampler kinds of kaos_b200.lib equal the header's KAOS_SAMPLE_*."""
    from kaos_b200 import lib as klib
    src = open(os.path.join(ROOT, "include", "kaos_gpu.h")).read()
    kinds = {m.group(1): int(m.group(2))
             for m in re.finditer(r"#define KAOS_SAMPLE_([A-Z0-9]+) (\d+)", src)}
    assert kinds == {"PHILOX": klib.SAMPLE_PHILOX, "GAUSS32": klib.SAMPLE_GAUSS32,
                     "GAUSS64": klib.SAMPLE_GAUSS64, "POISSON": klib.SAMPLE_POISSON,
                     "GAUSS64T": klib.SAMPLE_GAUSS64T}
