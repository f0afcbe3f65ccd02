"""The C-ABI library loads and exports every symbol include/admp_b200.h declares
(no compute calls: this runs without a GPU)."""
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "admp_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(admp_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    from admp_b200 import _lib
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.EXPORTS)


def test_status_strings_and_version():
    from admp_b200 import _lib
    lib = _lib.load()
    assert lib.admp_abi_version() == 1
    assert lib.admp_status_string(0) == b"ok"
    assert b"converged" in lib.admp_status_string(3)
    assert lib.admp_status_string(99) == b"unknown status"


def test_workspace_queries():
    from admp_b200 import _lib
    lib = _lib.load()
    kp, keep = _lib.int3([32, 32, 32])
    a = lib.admp_pme_recip_workspace_size(_lib.F64, 1, kp)
    b = lib.admp_pme_recip_workspace_size(_lib.F32, 1, kp)
    assert a > b > 32 ** 3 * 4
    kp2, keep2 = _lib.int3([32, 32, 32, 17, 19, 23])
    assert lib.admp_pme_recip_workspace_size(_lib.F64, 2, kp2) > a
    assert lib.admp_nblist_workspace_size(1000) > 1000 * 32
    assert lib.admp_qeq_workspace_size(_lib.F64, 3000, 100000, kp, 1) > 3000 * 8 * 6


def test_bad_args_return_status_without_gpu():
    from admp_b200 import _lib
    lib = _lib.load()
    # argument validation happens on the host before any launch
    assert lib.admp_pair_energy(_lib.F64, 7, 1, 10, 5, None, None, None, None, None, 0.3, 14.0, None, None, None,
                                None, None) == _lib.BAD_ARG
    assert b"mode" in lib.admp_last_error_message()
    with pytest.raises(ValueError):
        _lib.check(_lib.BAD_ARG, "x")
    with pytest.raises(AssertionError):
        _lib.check(_lib.CUTOFF, "x")
