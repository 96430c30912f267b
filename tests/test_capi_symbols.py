"""The C-ABI library loads and exports every symbol include/hippolbm.h declares; failures come
back as error codes with a message (the library never exits the process)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT
from hippolbm_b200 import capi

HEADER = os.path.join(ROOT, "include", "hippolbm.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hlbm_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert set(declared_symbols()) == set(capi.SIGNATURES)


def test_library_exports_all_symbols():
    lib = C.CDLL(capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_strings():
    L = capi.lib()
    assert b"sm_100a" in L.hlbm_version()
    assert isinstance(L.hlbm_last_error(), bytes)


def test_bad_arguments_return_codes_without_a_device():
    L = capi.lib()
    h = C.c_void_p()
    # inconsistent dx (domain_lbm.cpp:81-86) is rejected before any device work
    rc = L.hlbm_domain(capi.ivec([10, 10, 10]), capi.dvec([0, 0, 0]), capi.dvec([1.0, 1.0, 2.0]),
                       capi.ivec([0, 0, 0]), 0, 0, C.byref(h))
    assert rc == -2 and b"Dx" in L.hlbm_last_error()
    assert L.hlbm_domain(None, None, None, None, 0, 0, C.byref(h)) == -1
    assert L.hlbm_step(None, 1) == -1
    assert L.hlbm_collision(None, 3, None) == -1
