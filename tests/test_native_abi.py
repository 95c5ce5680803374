"""The C-ABI library builds, loads without a GPU and exports every entry
point declared in include/mam4b.h (no compute calls here)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(mam4b_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from mam4xx_b200 import build
    if not os.path.exists(build.LIB):
        build.build_product()
    return ctypes.CDLL(build.LIB)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("mam4b_create", "mam4b_step", "mam4b_step_slab", "mam4b_step_host",
              "mam4b_destroy", "mam4b_last_status", "mam4b_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_default_config(lib):
    from mam4xx_b200 import native
    assert native.lib().mam4b_abi_version() == 1
    c = native.default_config()
    assert (c.do_cond, c.do_rename, c.do_newnuc, c.do_coag) == (1, 1, 1, 1)
    assert c.gaexch_h2so4_uptake_optaa == 2 and c.n_so4_monolayers_pcage == 8


def test_invalid_arguments_are_rejected_without_a_device(lib):
    from mam4xx_b200 import native
    L = native.lib()
    # a null context is rejected before any CUDA call
    assert L.mam4b_step(None, None, None, 1, 1, 1.0, 0, None) == 1
    assert L.mam4b_step_slab(None, None, None, None, 0, 1, 1, 1.0, 0, None) == 1
    assert L.mam4b_destroy(None) == 1
    h = ctypes.c_void_p()
    bad = native.Config(1, 1, 1, 1, 7, 2, 8)  # optaa must be 1 or 2
    assert L.mam4b_create(ctypes.byref(h), ctypes.byref(bad)) == 1
