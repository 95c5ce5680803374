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
    assert L.mam4b_set_adjoint_checkpoint(None, 4) == 1
    h = ctypes.c_void_p()
    bad = native.Config(1, 1, 1, 1, 7, 2, 8)  # optaa must be 1 or 2
    assert L.mam4b_create(ctypes.byref(h), ctypes.byref(bad)) == 1


def test_tuning_file_round_trip_and_validation(tmp_path):
    """Tuning files are parsed on the host (no CUDA call): the committed one
    (when present) is valid, a written one reads back, and invalid shapes
    or incomplete files are rejected."""
    import json
    from mam4xx_b200 import native
    committed = os.path.join(ROOT, "mam4xx_b200", "mam4b_tuning.json")
    if os.path.exists(committed):
        t, dev = native.tuning_from_json(committed)
        assert dev and t.as_dict() == {k: json.load(open(committed))[k] for k in t.as_dict()}
    d = native.default_tuning().as_dict()
    d.update(pre_regs=168, post_block=64, soa_blocks_per_sm=3, cells_per_thread=2,
             inline_scale=16)
    p = tmp_path / "t.json"
    p.write_text(json.dumps(dict(d, device="NVIDIA B200", chosen_on={"tuned_ms": 1.0})))
    t, dev = native.tuning_from_json(str(p))
    assert t.as_dict() == d and dev == "NVIDIA B200"
    for bad in (dict(d, pre_regs=200), dict(d, size_block=512), dict(d, soa_blocks_per_sm=0),
                dict(d, cells_per_thread=3), dict(d, inline_scale=8),
                {k: v for k, v in d.items() if k != "soa_regs"}):
        p.write_text(json.dumps(bad))
        with pytest.raises(native.MicrophysicsError):
            native.tuning_from_json(str(p))
    with pytest.raises(native.MicrophysicsError):
        native.tuning_from_json(str(tmp_path / "missing.json"))
