"""The C-ABI library loads without a GPU and exports every entry point the
public headers declare; argument validation fails loudly without touching a
device."""
import ctypes as C
import os
import re

import pytest

import smina_b200 as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sgh?_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header", ["smina_b200.h", "smina_b200_host.h"])
def test_exports_every_declared_symbol(header):
    lib = sb.load()
    names = declared(header)
    assert len(names) > 5
    for n in names:
        assert hasattr(lib, n), f"{n} declared in {header} but not exported"


def test_no_fallback_when_library_missing(tmp_path):
    with pytest.raises(OSError):
        sb._lib_backup = sb._lib
        sb._lib = None
        try:
            sb.load(str(tmp_path / "nope.so"))
        finally:
            sb._lib = sb._lib_backup


def test_create_rejects_bad_arguments():
    lib = sb.load()
    h = C.c_void_p()
    assert lib.sg_create(0, 7, C.byref(h)) == sb.SG_ERR_ARG
    assert lib.sg_create(-1, 0, C.byref(h)) != sb.SG_OK


def test_host_errors_are_reported():
    with pytest.raises(sb.SminaError) as e:
        sb.Model("ROOT\nENDROOT\n")
    assert "atoms" in str(e.value) or "TORSDOF" in str(e.value)
    with pytest.raises(sb.SminaError):
        sb.Tables("no_such_function")
    with pytest.raises(sb.SminaError):
        sb.Tables("vina", custom_text="1.0 bogus_term(x=1)\n")


@pytest.mark.gpu
def test_device_info_reports_the_engine_device():
    e = sb.Engine(0, sb.PREC_FP32)
    try:
        info = e.device_info()
        assert info["device"] == 0 and info["num_sms"] > 0 and info["smem_optin"] >= 48 * 1024
    finally:
        e.close()
