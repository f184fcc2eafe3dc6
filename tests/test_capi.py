"""The C-ABI library loads and exports every entry point declared in include/*.h.  CPU only:
no compute calls are made here."""
import ctypes as C
import re
from pathlib import Path

import pytest

from lpmcxx_b200 import _capi

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols() -> set[str]:
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(lpm_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"lpm_ctx_create", "lpm_direct_sum_dev", "lpm_direct_sum_mesh"} <= names


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    assert declared_symbols() <= set(_capi.SIGNATURES)


def test_no_device_is_a_status_not_a_crash():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = _capi.lib().lpm_ctx_create(0, C.byref(h))
    assert rc == _capi.LPM_ERR_NO_DEVICE
    assert b"device" in _capi.lib().lpm_last_error()


def test_null_context_rejected():
    k = _capi.KernelDesc(_capi.LPM_KERNEL_BIOT_SAVART_SPHERE, 0, 1.0, 0.0)
    assert _capi.lib().lpm_direct_sum_dev(None, C.byref(k), 0, None, 0, None, 0, 0, None) == _capi.LPM_ERR_ARG
