"""The C-ABI library builds, loads and exports every entry point include/*.h declares
(CPU only: no compute calls)."""
import ctypes as C
import re
from pathlib import Path

import fumeng_b200

ROOT = Path(__file__).resolve().parents[1]


def declared_entry_points():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        src = h.read_text()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(fm_[a-z_0-9]+)\s*\(", src))
    return sorted(names)


def test_library_exports_declared_symbols(fm_lib):
    names = declared_entry_points()
    assert "fm_render" in names and "fm_trace_closest" in names
    lib = C.CDLL(str(fumeng_b200.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_declared_symbols():
    assert set(declared_entry_points()) <= set(fumeng_b200.EXPORTED_SYMBOLS)


def test_errors_without_device(fm_lib):
    import torch
    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    st = fm_lib.fm_ctx_create(0, C.byref(h))
    assert st == fumeng_b200.FM_ERR_NO_DEVICE
    assert not h.value
    assert fm_lib.fm_last_error(None) == b"null context"
