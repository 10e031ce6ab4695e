"""The C-ABI library loads here (no GPU needed to dlopen it) and exports every
entry point that include/firestep.h declares."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    txt = (ROOT / "include" / "firestep.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b(fs_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "fs_species_transport" in names and "fs_dom_solve" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    import ctypes
    from firewebapp_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.fail(f"{_lib.LIB_PATH} is missing: build with `make -C firewebapp_b200/csrc`")
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"symbols declared but not exported: {missing}"
    # every declared symbol also has a binding in the ctypes table
    unbound = [n for n in declared_symbols() if n not in _lib.SIGNATURES]
    assert not unbound, f"declared but not bound in _lib.SIGNATURES: {unbound}"


def test_bindings_resolve():
    from firewebapp_b200 import _lib
    L = _lib.lib()
    assert L.fs_version() == 1
    assert L.fs_edc_scratch_bytes(1 << 20) > 0


def test_ctx_create_rejects_an_invalid_case_without_a_gpu():
    """fs_ctx_create checks the case description before touching the device:
    a grid of zero cells is refused with FS_EARG (1) and a message."""
    import ctypes
    from firewebapp_b200 import _lib
    L = _lib.lib()
    desc = _lib.FsCaseDesc(nx=0, ny=0, nz=0)
    init = _lib.FsInitState()
    h = ctypes.c_void_p()
    assert L.fs_ctx_create(ctypes.byref(desc), ctypes.byref(init), ctypes.byref(h)) == 1
    assert h.value is None
    assert b"invalid case description" in L.fs_last_error()
