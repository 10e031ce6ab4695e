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


@pytest.mark.parametrize("lang", ["c99", "c++17"])
def test_header_compiles_for_c_and_cpp_hosts(tmp_path, lang):
    """A non-Python host includes include/firestep.h directly: it must build as
    strict C99 (no C++ types, no default arguments) and as C++17 without
    warnings."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c99" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / ("host.c" if lang == "c99" else "host.cpp")
    src.write_text('#include "firestep.h"\nint main(void) { return fs_version() == 0; }\n')
    cmd = [cc, f"-std={lang}", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
           f"-I{ROOT / 'include'}", str(src)]
    if lang == "c99":
        cmd.insert(2, "-pedantic")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


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


def test_index_division_is_exact():
    """The multiply-high division the kernels use to split flat cell indices
    (fs_index_divide runs the same formula on the host) equals integer
    division: every divisor up to 4096 against edge and random dividends,
    and large divisors against the full 32-bit range."""
    import numpy as np
    from firewebapp_b200 import _lib
    lib = _lib.lib()
    rng = np.random.default_rng(7)
    edge = np.array([0, 1, 2, 3, 2**31 - 1, 2**31, 2**32 - 2, 2**32 - 1], dtype=np.uint64)
    for d in list(range(1, 4097)) + [65535, 65536, 65537, 2**31 - 1, 2**31, 2**32 - 1]:
        x = np.concatenate([edge, rng.integers(0, 2**32, 64, dtype=np.uint64),
                            np.arange(3 * d, dtype=np.uint64)[:256] if d < 4097 else edge])
        x = x.astype(np.uint32)
        q = np.empty_like(x)
        assert lib.fs_index_divide(d, x.size, x.ctypes.data, q.ctypes.data) == 0
        assert np.array_equal(q, x // np.uint32(d)), d
    assert lib.fs_index_divide(0, 1, x.ctypes.data, q.ctypes.data) != 0
