"""The C ABI library loads and exports every function include/impes_b200.h declares."""
import ctypes
import os
import re

from conftest import REPO


def declared_functions():
    src = open(os.path.join(REPO, "include", "impes_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+|unsigned\s+|long\s+)*\w+\s*\*?\s*(impes_\w+)\s*\(",
                                 src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from impes_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.EXPORTED)


def test_abi_version_and_error_text():
    from impes_b200 import _lib
    assert _lib.lib.impes_abi_version() == 1
    # a null-handle call fails cleanly with a message (no device work)
    st = _lib.lib.impes_amg_num_levels(None, None)
    assert st == _lib.ERR_ARG
    assert b"null" in _lib.lib.impes_last_error()


def test_struct_sizes_match_header_layout():
    from impes_b200 import _lib
    # ctypes layouts follow the C declaration order; sizes are fixed by the ABI
    assert ctypes.sizeof(_lib.KrylovParams) == 32
    assert ctypes.sizeof(_lib.KrylovStats) == 32
    assert ctypes.sizeof(_lib.AmgParams) == 56
