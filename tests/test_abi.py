"""The C ABI library loads and exports every function include/impes_b200.h declares."""
import ctypes
import os
import re

from conftest import REPO


def declared_functions():
    with open(os.path.join(REPO, "include", "impes_b200.h")) as f:
        src = f.read()
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
    assert ctypes.sizeof(_lib.AmgParams) == 96


STRUCTS = {
    "AmgParams": "impes_amg_params",
    "LevelDesc": "impes_amg_level_desc",
    "KrylovParams": "impes_krylov_params",
    "KrylovStats": "impes_krylov_stats",
    "ModelDesc": "impes_model_desc",
    "WellDesc": "impes_well_desc",
    "WellState": "impes_well_state",
    "SatStats": "impes_sat_stats",
    "Timing": "impes_timing",
    "EnsembleMemberStats": "impes_ensemble_member_stats",
    "AdjointStats": "impes_adjoint_stats",
}


def test_ctypes_layouts_match_the_c_header(tmp_path):
    """Every ctypes structure of the Python binding has the size, field names,
    field offsets and field sizes that a C compiler gives the header's struct."""
    import shutil
    import subprocess
    from impes_b200 import _lib
    gcc = shutil.which("gcc")
    if gcc is None:
        import pytest
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include "impes_b200.h"', "int main(void) {"]
    for py, c in STRUCTS.items():
        lines.append(f'  printf("{py} . %zu %zu\\n", sizeof({c}), (size_t)0);')
        for name, _ in getattr(_lib, py)._fields_:
            lines.append(f'  printf("{py} {name} %zu %zu\\n", sizeof((({c}*)0)->{name}), offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-std=c11", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), str(src),
                    "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = 0
    for line in filter(None, out):
        py, name, size, off = line.split()
        cls = getattr(_lib, py)
        if name == ".":
            assert ctypes.sizeof(cls) == int(size), (py, ctypes.sizeof(cls), size)
        else:
            fld = getattr(cls, name)
            assert (fld.size, fld.offset) == (int(size), int(off)), (py, name, fld.size, fld.offset, size, off)
        seen += 1
    assert seen == sum(1 + len(getattr(_lib, py)._fields_) for py in STRUCTS)
    # and the header declares no field the binding leaves out
    with open(os.path.join(REPO, "include", "impes_b200.h")) as f:
        hdr = f.read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    for py, c in STRUCTS.items():
        body = re.search(r"typedef struct \{([^}]*)\}\s*" + c + r";", hdr).group(1)
        c_fields = []
        for decl in filter(None, (d.strip() for d in body.split(";"))):
            parts = [re.sub(r"\[.*?\]", "", q).strip() for q in decl.split(",")]
            c_fields.append(parts[0].split()[-1])     # "double dx" -> dx
            c_fields += parts[1:]                     # "int nx, ny, nz" -> ny, nz
        assert c_fields == [n for n, _ in getattr(_lib, py)._fields_], (py, c_fields)
