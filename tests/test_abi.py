"""The C-ABI library builds, loads without a GPU, and exports exactly what
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

from kratos_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(kr_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    if not os.path.exists(L.LIB_PATH):
        pytest.fail("libkrb200.so not built (python -m kratos_b200.build)")
    lib = ctypes.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert "kr_step" in names and "kr_ctx_create" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_the_header():
    assert declared_functions() <= set(L.SIGNATURES)


def test_config_struct_matches_header_defaults():
    lib = L.lib()
    c = L.kr_cfg()
    lib.kr_cfg_default(ctypes.byref(c))
    assert c.abi_version == L.KR_ABI_VERSION
    assert c.precision == 2 and c.riemann == 0
    assert abs(c.gamma - 1.66667) < 1e-12 and c.cfl == 0.3 and c.dt_expand == 2.0



def test_config_struct_layout_matches_c_compiler(tmp_path):
    """The ctypes mirror of kr_cfg has the C compiler's size and offsets."""
    import subprocess
    fields = [f for f, _ in L.kr_cfg._fields_]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"kratos_b200.h\"\nint main(void){\n"
    src += 'printf("%zu\\n", sizeof(kr_cfg));\n'
    src += "".join('printf("%%zu\\n", offsetof(kr_cfg, %s));\n' % f for f in fields)
    src += "return 0;}\n"
    c = tmp_path / "layout.c"
    c.write_text(src)
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)])
    out = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    assert out[0] == ctypes.sizeof(L.kr_cfg)
    assert out[1:] == [getattr(L.kr_cfg, f).offset for f in fields]


def test_create_rejects_bad_config_without_touching_a_gpu():
    lib = L.lib()
    c = L.kr_cfg()
    lib.kr_cfg_default(ctypes.byref(c))
    c.n[0] = 2                       # too small: validated before any CUDA call
    assert not lib.kr_ctx_create(ctypes.byref(c))
    assert b"n >= 4" in lib.kr_last_error(None)
    lib.kr_cfg_default(ctypes.byref(c))
    c.abi_version = 99
    assert not lib.kr_ctx_create(ctypes.byref(c))
    assert b"ABI" in lib.kr_last_error(None)


def test_noalloc_rejects_bad_config_without_touching_a_gpu():
    """kr_c2p_dt_noalloc checks the ABI version and the block size (each axis
    >= 4 cells, as kr_ctx_create) before any CUDA call."""
    lib = L.lib()
    c = L.kr_cfg()
    lib.kr_cfg_default(ctypes.byref(c))
    c.mhd = 1
    c.n[0], c.n[1], c.n[2] = 8, 8, 1                  # a one-cell axis
    dummy = ctypes.c_void_p(16)
    rc = lib.kr_c2p_dt_noalloc(ctypes.byref(c), dummy, dummy, dummy, dummy, None)
    assert rc == -1 and b"n >= 4" in lib.kr_last_error(None)
    lib.kr_cfg_default(ctypes.byref(c))
    c.n[0] = c.n[1] = c.n[2] = 8
    c.abi_version = L.KR_ABI_VERSION - 1
    rc = lib.kr_c2p_dt_noalloc(ctypes.byref(c), dummy, dummy, dummy, dummy, None)
    assert rc == -1 and b"ABI" in lib.kr_last_error(None)
