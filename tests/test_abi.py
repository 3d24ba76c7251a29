"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"SGPU_API\s+[\w\s\*]+?\b(sgpu_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("sgpu_scr_cg_prec", "sgpu_cr_cg_prec", "sgpu_assemble", "sgpu_matrix_pcg"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from ssf_b200 import _lib, build
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding knows every declared symbol too
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_version_string_without_gpu():
    from ssf_b200 import _lib
    assert b"sm_100a" in _lib.lib().sgpu_version()


def test_header_constants_match_the_binding():
    from ssf_b200 import _lib
    src = open(os.path.join(ROOT, "include", "sifelgpu.h")).read()
    m = re.search(r"#define\s+SGPU_NOALLOC_MAX_N\s+(\d+)", src)
    assert m and int(m.group(1)) == _lib.NOALLOC_MAX_N
