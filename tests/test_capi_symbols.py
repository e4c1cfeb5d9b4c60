"""The C-ABI library loads without a GPU and exports every function include/*.h declares."""
import ctypes
import os
import re

from vfs_b200.build import LIB, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = "\n".join(l for l in src.splitlines() if not l.lstrip().startswith("#"))
        body = src.split('extern "C" {', 1)[-1]
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", body):
            name = m.group(1)
            if name in ("if", "sizeof", "defined", "while", "for", "return"):
                continue
            # a declaration: preceded by a type on the same statement
            names.add(name)
    return names


def test_library_exports_declared_symbols():
    build()
    lib = ctypes.CDLL(LIB)
    names = declared_functions()
    assert "vfs_initialize" in names and "SolveStereo" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_without_gpu():
    build()
    lib = ctypes.CDLL(LIB)
    lib.vfs_status_string.restype = ctypes.c_char_p
    assert lib.vfs_status_string(0) == b"ok"
    assert lib.vfs_status_string(-1) == b"invalid argument"
    lib.vfs_version.restype = ctypes.c_int
    assert lib.vfs_version() >= 100
