"""The C ABI library loads on a CPU-only host and exports every function include/*.h declares."""
import glob
import os
import re
import subprocess

import mirage_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(mg_[a-z_0-9]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ("mg_open", "mg_score_batch", "mg_classify", "mg_score_candidates", "mg_server_submit",
              "mg_server_poll", "mg_close", "mg_strerror"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = M.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, missing


def test_dynamic_symbol_table():
    out = subprocess.run(["nm", "-D", "--defined-only", M.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mg_[a-z_0-9]+)$", out, re.M))
    assert declared_functions() <= exported


def test_strerror_and_inval_without_gpu():
    L = M.lib()
    assert L.mg_strerror(0) == b"ok"
    assert L.mg_strerror(-6).startswith(b"read contains")
    import ctypes as C

    h = C.c_void_p()
    assert L.mg_open(None, 31, 0, C.byref(h)) == -8
