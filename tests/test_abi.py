"""CPU-side checks of the C ABI: the library builds, loads, and exports every
function include/*.h declares; host-side argument checking needs no GPU."""
import ctypes
import os
import re

import pytest

from conftest import REPO
from chemgen_b200 import runtime


def declared_functions():
    names = set()
    for h in ("chemgen_b200.h", "chemgen_b200_probe.h"):
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("typedef"))
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s+\*?([a-z_][a-z0-9_]*)\s*\(", text,
                             flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = runtime.lib()
    names = declared_functions()
    assert "chemgen_getrates" in names and "getrates_hip_wrapper_v1" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    assert "sm_100a" in runtime.version()
    for s in range(9):
        assert runtime.lib().chemgen_status_string(s).decode() != "unknown status"


def test_create_rejects_bad_blob_without_touching_a_gpu():
    h = ctypes.c_void_p()
    assert runtime.lib().chemgen_create(b"not a mechanism", 15, 0, ctypes.byref(h)) == 2
    assert runtime.lib().chemgen_create(None, 0, 0, ctypes.byref(h)) == 1


def test_null_handle_calls_fail_cleanly():
    L = runtime.lib()
    assert L.chemgen_getrates(None, None, None, 10, None, None, None) == 1
    assert L.chemgen_getrates_host(None, 0, None, None, 10, None, None) == 1
    assert L.chemgen_num_species(None) == -1
