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


def test_surrogate_and_mlp_entry_points_validate_arguments_without_a_gpu():
    """Every check below returns before any CUDA call, so the fake (never
    dereferenced) pointers are safe."""
    L = runtime.lib()
    p = 4096                                  # a non-null, 16-byte-aligned stand-in
    # MLP building blocks
    assert L.chemgen_mlp_gemm(None, 1, 1, p, 1, 1, p, 8, 8, 8, 8, 0, None) == 1
    assert L.chemgen_mlp_gemm(p, 1, 1, p, 1, 1, p, 4, 8, 8, 8, 0, None) == 1      # ldc < N
    assert L.chemgen_mlp_gemm(p, 1, 1, p, 1, 1, p, 8, 0, 8, 8, 0, None) == 0      # empty product
    assert L.chemgen_mlp_bias_gelu(None, p, p, 8, 8, 1, None) == 1
    assert L.chemgen_mlp_adam(p, p, p, p, p, 8, None, 0.9, 0.999, 1e-8, 0.0, None) == 1   # no schedule row
    assert L.chemgen_mlp_mse_grad(p, p, p, p, p, None, 8, 8, None) == 1
    # feature / target / decode transforms
    assert L.chemgen_surrogate_features(p, p, p, 8, 53, 55, p, p, p, 0, None) == 1      # din < ns + 3
    assert L.chemgen_surrogate_features(p, p, p, 0, 53, 64, p, p, p, 0, None) == 0      # no points
    assert L.chemgen_surrogate_targets(p, 8, 53, 53, p, p, None) == 1                   # dout < ns + 1
    assert L.chemgen_surrogate_decode(p, 8, 53, 54, p, p, 0, None) == 1                # dout < ns + 2
    # fused inference
    infer = lambda img, ns, ng: L.chemgen_surrogate_infer(img, p, p, p, p, ns, p, p, ng, p, p, 0, 0, None)
    assert infer(None, 53, 8) == 1
    assert infer(p, 62, 8) == 6                                                         # ns beyond the outputs
    assert infer(p, 0, 8) == 6
    assert infer(p + 2, 53, 8) == 5                                                     # image not 16-byte aligned
    assert infer(p, 53, -1) == 1
    assert infer(p, 53, 0) == 0
    assert L.chemgen_surrogate_pack(p, p, p, None, p, None) == 1
    assert L.chemgen_surrogate_pack(p, p, p, p, p + 8, None) == 5
    assert L.chemgen_surrogate_image_elems() == 256 * 128 + 2 * 256 * 256 + 64 * 256
