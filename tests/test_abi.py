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


def _c_prototypes():
    """name -> number of parameters, for every function include/chemgen_b200.h declares."""
    text = open(os.path.join(REPO, "include", "chemgen_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"([a-zA-Z_][a-zA-Z0-9_]*)\s*\(([^()]*)\)\s*;", text):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    return out


def test_fortran_module_binds_exported_symbols_with_matching_arity():
    """include/chemgen_m.F90 (no Fortran compiler in this image): every
    bind(C) interface names a symbol the library exports and the header
    declares, with the header's number of arguments; the public names are
    the reference module's (chemgen/templates/chemgen_mod.j2:22-23)."""
    text = open(os.path.join(REPO, "include", "chemgen_m.F90")).read()
    protos = _c_prototypes()
    L = runtime.lib()
    binds = re.findall(r"(?:subroutine|function)\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", text)
    assert len(binds) >= 9
    for fname, args, cname in binds:
        assert fname == cname
        assert hasattr(L, cname), cname
        nargs = 0 if not args.strip() else len(args.split(","))
        assert protos.get(cname) == nargs, (cname, nargs, protos.get(cname))
    assert {f"getrates_hip_wrapper_v{v}" for v in (1, 2, 3, 4)} <= {c for _, _, c in binds}
    assert re.search(r"public\s*::\s*init_chemgen", text) and re.search(r"public\s*::\s*getrates_gpu", text)
    assert re.search(r"subroutine init_chemgen\(flag, ng\)", text)
    assert re.search(r"subroutine getrates_gpu\(P, T, ng, Y, wdot\)", text)


def test_process_wide_entry_points_fail_cleanly_without_a_mechanism(tmp_path):
    L = runtime.lib()
    assert L.chemgen_global_num_species() == -1
    L.allocate_intermediate_DeviceMemory(16)
    assert L.chemgen_last_wrapper_status() == 8
    assert L.chemgen_init_constants_file(str(tmp_path / "missing.blob").encode()) == 1
    (tmp_path / "empty.blob").write_bytes(b"")
    assert L.chemgen_init_constants_file(str(tmp_path / "empty.blob").encode()) == 1
    for v in (1, 2, 3, 4):
        getattr(L, f"getrates_hip_wrapper_v{v}")(0, 0, 1, 0, 0, 0, 0)
        assert L.chemgen_last_wrapper_status() == 8
