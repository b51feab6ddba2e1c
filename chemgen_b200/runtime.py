"""Python side of the C ABI (include/chemgen_b200.h), through ctypes.

PyTorch provides device memory and streams; every computation is a call into
libchemgen_b200.so.  There is no CPU fallback: when the library is missing or
cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Union

import numpy as np

from .mechanism import Mechanism
from .pack import pack

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchemgen_b200.so")

MODES = {"fp64": 0, "mixed": 1}
STATUS = {0: "ok", 1: "invalid argument", 2: "mechanism blob rejected", 3: "CUDA error",
          4: "out of device memory", 5: "pointer not 8-byte aligned", 6: "mechanism not supported by this path",
          7: "size exceeds a fixed capacity", 8: "no process-wide mechanism installed"}


class ChemgenError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, 'unknown status')} (status {status})")


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m chemgen_b200.build`")
    L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
    vp, i64, sz, ci = ctypes.c_void_p, ctypes.c_int64, ctypes.c_size_t, ctypes.c_int
    L.chemgen_version.restype = ctypes.c_char_p
    L.chemgen_status_string.restype = ctypes.c_char_p
    L.chemgen_status_string.argtypes = [ci]
    L.chemgen_create.argtypes = [vp, sz, ci, ctypes.POINTER(vp)]
    L.chemgen_destroy.argtypes = [vp]
    L.chemgen_num_species.argtypes = [vp]
    L.chemgen_num_reactions.argtypes = [vp]
    L.chemgen_getrates.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    L.chemgen_getrates_ex.argtypes = [vp, ci, vp, vp, i64, vp, vp, vp]
    L.chemgen_getrates_counted.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp]
    L.chemgen_workspace_bytes.argtypes = [vp, ci, i64, ctypes.POINTER(sz)]
    L.chemgen_getrates_ws.argtypes = [vp, ci, vp, vp, i64, vp, vp, vp, sz, vp]
    L.chemgen_getrates_host.argtypes = [vp, ci, vp, vp, i64, vp, vp]
    L.chemgen_init_constants.argtypes = [vp, sz]
    L.chemgen_free_constants.argtypes = []
    for v in (1, 2, 3, 4):
        f = getattr(L, f"getrates_hip_wrapper_v{v}")
        f.argtypes = [vp, vp, ci, vp, vp, vp, vp]
        f.restype = None
    L.allocate_intermediate_DeviceMemory.argtypes = [ci]
    L.allocate_intermediate_DeviceMemory.restype = None
    L.chemgen_init_constants_file.argtypes = [ctypes.c_char_p]
    L.chemgen_global_num_species.argtypes = []
    L.chemgen_last_wrapper_status.argtypes = []
    L.chemgen_probe_math.argtypes = [vp, ci, vp, vp, vp, vp]
    L.chemgen_probe_math.restype = ci
    L.chemgen_probe_umma.argtypes = [vp, vp, vp, ci, ci, vp]
    L.chemgen_probe_umma.restype = ci
    L.chemgen_jacobian.argtypes = [vp, ci, vp, vp, i64, vp, vp, vp]
    L.chemgen_getrates_vjp.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp, vp, vp]
    L.chemgen_getrates_noalloc.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    L.chemgen_getrates_noalloc.restype = ci
    f32 = ctypes.c_float
    L.chemgen_mlp_gemm.argtypes = [vp, i64, i64, vp, i64, i64, vp, i64, ci, ci, ci, ci, vp]
    L.chemgen_mlp_bias_gelu.argtypes = [vp, vp, vp, i64, ci, ci, vp]
    L.chemgen_mlp_gelu_backward.argtypes = [vp, vp, vp, vp, i64, vp]
    L.chemgen_mlp_mse_grad.argtypes = [vp, vp, vp, vp, vp, vp, i64, ci, vp]
    L.chemgen_mlp_colsum.argtypes = [vp, vp, i64, ci, vp]
    L.chemgen_mlp_adam.argtypes = [vp, vp, vp, vp, vp, i64, vp, f32, f32, f32, f32, vp]
    L.chemgen_surrogate_features.argtypes = [vp, vp, vp, i64, ci, ci, vp, vp, vp, vp, vp]
    L.chemgen_surrogate_targets.argtypes = [vp, i64, ci, ci, vp, vp, vp]
    L.chemgen_surrogate_decode.argtypes = [vp, i64, ci, ci, vp, vp, vp, vp]
    L.chemgen_mlp_gemm_tc.argtypes = [vp, i64, vp, i64, ci, ci, ci, ci, vp, vp, i64, vp, i64, vp, i64, vp, i64,
                                      ci, vp]
    L.chemgen_mlp_tc_error.argtypes = [ci]
    L.chemgen_mlp_transpose_bf16.argtypes = [vp, i64, ci, ci, vp, i64, vp]
    L.chemgen_mlp_adam_multi.argtypes = [ci, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, f32, f32, f32, vp]
    L.chemgen_mlp_forward_tc.argtypes = [vp, i64, ci, vp, vp, ci, vp, vp, vp, vp]
    L.chemgen_mlp_backward_tc.argtypes = [vp, vp, vp, ci, vp, vp, vp, vp, vp]
    L.chemgen_mlp_backward_tc_work_bytes.argtypes = [ci]
    L.chemgen_mlp_backward_tc_work_bytes.restype = ctypes.c_size_t
    L.chemgen_surrogate_image_elems.argtypes = []
    L.chemgen_surrogate_pack.argtypes = [vp, vp, vp, vp, vp, vp]
    L.chemgen_surrogate_infer.argtypes = [vp, vp, vp, vp, vp, ci, vp, vp, i64, vp, vp, vp, vp, vp]
    L.chemgen_surrogate_infer_error.argtypes = [ci]
    L.chemgen_gate_select.argtypes = [vp, f32, i64, vp, i64, vp, vp]
    L.chemgen_gate_gather.argtypes = [vp, vp, vp, ci, i64, vp, vp, i64, vp, vp, vp, vp]
    L.chemgen_gate_scatter.argtypes = [vp, ci, i64, vp, vp, vp, i64, vp]
    for f in ("chemgen_gate_select", "chemgen_gate_gather", "chemgen_gate_scatter"):
        getattr(L, f).restype = ci
    for f in ("chemgen_mlp_gemm", "chemgen_mlp_gemm_tc", "chemgen_mlp_tc_error", "chemgen_mlp_transpose_bf16",
              "chemgen_mlp_adam_multi", "chemgen_mlp_forward_tc", "chemgen_mlp_backward_tc",
              "chemgen_mlp_bias_gelu", "chemgen_mlp_gelu_backward", "chemgen_mlp_mse_grad",
              "chemgen_mlp_colsum", "chemgen_mlp_adam", "chemgen_surrogate_features", "chemgen_surrogate_targets",
              "chemgen_surrogate_decode", "chemgen_surrogate_image_elems", "chemgen_surrogate_pack",
              "chemgen_surrogate_infer", "chemgen_surrogate_infer_error"):
        getattr(L, f).restype = ci
    L.chemgen_use_generated.argtypes = [vp, ci]
    L.chemgen_kernel_kind.argtypes = [vp, ci]
    L.chemgen_register_kernels.argtypes = [ctypes.c_uint64, ci, ci, ctypes.c_uint, vp]
    for f in ("chemgen_create", "chemgen_destroy", "chemgen_num_species", "chemgen_num_reactions",
              "chemgen_getrates", "chemgen_getrates_ex", "chemgen_getrates_counted", "chemgen_workspace_bytes",
              "chemgen_getrates_ws",
              "chemgen_getrates_host", "chemgen_init_constants", "chemgen_free_constants",
              "chemgen_init_constants_file", "chemgen_global_num_species",
              "chemgen_last_wrapper_status", "chemgen_use_generated", "chemgen_kernel_kind",
              "chemgen_register_kernels", "chemgen_jacobian", "chemgen_getrates_vjp"):
        getattr(L, f).restype = ci
    _lib = L
    return L


def check(status: int, what: str) -> None:
    if status != 0:
        raise ChemgenError(status, what)


def _ptr(t) -> int:
    if t is None:
        return 0
    if isinstance(t, int):
        return t
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


_loaded_modules = {}


def load_generated(mech: Mechanism, build: bool = True) -> Optional[str]:
    """Load (building first if needed) the kernels generated for `mech`
    (generate_chemistry.py --language cuda); returns the module path or None."""
    from . import emit_cuda
    if mech.ns > emit_cuda.MAX_REG_SPECIES:
        return None
    path = emit_cuda.module_path(mech)
    if path in _loaded_modules:
        return path
    if not os.path.exists(path):
        if not build:
            return None
        emit_cuda.build_module(mech, out=path)
    lib()
    _loaded_modules[path] = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
    return path


class GpuMechanism:
    """A mechanism loaded on one GPU (one chemgen_handle).

    generated=True loads the mechanism-specialised kernels (compiling them on
    first use); generated=False keeps the table-driven kernels."""

    def __init__(self, mech: Union[Mechanism, bytes], device: int = 0, generated: bool = False):
        self.blob = mech if isinstance(mech, (bytes, bytearray)) else pack(mech).to_blob()
        self.mech = None if isinstance(mech, (bytes, bytearray)) else mech
        self.device = device
        if generated:
            if self.mech is None:
                raise ValueError("generated kernels need the Mechanism, not only its blob")
            load_generated(self.mech)
        self._buf = ctypes.create_string_buffer(bytes(self.blob), len(self.blob))
        h = ctypes.c_void_p()
        check(lib().chemgen_create(self._buf, len(self.blob), device, ctypes.byref(h)), "chemgen_create")
        self._h = h
        self.ns = lib().chemgen_num_species(h)
        self.nr = lib().chemgen_num_reactions(h)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().chemgen_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def kernel_kind(self, mode: str = "fp64") -> str:
        k = lib().chemgen_kernel_kind(self._h, MODES[mode])
        return {1: "generated", 0: "table", -1: "unavailable"}[k]

    def use_generated(self, enable: bool) -> None:
        check(lib().chemgen_use_generated(self._h, 1 if enable else 0), "chemgen_use_generated")

    def workspace_bytes(self, ng: int, mode: str = "fp64") -> int:
        out = ctypes.c_size_t()
        check(lib().chemgen_workspace_bytes(self._h, MODES[mode], ng, ctypes.byref(out)), "chemgen_workspace_bytes")
        return out.value

    def getrates_ptr(self, P: int, T: int, ng: int, Y: int, wdot: int, mode: str = "fp64", stream=None) -> None:
        """Raw device pointers (species-major Y/wdot)."""
        check(lib().chemgen_getrates_ex(self._h, MODES[mode], P, T, ng, Y, wdot, _stream(stream)),
              "chemgen_getrates_ex")

    def getrates(self, P, T, Y, out=None, mode: str = "fp64", stream=None, layout: str = "species_major"):
        """torch CUDA float64 tensors: P[ng], T[ng], Y[ns, ng] -> wdot[ns, ng].

        layout="point_major" takes Y as [ng, ns] (per point, species
        contiguous: the reference's Python getrates_i layout) and returns wdot
        the same way; the kernels run on a species-major copy."""
        import torch
        if layout not in ("species_major", "point_major"):
            raise ValueError("layout must be 'species_major' or 'point_major'")
        if layout == "point_major":
            if Y.dim() != 2 or Y.shape[1] != self.ns:
                raise ValueError(f"point-major Y must be [ng, {self.ns}]")
            w = self.getrates(P, T, Y.t().contiguous(), mode=mode, stream=stream)
            w = w.t()
            if out is not None:
                out.copy_(w)
                return out
            return w.contiguous()
        ns, ng = Y.shape
        if ns != self.ns:
            raise ValueError(f"Y has {ns} species, the mechanism {self.ns}")
        for name, t in (("P", P), ("T", T), ("Y", Y)):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError(f"{name} must be a contiguous float64 CUDA tensor")
        if P.numel() != ng or T.numel() != ng:
            raise ValueError("P and T must have ng entries")
        if out is None:
            out = torch.empty_like(Y)
        self.getrates_ptr(P.data_ptr(), T.data_ptr(), ng, Y.data_ptr(), out.data_ptr(), mode, stream)
        return out

    def jacobian(self, P, T, Y, precision: str = "fp64", out=None, stream=None):
        """Dense d wdot / d(T, Y): tensor [ns, ns+1, ng] (column 0 = T)."""
        import torch
        ns, ng = Y.shape
        dt = torch.float64 if precision == "fp64" else torch.float32
        if out is None:
            out = torch.empty((ns, ns + 1, ng), dtype=dt, device=Y.device)
        check(lib().chemgen_jacobian(self._h, 0 if precision == "fp64" else 1, P.data_ptr(), T.data_ptr(), ng,
                                     Y.data_ptr(), out.data_ptr(), _stream(stream)), "chemgen_jacobian")
        return out

    def vjp(self, P, T, Y, G, stream=None):
        """(dL/dT [ng], dL/dY [ns, ng], dL/dP [ng]) for G = dL/dwdot [ns, ng]."""
        import torch
        ns, ng = Y.shape
        gT = torch.empty_like(T)
        gY = torch.empty_like(Y)
        gP = torch.empty_like(P)
        check(lib().chemgen_getrates_vjp(self._h, P.data_ptr(), T.data_ptr(), ng, Y.data_ptr(), G.data_ptr(),
                                         gT.data_ptr(), gY.data_ptr(), gP.data_ptr(), _stream(stream)),
              "chemgen_getrates_vjp")
        return gT, gY, gP

    def getrates_ws(self, P, T, Y, out, workspace, mode: str = "fp64", stream=None):
        ns, ng = Y.shape
        wb = workspace.numel() * workspace.element_size() if workspace is not None else 0
        check(lib().chemgen_getrates_ws(self._h, MODES[mode], P.data_ptr(), T.data_ptr(), ng, Y.data_ptr(),
                                        out.data_ptr(), _ptr(workspace), wb, _stream(stream)),
              "chemgen_getrates_ws")
        return out

    def getrates_host(self, P: np.ndarray, T: np.ndarray, Y: np.ndarray, out: Optional[np.ndarray] = None,
                      mode: str = "fp64") -> np.ndarray:
        """Host (numpy or pinned torch CPU) arrays in, host wdot out."""
        ns, ng = Y.shape
        if out is None:
            out = np.empty((ns, ng))
        check(lib().chemgen_getrates_host(self._h, MODES[mode], _ptr(P), _ptr(T), ng, _ptr(Y), _ptr(out)),
              "chemgen_getrates_host")
        return out


def version() -> str:
    return lib().chemgen_version().decode()
