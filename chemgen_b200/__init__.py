"""chemgen_b200: Chemgen's getrates hot path (net molar production rates of a
chemical mechanism at many grid points) as CUDA kernels for B200.

    from chemgen_b200 import GpuMechanism, getrates, load_mechanism
    gm = GpuMechanism(load_mechanism("chem.inp", therm="therm.dat"), generated=True)
    wdot = getrates(gm, P, T, Y)               # differentiable, Y [ns, ng] float64 CUDA

The CUDA library (libchemgen_b200.so) is loaded on first use; there is no
CPU fallback.
"""
from .mechanism import Mechanism, load_mechanism  # noqa: F401


def __getattr__(name):
    # torch-dependent parts load lazily, so that the mechanism front end and
    # the generator CLI import without torch or a GPU
    if name in ("GpuMechanism", "ChemgenError"):
        from . import runtime
        return getattr(runtime, name)
    if name in ("getrates", "GetratesFn"):
        from . import autograd
        return getattr(autograd, name)
    raise AttributeError(name)
