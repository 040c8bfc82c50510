"""B200-native tight-binding eigensolver for NEMO-3D's hot path.

Hamiltonian assembly, H*x and the Lanczos driver of NEMO-3D, rebuilt as CUDA
kernels for sm_100a behind a C ABI (include/tbgpu.h, libtbgpu.so).  The Python
layer here is a thin ctypes front end (``tbgpu.Hamiltonian``) plus the
material tables and synthetic structure generators.
"""

from . import materials, workloads  # noqa: F401

__all__ = ["materials", "workloads", "Hamiltonian", "TbgpuError", "build"]


def __getattr__(name):
    if name in ("Hamiltonian", "TbgpuError", "prepare_params"):
        from . import tbgpu
        return getattr(tbgpu, name)
    if name == "build":
        from .build import build
        return build
    raise AttributeError(name)
