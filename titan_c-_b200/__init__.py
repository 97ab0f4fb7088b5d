"""B200 (sm_100a) implementation of TITAN's explicit finite-volume ideal-MHD
plasma time step on its moving unstructured hexahedral mesh.

The hot path lives in libtitan_b200.so (CUDA kernels + C ABI, include/titan_b200.h);
this package holds its ctypes view (`native`, `plasma`), the synthetic meshes
(`mesh`) and problems (`problems`) of the benchmark configurations, the
learned charge-exchange closure's host side (`closure`), and the build
script (`build`). The directory name is not a Python identifier, so it is
imported with importlib: ``importlib.import_module("titan_c-_b200")``.
"""
from . import closure, mesh, native, problems, shard  # noqa: F401
from .native import FIELDS, NV, TitanError  # noqa: F401
from .plasma import PlasmaStep, chlld  # noqa: F401

__all__ = ["PlasmaStep", "chlld", "closure", "mesh", "problems", "native", "TitanError", "FIELDS", "NV"]
