"""B200-native kernel-polynomial (Chebyshev) path of TBTK.

``tbtk_b200.kpm`` is the host layer over the C ABI (include/tbtkkpm.h,
libtbtkkpm.so); ``tbtk_b200.lattice`` generates seeded tight-binding
models in TBTK's basis order.
"""
from . import lattice  # noqa: F401

__all__ = ["lattice", "kpm"]


def __getattr__(name):
    if name == "kpm":
        import importlib
        kpm = importlib.import_module(__name__ + ".kpm")
        kpm.load_library()
        return kpm
    raise AttributeError(name)
