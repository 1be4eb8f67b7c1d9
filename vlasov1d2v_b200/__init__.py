"""B200-native (sm_100a) hot path of a 1D2V discontinuous-Galerkin Vlasov-Poisson solver.

Drop-in for the hot path of crewsdw/Vlasov1D2V: the classes keep the reference's names and call
signatures (``Basis1D``/``Basis3D``, ``Grid1D``/``Grid3D``/``Distribution``, ``Elliptic``,
``DGFlux``, ``Stepper``, ``Reference``), and their hot operators run as hand-written CUDA
kernels in ``libvlasov1d2v.so`` (C ABI: ``include/vlasov1d2v.h``), called through ctypes.
There is no CPU fallback: without the library or a CUDA device the GPU entry points raise.
"""
from . import basis, elliptic, fluxes, grid, reference, timestep  # noqa: F401
from .basis import Basis1D, Basis3D  # noqa: F401
from .elliptic import Elliptic  # noqa: F401
from .fluxes import DGFlux  # noqa: F401
from .grid import Distribution, Grid1D, Grid3D  # noqa: F401
from .reference import Reference  # noqa: F401
from .timestep import Stepper, get_max_speeds  # noqa: F401

__version__ = "0.1.0"
