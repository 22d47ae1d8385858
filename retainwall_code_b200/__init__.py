"""B200-native SPH geomechanics step with the reference's case/API surface.

``LoquatSph`` (the reference's class, src/loquat.h:44-126) runs a case through the
native library ``librw.so`` (hand-written sm_100a kernels behind the C ABI of
include/retainwall.h).  ``cases`` builds and reads/writes the reference's case files.
"""
from .sph import Batch, LoquatSph  # noqa: F401
from ._lib import RwError  # noqa: F401
