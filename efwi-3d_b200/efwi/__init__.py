"""B200 engine of the EFWI-3D elastic propagation operator.

* :mod:`efwi.engine`    -- :class:`Propagator`, the torch-facing wrapper of
  the C-ABI library ``libefwi.so`` (include/efwi.h).
* :mod:`efwi.config`    -- the reference's para/survey JSON and Shot_*.bin
  formats.
* :mod:`efwi.synthetic` -- seeded problems of the benchmark configurations.

The drop-in modules of the reference's Python API, ``FWI_ops_3d`` and
``fwi_utils``, sit next to this package.
"""
from .engine import Grid, Propagator, Shot  # noqa: F401
from ._lib import CourantError, EfwiError  # noqa: F401

__version__ = "0.1.0"
