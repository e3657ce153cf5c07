"""CPU checkers for the elastic propagation operator.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py``.  The product path never imports this package.

* :func:`port` -- the FP64 C++ restatement of the reference algorithm
  (``oracle/efwi_oracle.cpp``).
* :func:`ref` -- the reference's own kernel sources compiled for the CPU
  (``oracle/_ref/libefwi_ref.so``), FP32.
"""
from .pyoracle import (  # noqa: F401
    Case,
    build,
    port,
    ref,
    ref_available,
)
