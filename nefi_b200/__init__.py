"""nefi_b200 — B200-native acoustic leapfrog propagator and exact adjoint for NEFI.

Public API:

* :class:`WaveOperatorB200` — FWI operator, drop-in for ``nefi.physics.wave.WaveOperator``.
* :class:`WaveInitialConditionOperatorB200` — photoacoustic operator, drop-in for
  ``nefi.physics.wave.WaveInitialConditionOperator``.
* :func:`time_reversal` — the classical PAT baseline, drop-in for ``nefi.physics.wave.time_reversal``.

The compute path is the in-tree CUDA library ``libnefiwave.so`` (C ABI in
``include/nefi_wave.h``); build it with ``python -m nefi_b200.build``.
"""

from .operators import WaveInitialConditionOperatorB200, WaveOperatorB200
from .reversal import time_reversal

__all__ = ["WaveInitialConditionOperatorB200", "WaveOperatorB200", "time_reversal"]
__version__ = "0.1.0"
