"""B200-native (sm_100a) CCSD hot path of the eT coupled-cluster program.

``et_b200.ccsd.CCSD`` mirrors eT's CCSD wavefunction entry points over the C ABI
declared in ``include/ccsd_gpu.h`` and implemented in ``libccsd_gpu.so``.
"""

from .ccsd import CCSD, CCSDGPUError, FP64, MIXED, load_library, solve_ground_states  # noqa: F401

__all__ = ["CCSD", "CCSDGPUError", "FP64", "MIXED", "load_library", "solve_ground_states"]
