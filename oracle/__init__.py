"""FP64 CPU oracle of the reference MPM step -- test infrastructure only.

Only the tests, the smoke check and the benchmark's CPU-baseline leg may import
this package, as the checker.  The product (icempm_2d_sp_b200) never does.
"""
from .oracle import *  # noqa: F401,F403
