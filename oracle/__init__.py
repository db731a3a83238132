"""CPU oracle for the VUMPS/TDVP inner loop of InfiniteMPSAlgorithms.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this package: only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference
legs of ``bench.py`` use it, and only as the checker or the timed CPU
baseline.  See ``oracle/imps_oracle.py`` for the restatement itself and for the
parity-pinning status of each part.
"""
from .imps_oracle import *  # noqa: F401,F403
