"""CPU oracle for the hysteresis hot path (test infrastructure, not product code).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference
arm import this package, and only to check or time against it.  The product path
(``mammos_mumag`` over ``libmumag_b200.so``) never routes through it.
"""

from .mumag_oracle import *  # noqa: F401,F403
