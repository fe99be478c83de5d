"""CPU oracle (test infrastructure only): numpy restatement of PtychoX's operators.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs use it,
as the checker.  The ``ptychox_b200`` product path never imports it.
"""

from .ptycho_oracle import *  # noqa: F401,F403
