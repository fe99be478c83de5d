"""Convenience imports for the operators (mirror of ``python/ptychoX/ops.py``)."""

from . import *  # noqa: F401,F403
from . import __all__  # noqa: F401
