"""Host-side binding of the B200 phase-field step (C-ABI in include/rs_b200.h)."""
from ._abi import *  # noqa: F401,F403
from . import configs  # noqa: F401
