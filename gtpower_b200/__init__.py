"""gtpower_b200 — B200 (sm_100a) engine for GTPower's time-based power path.

Public entry points:
    B200Power            the Power-interface mirror over the C ABI (power.py)
    Design, Events       host containers for the design and the event CSR
    CellLibrary          packed Liberty power groups
    windows              splits an event CSR into time windows with context
"""
from .design import CellLibrary, Design, Events, pack_values, unpack_values  # noqa: F401
from .power import B200Power, PowerResult, Results  # noqa: F401
from . import windows  # noqa: F401
