"""psphray_b200: B200-native trace -> deposit -> solve hot path of psphray.

The compute path is libpsg.so (CUDA, sm_100a) behind the C ABI in
include/psg.h; ``psphray_b200.api`` binds it for Python. ``fields`` makes the
seeded synthetic fields and host-generated rays, ``units`` restates the
reference's unit system.
"""
from .units import Units  # noqa: F401
