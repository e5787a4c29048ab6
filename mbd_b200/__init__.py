"""B200-native MBD@rsSCS engine (drop-in for the pmbd.x hot path of 000Justin000/MBD).

The compute path is libmbd_b200.so (CUDA, sm_100a) behind the C ABI of
include/mbd_b200.h; this package holds its ctypes binding (``engine``), the
geometry.in / setting.in readers and report printer (``io``), the seeded
synthetic workloads (``synthetic``) and the in-tree build (``build``).
"""
from .io import (Geometry, InputError, Settings, format_report, parse_geometry, parse_settings, tile,  # noqa: F401
                 write_geometry, write_settings)
from .engine import EXPORTED, LIB_PATH, Engine, MbdError, Result, load_library  # noqa: F401
