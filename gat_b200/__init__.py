"""gat_b200: B200-native trajectory range and EDR top-k queries (GAT's hot paths).

The compute path is libgat_b200.so (hand-written sm_100a CUDA behind the C ABI in
include/gat_b200.h); this package is its Python mirror. Importing it loads the library and
fails loudly when it has not been built (`python -m gat_b200.build`).
"""
from . import _lib  # noqa: F401  (loads libgat_b200.so or raises)
from .api import (FSG, STIG, Context, GatError, Grid, MortonGrid, RangeResult, Server, SystemTest,  # noqa: F401
                  TrajectorySet, edr_pairs)
from .data import BOX, Trajectories  # noqa: F401
