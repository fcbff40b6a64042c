"""B200-native D3Q27 cumulant lattice-Boltzmann time step (drop-in for LBM3's hot path).

The compute path is the in-tree CUDA library ``_lib/liblbm3_b200.so``
(sm_100a), reached through the C ABI in ``include/lbm3_b200.h``.  This
package is the host-side mirror of the reference driver API.
"""
from . import _abi
from ._abi import LbmCase, LbmError, LbmFaceBC, LbmGridInfo, lib
from .cases import (flow_around_sphere, open_channel, periodic_box, set_hooks, set_refine_box, taylor_green,
                    taylor_green_refined, tgv_plain_method)
from .grids import Grids, PackedBatch, Plan, apply_collision_batch, build_grids, update_batch

__all__ = [
    "LbmCase", "LbmError", "LbmFaceBC", "LbmGridInfo", "lib", "Grids", "Plan",
    "build_grids", "update_batch", "PackedBatch", "apply_collision_batch", "taylor_green", "tgv_plain_method",
    "periodic_box", "open_channel", "flow_around_sphere", "_abi", "set_refine_box", "taylor_green_refined",
    "set_hooks",
]
