"""latticeyangmills_b200 — B200-native (sm_100a) Wilson gradient flow.

The compute path is libymflow.so (CUDA kernels behind the C ABI of
include/ymflow.h); this package is its Python host mirror.
"""
from ._native import EXPORTS, Obs, YmflowError, load  # noqa: F401
from .flow import (Ensemble, GluonField, SuperObs, WilsonFlow, block_group_flow, block_halo_plan,  # noqa: F401
                   block_layout, get_input_list, nccl_unique_id,
                   read_conf, slab_group_flow, slab_halo_plan, slab_partition, su3_exp, tile_option, volume,
                   write_conf, write_flow_obs)

__all__ = ["Ensemble", "GluonField", "SuperObs", "WilsonFlow", "read_conf", "write_conf", "get_input_list",
           "write_flow_obs", "volume", "su3_exp", "YmflowError", "Obs", "load", "EXPORTS", "nccl_unique_id",
           "slab_partition", "slab_group_flow", "slab_halo_plan", "tile_option", "block_layout", "block_halo_plan",
           "block_group_flow"]
