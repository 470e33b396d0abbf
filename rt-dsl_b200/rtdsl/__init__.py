"""rtdsl -- B200-native spatial search for rt-dsl (k-NN, range, Barnes-Hut).

All compute runs in librtdsl.so (hand-written sm_100a CUDA behind the C ABI
of include/rtdsl.h); this package binds it with ctypes and mirrors the
reference's k_nn! / range_query! / barnes_hut! interface.
"""
from ._capi import (BH_LAW_PLUMMER, BH_LAW_REFERENCE, EMPTY_ID, RADIUS_FIXED,
                    RADIUS_MORTON_WINDOW, RADIUS_SAMPLED_MAX, RADIUS_SAMPLED_NN, RADIUS_SAMPLED_PERCENTILE, BhParams,
                    RtdError, Schedule, default_batch_schedule, default_bh_params,
                    default_schedule, load)
from .api import (Context, Index, KnnGraph, KnnHostGraph, dbscan, k_nn, k_nn_array, knn_backward, range_query,
                  spatial_join)
from .batch import Batch
from .bh import BarnesHut, barnes_hut

__all__ = [
    "BH_LAW_PLUMMER", "BH_LAW_REFERENCE", "EMPTY_ID", "RADIUS_FIXED", "RADIUS_MORTON_WINDOW",
    "RADIUS_SAMPLED_MAX",
    "RADIUS_SAMPLED_NN", "RADIUS_SAMPLED_PERCENTILE", "BhParams", "RtdError", "Schedule",
    "default_batch_schedule", "default_bh_params", "default_schedule", "load", "Context", "Index", "KnnGraph", "KnnHostGraph", "k_nn", "k_nn_array",
    "knn_backward", "range_query", "spatial_join", "dbscan", "Batch", "BarnesHut", "barnes_hut",
]
