"""voxelg_b200 -- B200-native voxel ray traversal for voxelG.

The product is libvoxrt.so (include/voxrt.h): hand-written sm_100a CUDA
kernels behind a C ABI.  This package is the Python host side over that ABI.
"""
from . import _lib
from .configs import CONFIGS, WorldConfig
from .trace import (KIND_ANY, KIND_NO_WATER, KIND_TRACE, PickHit, camera_from_pose,
                    default_camera, default_params, project_dirty, raycast, raycast_batch,
                    render_ao,
                    records, render_host_wait, render_primary, render_primary_gated,
                    render_primary_host, render_primary_host_async,
                    render_primary_host_packed, render_primary_host_packed_async,
                    render_primary_host_compact, render_primary_host_compact_async,
                    unpack_compact_records,
                    render_primary_rows, render_primary_timed, render_stats, shadows,
                    tile_mask_words, tile_refresh, trace, unpack_records)
from .world import DeviceWorld, HostWorld, TerrainParams, dims_counts, empty_arrays

__all__ = [
    "CONFIGS", "WorldConfig", "DeviceWorld", "HostWorld", "TerrainParams", "PickHit",
    "KIND_TRACE", "KIND_ANY", "KIND_NO_WATER", "camera_from_pose", "default_camera",
    "default_params", "raycast", "raycast_batch", "records", "render_ao", "render_primary",
    "render_primary_host", "render_primary_host_async", "render_host_wait", "render_primary_rows",
    "render_primary_host_packed", "render_primary_host_packed_async", "unpack_records",
    "render_primary_host_compact", "render_primary_host_compact_async",
    "unpack_compact_records",
    "render_primary_timed", "render_stats", "shadows", "trace",
    "dims_counts", "empty_arrays", "project_dirty", "render_primary_gated", "tile_mask_words",
    "tile_refresh",
]
