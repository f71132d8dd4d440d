"""Algorithmic bytes of the fused kernels, for the roofline in bench.py.

Each entry is (kind, bytes): kind "dense" = bytes per voxel of the grid,
"active" = per voxel of active bricks, "fused" = a function (n, active, bricks)
giving the bytes of one launch.
"""
KERNEL_BYTES = {}
