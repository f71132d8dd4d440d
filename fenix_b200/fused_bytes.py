"""Algorithmic bytes of the fused kernels, for the roofline in bench.py.

Compulsory HBM traffic of each kernel at f32 storage (velocity 12 B per voxel),
counting each input and output once and excluding halo re-reads. Each entry is
(kind, bytes per voxel): "dense" counts every voxel of the grid, "active" the
voxels of active bricks, "fused" is a function (n, active, bricks) -> bytes of
one launch.
"""

KERNEL_BYTES = {
    # p 4 + div 4 read, p 4 written
    "fused_sweep": ("dense", 12.0),
    # the same plus the mid-level pressure (one mid value per 8 fine voxels)
    "fused_sweep_prolong": ("dense", 12.5),
    # velocity 12 read; divergence 4, first sweep 4, mid divergence 0.5 written
    "fused_div_first_sweep": ("dense", 20.5),
    # pressure 4 + velocity 12 read, velocity 12 written
    "fused_project": ("dense", 28.0),
    # velocity 12 read, 12 written
    "fused_advect_velocity": ("dense", 24.0),
    # scalars 16 + velocity 12 read, scalars 16 written
    "fused_advect_scalars": ("active", 44.0),
    # scalars 16 read, 16 written
    "fused_combustion": ("active", 32.0),
    # density, temperature, reaction 12 read; velocity 12 read, 12 written
    "fused_buoyancy": ("active", 36.0),
    # velocity 12 read, |w| 4 written
    "fused_vorticity": ("dense", 16.0),
    # velocity 12 + |w| 4 read and velocity 12 written everywhere; scalars 12 read in active bricks
    "fused_confinement": ("fused", lambda n, a, nb: 28.0 * n + 12.0 * a),
}
