"""Algorithmic bytes of the fused kernels, for the roofline in bench.py.

Compulsory HBM traffic of each kernel, counting each input and output once and
excluding halo re-reads. Velocity and pressure are f32 (velocity 12 B per
voxel); a scalar (density, temperature, fuel, reaction) is 4 B at f32 storage
and 2 B at FP16 storage. Each entry is (kind, bytes per voxel): "dense" counts
every voxel of the grid, "active" the voxels of active bricks, "fused" is a
function (n, active, bricks) -> bytes of one launch. The sparse-mode kernels
(sparse_*) run on the bricks flagged in the current or the next set; their bytes
are counted per voxel of the active bricks, which that set is close to.
"""


def kernel_bytes_table(storage: str = "f32") -> dict:
    s = {"f32": 4.0, "f16": 2.0, "f16-nearest": 2.0}[storage]
    return {
        # p 4 + div 4 read, p 4 written
        "fused_sweep": ("dense", 12.0),
        # the same kernel beside the mid and coarse levels, on half the resident blocks
        "fused_sweep_shared": ("dense", 12.0),
        # the same plus the mid-level pressure (one mid value per 8 fine voxels)
        "fused_sweep_prolong": ("dense", 12.5),
        # velocity 12 read; divergence 4, first sweep 4, mid divergence 0.5 written
        "fused_div_first_sweep": ("dense", 20.5),
        # pressure 4 + velocity 12 read, velocity 12 written
        "fused_project": ("dense", 28.0),
        # velocity 12 read, 12 written
        "fused_advect_velocity": ("dense", 24.0),
        # 4 scalars + velocity 12 read, 4 scalars written
        "fused_advect_scalars": ("active", 8.0 * s + 12.0),
        # 4 scalars read, 4 written
        "fused_combustion": ("active", 8.0 * s),
        # density, temperature, reaction read; velocity 12 read, 12 written
        "fused_buoyancy": ("active", 3.0 * s + 24.0),
        # velocity 12 read, |w| 4 written
        "fused_vorticity": ("dense", 16.0),
        # velocity 12 + |w| 4 read and velocity 12 written everywhere; 3 scalars read in active bricks
        "fused_confinement": ("fused", lambda n, a, nb, s=s: 28.0 * n + 3.0 * s * a),
        # sparse mode: the same passes over the active bricks
        "sparse_sweep": ("active", 12.0),
        "sparse_sweep_prolong": ("active", 12.5),
        "sparse_div_first_sweep": ("active", 20.5),
        "sparse_project": ("active", 28.0),
        "sparse_advect_velocity": ("active", 24.0),
        "sparse_vorticity": ("active", 16.0),
        "sparse_confinement": ("active", 28.0 + 3.0 * s),
    }


KERNEL_BYTES = kernel_bytes_table("f32")
