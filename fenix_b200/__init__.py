"""fenix_b200: a B200 (sm_100a) CUDA implementation of fenix's per-frame
combustion-volume simulation step, behind the reference's simulation API.

The step itself lives in libfenixcuda.so (C ABI in include/fenix_cuda.h); this
package holds the Python host mirror of the reference interface.
"""
from .emitters import (
    BurstEmitter,
    IgniterEmitter,
    ScalarEmitter,
    VelocityEmitter,
    packEmitterSources,
    pack_emitter_sources,
)
from .simulation import (
    CombustionVolumeSimulation,
    createCombustionVolumeSimulation,
    create_combustion_volume_simulation,
    createSimulationQualitySettings,
    defaultSimulationQualitySettings,
)

__all__ = [
    "BurstEmitter",
    "IgniterEmitter",
    "ScalarEmitter",
    "VelocityEmitter",
    "packEmitterSources",
    "pack_emitter_sources",
    "CombustionVolumeSimulation",
    "createCombustionVolumeSimulation",
    "create_combustion_volume_simulation",
    "createSimulationQualitySettings",
    "defaultSimulationQualitySettings",
]
