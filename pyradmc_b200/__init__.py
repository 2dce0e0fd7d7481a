"""pyradmc_b200: a B200-native Monte Carlo dose backend for pyRadMC.

``B200Engine`` is a drop-in for pyRadMC's ``WarpEngine(device="cuda:0")``: the
same ``run`` / ``run_dij`` calls, with the transport, scoring, batch statistics
and Dij compaction running as hand-written sm_100a CUDA behind the C-ABI of
``include/pyradmc_b200.h``.
"""

from pyradmc_b200.collimation import CollimatedBeamletSource, CollimatedSource
from pyradmc_b200.engine import B200Engine
from pyradmc_b200.model import (
    AnalyticWaterTables,
    BeamletGridSource,
    CompositeBeamletSource,
    ConcatenatedBeamletSource,
    CylindricalScoringGrid,
    DijResult,
    PackedCrossSections,
    ParallelBeamSource,
    PencilBeamSource,
    ScoringGrid,
    SpectralBeamletSource,
    SpectralBeamSource,
    Spectrum,
    TransmissionMaskBeamletSource,
    TransmissionMaskSource,
    TransportResult,
    VoxelGrid,
    ali_rogers_varian_6mv,
    geometric_edges,
    save_pack,
    uniform_edges,
)

__all__ = [
    "AnalyticWaterTables",
    "B200Engine",
    "BeamletGridSource",
    "CollimatedBeamletSource",
    "CollimatedSource",
    "CompositeBeamletSource",
    "ConcatenatedBeamletSource",
    "CylindricalScoringGrid",
    "DijResult",
    "PackedCrossSections",
    "ParallelBeamSource",
    "PencilBeamSource",
    "ScoringGrid",
    "SpectralBeamSource",
    "SpectralBeamletSource",
    "Spectrum",
    "TransmissionMaskBeamletSource",
    "TransmissionMaskSource",
    "TransportResult",
    "VoxelGrid",
    "ali_rogers_varian_6mv",
    "geometric_edges",
    "save_pack",
    "uniform_edges",
]
