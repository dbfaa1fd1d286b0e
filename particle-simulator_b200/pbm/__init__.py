"""The parts of the reference's population-balance package that sit on the DEM
hot path: the volume grid and the collision-frequency counts between volume
classes (pbm/collision_frequency of ddkx21/particle-simulator).  The PBM
solver and the DEM-PBM coupling are not part of this package."""

from .volume_grid import VolumeGrid

__all__ = ["VolumeGrid"]
