from .collision_detector_base import CollisionDetector
from .spatial_hash_collision_detector import SpatialHashCollisionDetector

__all__ = ["CollisionDetector", "SpatialHashCollisionDetector"]
