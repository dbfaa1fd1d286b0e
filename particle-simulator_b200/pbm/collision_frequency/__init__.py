from .direct_collision_freq import DirectCollisionFrequency
from .tree_collision_freq import TreeCollisionFrequency

__all__ = ["DirectCollisionFrequency", "TreeCollisionFrequency"]
