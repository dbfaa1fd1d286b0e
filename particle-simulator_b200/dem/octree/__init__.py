"""Flat Barnes-Hut octree (dem/octree of the reference) on the B200."""

from .flat_tree import FlatOctree, OctreeNode
from .force_tree import TreeDropletForceCalculator
from .morton_tree import MortonTreeForceCalculator

__all__ = ["FlatOctree", "OctreeNode", "TreeDropletForceCalculator", "MortonTreeForceCalculator"]
