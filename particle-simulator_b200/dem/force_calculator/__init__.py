from .direct_droplet_force_calculator import DirectDropletForceCalculator
from .force_calculator_base import ForceCalculator

__all__ = ["DirectDropletForceCalculator", "ForceCalculator"]
