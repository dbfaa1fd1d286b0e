from .lognormal_droplet_generator import LognormalDropletGenerator, box_side_for_volume_fraction
from .uniform_droplet_generator import UniformDropletGenerator

__all__ = ["LognormalDropletGenerator", "UniformDropletGenerator", "box_side_for_volume_fraction"]
