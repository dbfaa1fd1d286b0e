from .lognormal_droplet_generator import LognormalDropletGenerator, box_side_for_volume_fraction

__all__ = ["LognormalDropletGenerator", "box_side_for_volume_fraction"]
