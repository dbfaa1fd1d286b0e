from .droplet_ensemble import DropletEnsemble, stokes_factor

__all__ = ["DropletEnsemble", "stokes_factor"]
