from .droplet_solution import DropletSolution

__all__ = ["DropletSolution"]
