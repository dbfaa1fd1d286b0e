from .euler_droplet_solver import EulerDropletSolver

__all__ = ["EulerDropletSolver"]
