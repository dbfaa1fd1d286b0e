from .droplet_state import DropletState

__all__ = ["DropletState"]
