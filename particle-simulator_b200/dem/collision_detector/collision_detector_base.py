class CollisionDetector:
    """Base class of the collision detectors
    (dem/collision_detector/collision_detector_base.py:4-28)."""

    def detect(self, positions, radii, *, L=None, boundary_mode=None):
        raise NotImplementedError
