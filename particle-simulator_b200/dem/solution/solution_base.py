class Solution:
    """Base class of the solution containers (dem/solution/solution_base.py)."""

    def __init__(self):
        pass

    def save_step(self, t, positions):
        raise NotImplementedError("save_step must be implemented by a subclass")
