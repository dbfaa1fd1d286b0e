class ForceCalculator:
    """Base class of the force calculators (dem/force_calculator/force_calculator_base.py:1-10)."""

    def calculate(self, positions, radii):
        raise NotImplementedError("calculate must be implemented by a subclass")

    def calculate_forces_and_convection(self, positions, radii):
        raise NotImplementedError("calculate_forces_and_convection must be implemented by a subclass")
