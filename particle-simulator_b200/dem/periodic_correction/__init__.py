from .comsol_lattice_correction import COMSOLLatticeCorrection

__all__ = ["COMSOLLatticeCorrection"]
